// The B200 FFT provider module: C ABI v1 (include/syclfft_b200_provider.h).
//
// Implements the device-provider contract of the reference's cuFFT module
// (src/providers/cufft/cufft_provider.cpp:184-248: supports / create / destroy /
// execute with a 1024-byte error buffer and no exceptions across the boundary) on
// top of the B200 planner and pass kernels. A plan owns its device tables (twiddles,
// chirps, chirp spectra; generated in FP64, stored in the plan precision) and one
// scratch buffer; execute enqueues the plan's passes on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/syclfft_b200_provider.h"
#include "bluestein_init.hpp"
#include "cluster_launch.hpp"
#include "fixed_launch.hpp"
#include "launch.hpp"
#include "lean_launch.hpp"
#include "piped_launch.hpp"
#include "tc_launch.hpp"
#include "tma_launch.hpp"
#include "real_launch.hpp"
#include "layout_launch.hpp"
#include "cluster_pipe.hpp"
#include "bluestein_launch.hpp"
#include "fused4_launch.hpp"
#include "planner.hpp"

namespace sfb {
namespace {

void set_error(char* err, size_t cap, const std::string& msg) {
    // provider_error_buffer.hpp:10-18 semantics: NUL-terminated, truncated to cap-1
    if (!err || cap == 0) return;
    const size_t n = std::min(cap - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

class DeviceGuard {
public:
    explicit DeviceGuard(int device) {
        check(cudaGetDevice(&prev_), "cudaGetDevice");
        if (device >= 0 && device != prev_) {
            check(cudaSetDevice(device), "cudaSetDevice");
            switched_ = true;
        }
    }
    ~DeviceGuard() {
        if (switched_) cudaSetDevice(prev_);
    }

private:
    int prev_ = 0;
    bool switched_ = false;
};

struct BoundPass {
    PassParams p;
    const PassSpec* spec_ptr = nullptr;  // the plan's PassSpec (stable: plan->spec.passes)
    const PassSpec& spec_ref() const { return *spec_ptr; }
    FixedParams fp;    // used when spec.fixed_id >= 0
    ClusterParams cp;  // used when spec.cluster_id >= 0
    PipedParams pp;    // used when spec.piped_id >= 0 and the buffers are 16-byte aligned
    TcParams tp;       // used when spec.tc_id >= 0
    ClusterPipeParams kp;  // used when spec.cluster_pipe and the buffers are 16-byte aligned
    // four-step column pass whose row pass (the next pass) can run with it in one fused launch
    // (fused4_kernel.cuh), or nullptr
    const Fused4Entry* fused4 = nullptr;
    // Bluestein forward column pass whose row and inverse column passes (the next two) can run
    // with it in one fused launch, or nullptr
    const FusedBlueEntry* fusedblue = nullptr;
};

TcParams to_tc(const PassParams& p, const void* tw, int* status) {
    TcParams q;
    q.n_outer = p.n_outer;
    q.n_cols = p.n_cols;
    q.col_tiles = p.col_tiles;
    q.tiles = p.tiles;
    q.in = p.in;
    q.out = p.out;
    q.scale = static_cast<float>(p.scale);
    q.conj_in = p.conj_in;
    q.conj_out = p.conj_out;
    q.tw = tw;
    q.status = status;
    return q;
}

PipedParams to_piped(const PassParams& p, int* status) {
    PipedParams q;
    q.lines = p.n_cols;
    q.in_pitch = p.in.cs;
    q.out_pitch = p.out.cs;
    q.tw = p.fft1.tw;
    q.conj_in = p.conj_in;
    q.conj_out = p.conj_out;
    q.scale = p.scale;
    q.status = status;
    return q;
}

ClusterParams to_cluster(const PassParams& p) {
    ClusterParams c;
    c.lines = p.n_cols;
    c.in_pitch = p.in.cs;
    c.out_pitch = p.out.cs;
    c.tw1 = p.fft1.tw;
    c.tw2 = p.fft2.tw;
    c.tw4_hi = p.tw4_hi;
    c.tw4_lo = p.tw4_lo;
    c.tw4_shift = p.tw4_shift;
    c.conj_in = p.conj_in;
    c.conj_out = p.conj_out;
    c.scale = p.scale;
    return c;
}

FixedParams to_fixed(const PassParams& p) {
    FixedParams f;
    f.n_cols = p.n_cols;
    f.col_tiles = p.col_tiles;
    f.w = p.w;
    f.in_hi = p.in.hi;
    f.out_hi = p.out.hi;
    f.in_pitch = p.in.cs;
    f.out_pitch = p.out.cs;
    f.in_ks = p.in.ks;
    f.out_ks = p.out.ks;
    f.tw = p.fft1.tw;
    f.conj_in = p.conj_in;
    f.conj_out = p.conj_out;
    f.scale = p.scale;
    f.tw4_hi = p.tw4_hi;
    f.tw4_lo = p.tw4_lo;
    f.tw4_shift = p.tw4_shift;
    f.rows = p.ts_rows ? p.ts_rows : (p.sel_mode == kSelColMod ? p.sel_d : 1);
    f.line = p.ts_line;
    auto clamp = [](int64_t v) { return static_cast<int>(std::min<int64_t>(v, INT32_MAX)); };
    f.premul = p.premul;
    f.postmul = p.postmul;
    f.pointwise = p.pointwise;
    f.g_k = clamp(p.g_k);
    f.in_len = clamp(p.in_len);
    f.out_len = clamp(p.out_len);
    f.pw_stride = clamp(p.pw_stride);
    f.conj_mid = p.conj_mid;
    f.flip_in = p.flip_in;
    f.flip_out = p.flip_out;
    f.perm_in = static_cast<const int*>(p.perm_in);
    f.perm_out = static_cast<const int*>(p.perm_out);
    return f;
}

// Per-device stream for plan memory: allocations and frees are stream-ordered
// (cudaMallocAsync / cudaFreeAsync), so releasing a plan never synchronizes the device.
cudaStream_t memory_stream(int device) {
    static std::mutex mu;
    static std::map<int, cudaStream_t> streams;
    std::lock_guard<std::mutex> lock(mu);
    auto it = streams.find(device);
    if (it != streams.end()) return it->second;
    cudaStream_t s = nullptr;
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = uint64_t(4) << 30;  // keep up to 4 GiB of freed plan memory for the next plans
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    streams[device] = s;
    return s;
}

// Status words of plans: 4-byte slots of page-locked host memory mapped into every device
// (the kernels store to them directly; the host reads them after an execution completed,
// without a device synchronisation). Blocks are never freed (cudaFreeHost would synchronize
// the device); slots return to the pool in stream order after a plan's last execution.
class StatusPool {
public:
    int* acquire() {
        std::lock_guard<std::mutex> lock(mu_);
        if (free_.empty()) {
            constexpr int kBlock = 1024;
            void* block = nullptr;
            check(cudaHostAlloc(&block, kBlock * sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable),
                  "cudaHostAlloc(status words)");
            int* words = static_cast<int*>(block);
            for (int i = kBlock - 1; i >= 0; --i) free_.push_back(words + i);
        }
        int* w = free_.back();
        free_.pop_back();
        __atomic_store_n(w, 0, __ATOMIC_SEQ_CST);
        return w;
    }
    void release(int* w) {
        std::lock_guard<std::mutex> lock(mu_);
        free_.push_back(w);
    }

private:
    std::mutex mu_;
    std::vector<int*> free_;
};

StatusPool& status_pool() {
    static StatusPool* pool = new StatusPool;  // outlives host callbacks still queued at exit
    return *pool;
}

void release_status_word(void* w) { status_pool().release(static_cast<int*>(w)); }

struct DevicePlan {
    PlanSpec spec;
    int device = 0;
    void* table_mem = nullptr;
    size_t table_bytes = 0;  // size of table_mem
    void* scratch = nullptr;
    // Status word (StatusPool): non-zero after a bounded wait in one of the plan's kernels gave
    // up. Plans built over other plans (real, strided) point at a child's word.
    int* status = nullptr;
    bool owns_status = false;
    long long wait_polls = kSpinLimit;  // polls before a bounded wait in the plan's kernels gives up
    int sms = 148;
    std::vector<BoundPass> passes;
    cudaEvent_t done = nullptr;
    cudaEvent_t ready = nullptr;  // tables complete (recorded on the memory stream at creation)
    bool ready_done = false;      // `ready` has completed: executes need not wait for it
    bool stream_scratch = false;  // scratch comes from the executing stream's arena
    std::mutex mu;
    // Real transforms (syclfft_b200_create_real): a complex plan of half the length, with the
    // post-process (R2C) or pre-process (C2R) of real_kernel.cu around it.
    int real_kind = 0;              // 0 complex, 1 R2C, 2 C2R
    int64_t real_n = 0;             // real length N (even)
    std::unique_ptr<DevicePlan> inner;
    void* real_buf = nullptr;       // half-length spectra: batch x N/2 complex
    void* real_tw = nullptr;        // W_N^k, k = 0..N/2 (then the fused kernel's base twiddles)
    const RealFusedEntry* real_fused = nullptr;  // one-pass kernel for N/2 (real_kernel.cu), or none
    int64_t real_base_off = 0;      // complex elements from real_tw to the base twiddles
    // Real transforms of rank 2-3: `inner` is the 1D real plan of the last axis over every outer
    // line, `outer` the complex plan over the outer axes (last axis untransformed), md_buf the
    // C2R intermediate (batch x outer lines x (N/2+1) complex).
    bool real_md = false;
    int64_t real_outer = 1;
    std::unique_ptr<DevicePlan> outer;
    void* md_buf = nullptr;
    // Strided layouts (syclfft_b200_create_strided): the contiguous plan `inner` with gather /
    // scatter passes (layout_kernel.cu) on the sides that are not contiguous.
    bool strided = false;
    Layout in_layout, out_layout;
    bool in_contig = true, out_contig = true;
    bool interleaved = false;       // both sides the dense [L.., batch] array: `inner` runs on it directly
    void* pack_buf = nullptr;       // contiguous batch x prod(L) complex

    ~DevicePlan() {
        int prev = 0;
        if (cudaGetDevice(&prev) == cudaSuccess && prev != device) cudaSetDevice(device);
        cudaStream_t ms = nullptr;
        try {
            ms = memory_stream(device);
        } catch (...) {
        }
        if (ms) {
            // free after the plan's last execution, without blocking host or device
            if (done) cudaStreamWaitEvent(ms, done, 0);
            if (scratch) cudaFreeAsync(scratch, ms);
            if (table_mem) cudaFreeAsync(table_mem, ms);
            if (real_buf) cudaFreeAsync(real_buf, ms);
            if (real_tw) cudaFreeAsync(real_tw, ms);
            if (pack_buf) cudaFreeAsync(pack_buf, ms);
            if (md_buf) cudaFreeAsync(md_buf, ms);
            if (owns_status && cudaLaunchHostFunc(ms, release_status_word, status) == cudaSuccess)
                owns_status = false;
        } else {
            if (done) cudaEventSynchronize(done);
            if (scratch) cudaFree(scratch);
            if (table_mem) cudaFree(table_mem);
            if (real_buf) cudaFree(real_buf);
            if (real_tw) cudaFree(real_tw);
            if (pack_buf) cudaFree(pack_buf);
            if (md_buf) cudaFree(md_buf);
        }
        if (owns_status) status_pool().release(status);
        if (done) cudaEventDestroy(done);
        if (ready) cudaEventDestroy(ready);
        if (prev != device) cudaSetDevice(prev);
    }
};

// Scratch arenas, one per (device, stream): stream-ordered (cudaMallocAsync on the stream
// itself), grown on demand, shared by every stream-scratch plan executed on that stream.
struct StreamArena {
    void* ptr = nullptr;
    size_t size = 0;
};
std::mutex g_arena_mu;
std::map<std::pair<int, cudaStream_t>, StreamArena> g_arenas;

void* stream_arena(int device, cudaStream_t stream, size_t bytes, bool capturing) {
    auto& arenas = g_arenas;
    using Arena = StreamArena;
    std::lock_guard<std::mutex> lock(g_arena_mu);
    Arena& a = arenas[{device, stream}];
    if (a.size < bytes) {
        // memory allocated inside a CUDA-graph capture would belong to the graph
        if (capturing)
            throw std::runtime_error("stream scratch arena too small under CUDA-graph capture: execute this plan once "
                                     "on the stream before capturing");
        if (a.ptr) check(cudaFreeAsync(a.ptr, stream), "cudaFreeAsync(arena)");
        a.ptr = nullptr;
        a.size = 0;
        size_t grow = bytes + bytes / 4;
        check(cudaMallocAsync(&a.ptr, grow, stream), "cudaMallocAsync(arena)");
        a.size = grow;
    }
    return a.ptr;
}

// Page-locked staging buffers for plan-table uploads, per device. A copy from pageable memory
// first waits for everything queued on the memory stream (other plans' chirp and spectrum
// work), which serialised concurrent plan creations behind each other's device work; a copy
// from page-locked memory is asynchronous. A buffer is reused once the event recorded after
// its copy has completed; buffers are never freed (cudaFreeHost would synchronize the device).
class UploadStaging {
public:
    struct Buffer {
        unsigned char* data = nullptr;
        size_t cap = 0;
        cudaEvent_t copied = nullptr;
        bool in_use = false;  // acquired and not yet released
        bool pending = false; // a copy from it may still run
    };
    Buffer* acquire(size_t bytes) {
        std::lock_guard<std::mutex> lock(mu_);
        Buffer* pick = nullptr;
        for (auto& b : buffers_) {
            if (b->in_use || b->cap < bytes) continue;
            if (b->pending) {
                if (cudaEventQuery(b->copied) != cudaSuccess) {
                    cudaGetLastError();  // not ready yet
                    continue;
                }
                b->pending = false;
            }
            if (!pick || b->cap < pick->cap) pick = b.get();
        }
        if (!pick) {
            auto b = std::make_unique<Buffer>();
            b->cap = std::max<size_t>((bytes + (1u << 20) - 1) & ~size_t((1u << 20) - 1), size_t(1) << 20);
            void* p = nullptr;
            check(cudaHostAlloc(&p, b->cap, cudaHostAllocPortable), "cudaHostAlloc(table staging)");
            b->data = static_cast<unsigned char*>(p);
            check(cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming), "cudaEventCreate");
            pick = b.get();
            buffers_.push_back(std::move(b));
        }
        pick->in_use = true;
        return pick;
    }
    // The copy from `b` was enqueued on `stream`: the buffer is free again once it completed.
    void release(Buffer* b, cudaStream_t stream) {
        std::lock_guard<std::mutex> lock(mu_);
        b->pending = cudaEventRecord(b->copied, stream) == cudaSuccess;
        if (!b->pending) cudaStreamSynchronize(stream);  // could not track it: wait instead
        b->in_use = false;
    }

private:
    std::mutex mu_;
    std::vector<std::unique_ptr<Buffer>> buffers_;
};

UploadStaging& upload_staging(int device) {
    static std::mutex mu;
    static std::map<int, UploadStaging*> all;  // never destroyed: buffers outlive static teardown
    std::lock_guard<std::mutex> lock(mu);
    auto& s = all[device];
    if (!s) s = new UploadStaging;
    return *s;
}

template <class T>
void pack_table(const std::vector<std::complex<double>>& t, unsigned char* blob, size_t off) {
    T* dst = reinterpret_cast<T*>(blob + off);
    for (size_t i = 0; i < t.size(); ++i) {
        dst[2 * i] = static_cast<T>(t[i].real());
        dst[2 * i + 1] = static_cast<T>(t[i].imag());
    }
}

DevicePlan* create_plan(const syclfft_b200_plan_config_v1& cfg, uint32_t flags = 0, uint32_t skip_axes = 0);
void execute_plan(DevicePlan* plan, const void* in, void* out, cudaStream_t stream, uint64_t batch = 0,
                  int direction = 0, int normalization = -1);

// FP64 forward in-place FFT plans of length M used to make chirp spectra; kept for the process.
DevicePlan* spectrum_plan(int device, int64_t M) {
    static std::mutex mu;
    static std::map<std::pair<int, int64_t>, DevicePlan*> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({device, M});
    if (it != cache.end()) return it->second;
    syclfft_b200_plan_config_v1 c{};
    c.abi_version = SYCLFFT_B200_PROVIDER_ABI_VERSION;
    c.scalar = SYCLFFT_B200_SCALAR_DOUBLE;
    c.direction = -1;
    c.rank = 1;
    c.lengths[0] = static_cast<uint64_t>(M);
    c.batch_count = 1;
    c.in_place = 1;
    c.device = device;
    DevicePlan* p = create_plan(c);
    cache[{device, M}] = p;
    return p;
}

DevicePlan* build_plan(PlanRequest req, int device, uint32_t flags, const std::string& tuning);
PlanRequest tune(const PlanRequest& req, int device, std::string* report);

DevicePlan* create_plan(const syclfft_b200_plan_config_v1& cfg, uint32_t flags, uint32_t skip_axes) {
    if (cfg.abi_version != SYCLFFT_B200_PROVIDER_ABI_VERSION) throw std::runtime_error("B200 provider ABI mismatch");
    if (cfg.scalar != SYCLFFT_B200_SCALAR_FLOAT && cfg.scalar != SYCLFFT_B200_SCALAR_DOUBLE)
        throw std::invalid_argument("unsupported scalar type");
    if (cfg.rank == 0 || cfg.rank > 3) throw std::invalid_argument("FFT rank must be between 1 and 3");
    PlanRequest req;
    req.dbl = cfg.scalar == SYCLFFT_B200_SCALAR_DOUBLE;
    req.direction = cfg.direction;
    req.normalization = static_cast<int>(cfg.normalization);
    req.in_place = cfg.in_place != 0;
    req.shape.assign(cfg.lengths, cfg.lengths + cfg.rank);
    req.batch = cfg.batch_count;
    req.split_bf16 = !req.dbl && (flags & SYCLFFT_B200_CREATE_SPLIT_BF16) != 0;
    req.skip_axes = skip_axes;
    // SYCLFFT_B200_KERNELS=generic: plan every pass on the runtime-parameterised kernel
    // (used to test and compare it against the size-specialised kernels).
    if (const char* k = std::getenv("SYCLFFT_B200_KERNELS")) req.no_fixed = std::strcmp(k, "generic") == 0;
    // SYCLFFT_B200_SPLIT_N1=<n1>: four-step column length, where it divides the axis.
    if (const char* k = std::getenv("SYCLFFT_B200_SPLIT_N1")) req.force_n1 = std::atoi(k);
    // SYCLFFT_B200_TMA=1: four-step column passes on the TMA-staged kernels.
    if (const char* k = std::getenv("SYCLFFT_B200_TMA")) req.use_tma = std::strcmp(k, "1") == 0;
    // SYCLFFT_B200_PIPED=0: never use the copy-engine-pipelined kernels.
    if (const char* k = std::getenv("SYCLFFT_B200_PIPED")) req.no_piped = std::strcmp(k, "0") == 0;
    // SYCLFFT_B200_RADER=0: prime lengths keep Bluestein's convolution (tests, comparisons).
    if (const char* k = std::getenv("SYCLFFT_B200_RADER")) req.no_rader = std::strcmp(k, "0") == 0;
    if (const char* k = std::getenv("SYCLFFT_B200_FUSED4_SINGLE")) req.fused_single = std::strcmp(k, "1") == 0;
    if (const char* k = std::getenv("SYCLFFT_B200_FUSED4")) {
        if (std::strcmp(k, "1") != 0) req.fused_single = false;
    } else {
        req.fused_single = false;  // the fused kernels are opt-in
    }
    // SYCLFFT_B200_CLUSTER=off: long lines take the two-pass four-step; =8 / =16: cluster size.
    // =pipe: complex<double> 65536-point lines on the pipelined 16-CTA cluster kernel.
    if (const char* k = std::getenv("SYCLFFT_B200_CLUSTER")) {
        if (std::strcmp(k, "off") == 0) {
            req.no_cluster = true;
        } else if (std::strcmp(k, "pipe") == 0) {
            req.cluster_p = 16;
            req.cluster_pipe = true;
        } else {
            req.cluster_p = std::atoi(k);
        }
    }

    int device = cfg.device;
    if (device < 0) check(cudaGetDevice(&device), "cudaGetDevice");
    DeviceGuard guard(device);
    std::string tuning;
    if (cfg.measure) {
        // planning_mode::measure: time the candidate decompositions and kernels
        (void)make_plan(req);  // argument validation before any device work
        req = tune(req, device, &tuning);
    }
    return build_plan(req, device, flags, tuning);
}

DevicePlan* build_plan(PlanRequest req, int device, uint32_t flags, const std::string& tuning) {
    int smem_optin = 0;
    check(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "cudaDeviceGetAttribute");
    req.smem_limit = smem_optin;
    req.device_spectrum = true;
    if (flags & SYCLFFT_B200_CREATE_SPLIT_BF16) req.split_bf16 = !req.dbl;

    auto plan = std::make_unique<DevicePlan>();
    plan->device = device;
    plan->spec = make_plan(req);
    plan->spec.tuning = tuning;
    const size_t cs = req.dbl ? 16 : 8;

    // All tables in one allocation, each 256-byte aligned: the complex tables (cast to the
    // plan precision), then the int32 index tables.
    std::vector<size_t> offsets(plan->spec.tables.size()), ioffsets(plan->spec.index_tables.size());
    size_t total = 0;
    for (size_t i = 0; i < plan->spec.tables.size(); ++i) {
        offsets[i] = total;
        total += (plan->spec.table_sizes[i] * cs + 255) / 256 * 256;
    }
    for (size_t i = 0; i < plan->spec.index_tables.size(); ++i) {
        ioffsets[i] = total;
        total += (plan->spec.index_tables[i].size() * sizeof(int32_t) + 255) / 256 * 256;
    }
    const size_t table_bytes = std::max<size_t>(total, 256);
    cudaStream_t ms = memory_stream(device);
    UploadStaging& staging = upload_staging(device);
    UploadStaging::Buffer* blob = staging.acquire(table_bytes);
    std::memset(blob->data, 0, table_bytes);
    for (size_t i = 0; i < plan->spec.tables.size(); ++i) {
        if (req.dbl) pack_table<double>(plan->spec.tables[i], blob->data, offsets[i]);
        else pack_table<float>(plan->spec.tables[i], blob->data, offsets[i]);
    }
    for (size_t i = 0; i < plan->spec.index_tables.size(); ++i) {
        const auto& t = plan->spec.index_tables[i];
        if (!t.empty()) std::memcpy(static_cast<unsigned char*>(blob->data) + ioffsets[i], t.data(), t.size() * sizeof(int32_t));
    }
    cudaError_t up = cudaMallocAsync(&plan->table_mem, table_bytes, ms);
    if (up == cudaSuccess) up = cudaMemcpyAsync(plan->table_mem, blob->data, table_bytes, cudaMemcpyHostToDevice, ms);
    staging.release(blob, ms);
    check(up, "plan table upload");
    plan->table_bytes = table_bytes;
    plan->status = status_pool().acquire();
    plan->owns_status = true;
    // failure-detection testing: SYCLFFT_B200_WAIT_POLLS sets the wait limit of new plans
    if (const char* v = std::getenv("SYCLFFT_B200_WAIT_POLLS")) {
        char* end = nullptr;
        const long long polls = std::strtoll(v, &end, 10);
        if (end != v && polls >= 0) plan->wait_polls = polls;
    }
    check(cudaDeviceGetAttribute(&plan->sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    plan->stream_scratch = (flags & SYCLFFT_B200_CREATE_STREAM_SCRATCH) != 0;
    if (plan->spec.scratch_elements && !plan->stream_scratch) {
        check(cudaMallocAsync(&plan->scratch, plan->spec.scratch_elements * cs, ms), "cudaMallocAsync(scratch)");
    }
    check(cudaEventCreateWithFlags(&plan->done, cudaEventDisableTiming), "cudaEventCreate");
    if (!plan->spec.bluestein_jobs.empty()) {
        // chirps and chirp spectra on the device: exact-integer chirp, FP64 FFT of length M
        int64_t maxM = 0;
        for (const auto& j : plan->spec.bluestein_jobs) maxM = std::max(maxM, j.M);
        void* kern = nullptr;
        check(cudaMallocAsync(&kern, static_cast<size_t>(maxM) * 16, ms), "cudaMallocAsync(chirp kernel)");
        try {
            for (const auto& j : plan->spec.bluestein_jobs) {
                void* chirp = static_cast<unsigned char*>(plan->table_mem) + offsets[j.chirp_table];
                void* spec = static_cast<unsigned char*>(plan->table_mem) + offsets[j.spectrum_table];
                check(bluestein_chirp(req.dbl, chirp, kern, j.L, j.M, j.sgn, ms), "chirp kernel");
                execute_plan(spectrum_plan(device, j.M), kern, kern, ms, 0);
                check(bluestein_spectrum(req.dbl, spec, kern, j.M, j.n1, j.n2, j.large, ms), "spectrum kernel");
            }
        } catch (...) {
            cudaFreeAsync(kern, ms);
            cudaStreamSynchronize(ms);
            throw;
        }
        cudaFreeAsync(kern, ms);
    }
    // executes wait for the tables (and chirp spectra) on the device; the host does not
    check(cudaEventCreateWithFlags(&plan->ready, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventRecord(plan->ready, ms), "cudaEventRecord");
    if (flags & SYCLFFT_B200_CREATE_SYNC) check(cudaStreamSynchronize(ms), "plan tables");

    auto tab = [&](int id) -> const void* {
        return id < 0 ? nullptr : static_cast<const unsigned char*>(plan->table_mem) + offsets[id];
    };
    for (const PassSpec& ps : plan->spec.passes) {
        if (ps.fixed_id < 0 && ps.cluster_id < 0 && ps.tc_id < 0 && ps.blue_id < 0 && !has_variant(req.dbl, ps.kc.maxv, ps.kc.maxt))
            throw std::runtime_error("no kernel variant for pass");
        BoundPass bp;
        bp.spec_ptr = &ps;  // plan->spec.passes is not modified after this point
        bp.p = ps.p;
        bp.p.fft1.tw = tab(ps.tables.tw1);
        bp.p.fft2.tw = tab(ps.tables.tw2);
        bp.p.premul = tab(ps.tables.premul);
        bp.p.pointwise = tab(ps.tables.pointwise);
        bp.p.postmul = tab(ps.tables.postmul);
        bp.p.tw4_hi = tab(ps.tables.tw4_hi);
        bp.p.tw4_lo = tab(ps.tables.tw4_lo);
        auto itab = [&](int id) -> const void* {
            return id < 0 ? nullptr : static_cast<const unsigned char*>(plan->table_mem) + ioffsets[id];
        };
        bp.p.perm_in = itab(ps.tables.perm_in);
        bp.p.perm_out = itab(ps.tables.perm_out);
        bp.fp = to_fixed(bp.p);
        bp.cp = to_cluster(bp.p);
        if (ps.cluster_pipe) {
            bp.kp.lines = bp.p.n_cols;
            bp.kp.in_pitch = bp.p.in.cs;
            bp.kp.out_pitch = bp.p.out.cs;
            bp.kp.tw_base = tab(ps.tables.cl_base);
            bp.kp.tw4_hi = bp.p.tw4_hi;
            bp.kp.tw4_lo = bp.p.tw4_lo;
            bp.kp.tw4_shift = bp.p.tw4_shift;
            bp.kp.conj_in = bp.p.conj_in;
            bp.kp.conj_out = bp.p.conj_out;
            bp.kp.scale = bp.p.scale;
            bp.kp.status = plan->status;
        }
        bp.pp = to_piped(bp.p, plan->status);
        bp.tp = to_tc(bp.p, tab(ps.tables.tc_tw), plan->status);
        plan->passes.push_back(bp);
    }
    // four-step column + row passes (and Bluestein's three passes) of a contiguous axis with a
    // fused kernel: one launch, the intermediate in an L2-resident ring. Opt-in
    // (SYCLFFT_B200_FUSED4=1): measured slower than the separate launches on B200.
    const char* f4 = std::getenv("SYCLFFT_B200_FUSED4");
    const bool fused_ok = f4 && f4[0] == '1' && !req.no_fixed;
    for (size_t i = 0; fused_ok && i + 1 < plan->passes.size(); ++i) {
        const PassSpec& a = plan->passes[i].spec_ref();
        const PassSpec& b = plan->passes[i + 1].spec_ref();
        if (a.kind == "fourstep_cols" && b.kind == "fourstep_rows" && a.fixed_id >= 0 && b.fixed_id >= 0 &&
            a.p.mode == kModeC && b.p.mode == kModeK && a.dst == Buf::Scratch && b.src == Buf::Scratch)
            plan->passes[i].fused4 = find_fused4(req.dbl, a.fixed_id, b.fixed_id);
        if (i + 2 < plan->passes.size() && a.kind == "bluestein_cols_fwd" && b.kind == "bluestein_rows_conv") {
            const PassSpec& c = plan->passes[i + 2].spec_ref();
            if (c.kind == "bluestein_cols_inv" && a.blue_id >= 0 && b.blue_id >= 0 && c.blue_id >= 0 &&
                a.dst == Buf::Scratch && b.src == Buf::Scratch && b.dst == Buf::Scratch && c.src == Buf::Scratch)
                plan->passes[i].fusedblue = find_fusedblue(req.dbl, a.blue_id, b.blue_id, c.blue_id);
        }
    }
    return plan.release();
}

// Line counts of a pass for the first `batch` transforms of a plan made for `planned`.
BoundPass rescale(const BoundPass& bp, uint64_t batch, uint64_t planned) {
    if (batch == planned) return bp;
    if (bp.spec_ref().batch_dim < 0) throw std::invalid_argument("plan cannot run a smaller batch");
    BoundPass r = bp;
    PassParams& p = r.p;
    const int64_t b = static_cast<int64_t>(batch), B = static_cast<int64_t>(planned);
    if (bp.spec_ref().batch_dim == 0) p.n_outer = p.n_outer / B * b;
    else p.n_cols = p.n_cols / B * b;
    p.col_tiles = (p.n_cols + p.w - 1) / p.w;
    p.tiles = p.n_outer * p.col_tiles;
    r.fp.n_cols = p.n_cols;
    r.fp.col_tiles = p.col_tiles;
    r.cp.lines = p.n_cols;
    r.kp.lines = p.n_cols;
    r.pp.lines = p.n_cols;
    r.tp.n_outer = p.n_outer;
    r.tp.n_cols = p.n_cols;
    r.tp.col_tiles = p.col_tiles;
    r.tp.tiles = p.tiles;
    if (bp.spec_ref().cluster_id >= 0) p.tiles = p.n_cols * bp.spec_ref().cl_p;
    return r;
}

// Direction / normalization override: conj(F(conj x)) turns a plan's transform into the
// other direction (conjugation on the first load and the last store; intermediate passes
// keep their own conjugation pairs), and the last store carries the requested scale.
void apply_override(BoundPass& bp, bool first, bool last_pass, bool flip, double scale, bool set_scale) {
    bool last = last_pass;
    const PassSpec& ps = bp.spec_ref();
    if (flip && first && (ps.tables.premul >= 0 || ps.tables.perm_in >= 0)) {
        bp.p.flip_in ^= 1;  // conjugate before the chirp pre-multiply (the Rader gather)
        bp.fp.flip_in ^= 1;
        first = false;
    }
    if (flip && last && (ps.tables.postmul >= 0 || ps.tables.perm_out >= 0)) {
        bp.p.flip_out ^= 1;  // conjugate after the chirp post-multiply (the Rader scatter)
        bp.fp.flip_out ^= 1;
        last = false;
    }
    if (flip) {
        if (first) {
            bp.p.conj_in ^= 1;
            bp.fp.conj_in ^= 1;
            bp.cp.conj_in ^= 1;
            bp.kp.conj_in ^= 1;
            bp.pp.conj_in ^= 1;
            bp.tp.conj_in ^= 1;
        }
        if (last) {
            bp.p.conj_out ^= 1;
            bp.fp.conj_out ^= 1;
            bp.cp.conj_out ^= 1;
            bp.kp.conj_out ^= 1;
            bp.pp.conj_out ^= 1;
            bp.tp.conj_out ^= 1;
        }
    }
    if (last_pass && set_scale) {
        bp.p.scale = bp.fp.scale = bp.cp.scale = bp.kp.scale = bp.pp.scale = scale;
        bp.tp.scale = static_cast<float>(scale);
    }
}

// Real transform of even length N over a complex plan of length N/2 (see real_kernel.cu).
DevicePlan* create_real_plan_1d(const syclfft_b200_plan_config_v1& cfg, int kind, uint32_t flags) {
    if (kind != SYCLFFT_B200_REAL_R2C && kind != SYCLFFT_B200_REAL_C2R)
        throw std::invalid_argument("real transform kind must be R2C or C2R");
    if (cfg.rank != 1) throw std::invalid_argument("real transforms are one-dimensional (batched)");
    const uint64_t n = cfg.lengths[0];
    if (n < 2 || n % 2) throw std::invalid_argument("real transforms need an even length >= 2");
    if (cfg.in_place) throw std::invalid_argument("real transforms are out of place");
    const int dir = kind == SYCLFFT_B200_REAL_R2C ? -1 : 1;
    if (cfg.direction != dir)
        throw std::invalid_argument(dir < 0 ? "R2C transforms are forward" : "C2R transforms are backward");
    if (cfg.normalization > 3) throw std::invalid_argument("Invalid normalization");
    syclfft_b200_plan_config_v1 ic = cfg;
    ic.lengths[0] = n / 2;
    ic.in_place = 0;
    ic.normalization = 0;
    std::unique_ptr<DevicePlan> inner(create_plan(ic, flags | SYCLFFT_B200_CREATE_SYNC));
    auto plan = std::make_unique<DevicePlan>();
    plan->device = inner->device;
    plan->sms = inner->sms;
    plan->spec.req = inner->spec.req;
    plan->spec.req.shape = {n};
    plan->spec.req.direction = dir;
    plan->spec.req.normalization = static_cast<int>(cfg.normalization);
    plan->spec.transform_size = n;
    plan->spec.elements = n * cfg.batch_count;
    plan->status = inner->status;
    plan->real_kind = kind;
    plan->real_n = static_cast<int64_t>(n);
    const bool dbl = plan->spec.req.dbl;
    const size_t cs = dbl ? 16 : 8;
    const uint64_t h = n / 2;
    // One pass when N/2 has a fused kernel (not for split-precision plans, whose inner FFT runs
    // on the tensor cores); SYCLFFT_B200_REAL_FUSED=0 keeps the two-pass form.
    const char* fused_env = std::getenv("SYCLFFT_B200_REAL_FUSED");
    const bool split = !dbl && (flags & SYCLFFT_B200_CREATE_SPLIT_BF16) != 0;
    if (!split && !(fused_env && std::strcmp(fused_env, "0") == 0))
        plan->real_fused = find_real_fused(dbl, static_cast<int64_t>(h));
    plan->spec.scratch_elements = plan->real_fused ? 0 : inner->spec.scratch_elements + h * cfg.batch_count;
    DeviceGuard guard(plan->device);
    cudaStream_t ms = memory_stream(plan->device);
    std::vector<std::complex<double>> table;
    for (uint64_t k = 0; k <= h; ++k) table.push_back(cis_neg(static_cast<int64_t>(k), static_cast<int64_t>(n)));
    plan->real_base_off = static_cast<int64_t>(table.size());
    if (plan->real_fused) {
        int64_t ns = 1;  // base twiddles of the fused kernel's stages: W_(ns*R)^jm, jm < ns
        for (int s = 0; s < plan->real_fused->nstages; ++s) {
            const int R = plan->real_fused->radices[s];
            for (int64_t jm = 0; jm < ns; ++jm) table.push_back(cis_neg(jm, ns * R));
            ns *= R;
        }
    }
    std::vector<unsigned char> tw(table.size() * cs);
    for (size_t k = 0; k < table.size(); ++k) {
        if (dbl) {
            reinterpret_cast<double*>(tw.data())[2 * k] = table[k].real();
            reinterpret_cast<double*>(tw.data())[2 * k + 1] = table[k].imag();
        } else {
            reinterpret_cast<float*>(tw.data())[2 * k] = static_cast<float>(table[k].real());
            reinterpret_cast<float*>(tw.data())[2 * k + 1] = static_cast<float>(table[k].imag());
        }
    }
    check(cudaMallocAsync(&plan->real_tw, tw.size(), ms), "cudaMallocAsync(real twiddles)");
    check(cudaMemcpyAsync(plan->real_tw, tw.data(), tw.size(), cudaMemcpyHostToDevice, ms), "cudaMemcpy(real twiddles)");
    if (!plan->real_fused)
        check(cudaMallocAsync(&plan->real_buf, h * cfg.batch_count * cs, ms), "cudaMallocAsync(real spectra)");
    check(cudaStreamSynchronize(ms), "real plan tables");
    check(cudaEventCreateWithFlags(&plan->done, cudaEventDisableTiming), "cudaEventCreate");
    plan->inner = std::move(inner);
    return plan.release();
}

// Real transforms of rank 1-3 over the last axis (even length N): R2C is the 1D real plan of the
// last axis over every outer line, then the complex FFT over the outer axes of the
// [outer.., N/2+1] spectrum in place (numpy.fft.rfftn's order); C2R runs the inverse complex
// FFT over the outer axes into a scratch spectrum first, then the 1D C2R of the last axis
// (numpy.fft.irfftn's order: the imaginary parts of bins 0 and N/2 are dropped per line).
// The normalization is relative to the whole transform size and applied by the last-axis pass.
DevicePlan* create_real_plan(const syclfft_b200_plan_config_v1& cfg, int kind, uint32_t flags) {
    if (cfg.rank == 0 || cfg.rank > 3) throw std::invalid_argument("FFT rank must be between 1 and 3");
    if (cfg.rank == 1) return create_real_plan_1d(cfg, kind, flags);
    if (kind != SYCLFFT_B200_REAL_R2C && kind != SYCLFFT_B200_REAL_C2R)
        throw std::invalid_argument("real transform kind must be R2C or C2R");
    const uint32_t r = cfg.rank;
    for (uint32_t k = 0; k < r; ++k)
        if (cfg.lengths[k] == 0) throw std::invalid_argument("FFT dimensions must be non-zero");
    if (cfg.batch_count == 0) throw std::invalid_argument("FFT batch count must be non-zero");
    const uint64_t n = cfg.lengths[r - 1];
    if (n < 2 || n % 2) throw std::invalid_argument("real transforms need an even last length >= 2");
    if (cfg.in_place) throw std::invalid_argument("real transforms are out of place");
    const int dir = kind == SYCLFFT_B200_REAL_R2C ? -1 : 1;
    if (cfg.direction != dir)
        throw std::invalid_argument(dir < 0 ? "R2C transforms are forward" : "C2R transforms are backward");
    if (cfg.normalization > 3) throw std::invalid_argument("Invalid normalization");
    uint64_t outer = 1;
    for (uint32_t k = 0; k + 1 < r; ++k) outer *= cfg.lengths[k];
    const uint64_t h = n / 2 + 1;
    // last axis: one line per (batch, outer index), scaled for the whole transform
    syclfft_b200_plan_config_v1 c1 = cfg;
    c1.rank = 1;
    c1.lengths[0] = n;
    c1.lengths[1] = c1.lengths[2] = 0;
    c1.batch_count = cfg.batch_count * outer;
    std::unique_ptr<DevicePlan> last(create_real_plan_1d(c1, kind, flags));
    last->spec.transform_size = n * outer;
    // outer axes of the [outer.., N/2+1] spectrum, the last axis left untransformed
    syclfft_b200_plan_config_v1 co = cfg;
    co.lengths[r - 1] = h;
    co.normalization = 0;
    co.in_place = kind == SYCLFFT_B200_REAL_R2C ? 1 : 0;
    std::unique_ptr<DevicePlan> outer_plan(create_plan(co, flags | SYCLFFT_B200_CREATE_SYNC, 1u << (r - 1)));
    auto plan = std::make_unique<DevicePlan>();
    plan->device = last->device;
    plan->sms = last->sms;
    plan->spec.req = last->spec.req;
    plan->spec.req.shape.assign(cfg.lengths, cfg.lengths + r);
    plan->spec.req.batch = cfg.batch_count;
    plan->spec.req.direction = dir;
    plan->spec.req.normalization = static_cast<int>(cfg.normalization);
    plan->spec.transform_size = n * outer;
    plan->spec.elements = n * outer * cfg.batch_count;
    plan->status = last->status;
    plan->real_kind = kind;
    plan->real_n = static_cast<int64_t>(n);
    plan->real_md = true;
    plan->real_outer = static_cast<int64_t>(outer);
    const size_t cs = plan->spec.req.dbl ? 16 : 8;
    const uint64_t spec_elems = cfg.batch_count * outer * h;
    plan->spec.scratch_elements = last->spec.scratch_elements + outer_plan->spec.scratch_elements +
                                  (kind == SYCLFFT_B200_REAL_C2R ? spec_elems : 0);
    DeviceGuard guard(plan->device);
    if (kind == SYCLFFT_B200_REAL_C2R) {
        cudaStream_t ms = memory_stream(plan->device);
        check(cudaMallocAsync(&plan->md_buf, spec_elems * cs, ms), "cudaMallocAsync(real spectrum scratch)");
        check(cudaStreamSynchronize(ms), "real spectrum scratch");
    }
    check(cudaEventCreateWithFlags(&plan->done, cudaEventDisableTiming), "cudaEventCreate");
    plan->inner = std::move(last);
    plan->outer = std::move(outer_plan);
    return plan.release();
}

Layout make_layout(const syclfft_b200_plan_config_v1& cfg, const int64_t* strides, int64_t dist) {
    Layout l;
    l.rank = static_cast<int>(cfg.rank);
    for (int k = 0; k < l.rank; ++k) {
        l.len[k] = static_cast<int64_t>(cfg.lengths[k]);
        l.stride[k] = strides[k];
    }
    l.dist = dist;
    l.batch = static_cast<int64_t>(cfg.batch_count);
    return l;
}

bool layout_contiguous(const Layout& l) {
    int64_t step = 1;
    for (int k = l.rank - 1; k >= 0; --k) {
        if (l.len[k] > 1 && l.stride[k] != step) return false;
        step *= l.len[k];
    }
    return l.batch == 1 || l.dist == step;
}

bool layout_same(const Layout& a, const Layout& b) {
    for (int k = 0; k < a.rank; ++k)
        if (a.len[k] > 1 && a.stride[k] != b.stride[k]) return false;
    return a.batch == 1 || a.dist == b.dist;
}

// The batch is the innermost, unit-stride index and the axes are dense C order around it.
bool layout_interleaved(const Layout& l) {
    if (l.dist != 1) return false;
    int64_t step = l.batch;
    for (int k = l.rank - 1; k >= 0; --k) {
        if (l.len[k] > 1 && l.stride[k] != step) return false;
        step *= l.len[k];
    }
    return true;
}

// Checks strides and distances; for the output side also that no two elements share an address
// (sufficient test: sorted by stride, each stride exceeds the span of the smaller ones).
void check_layout(const Layout& l, bool output) {
    const char* side = output ? "output" : "input";
    std::vector<std::pair<int64_t, int64_t>> dims;  // (stride, extent)
    for (int k = 0; k < l.rank; ++k) {
        if (l.stride[k] < 1) throw std::invalid_argument(std::string(side) + " strides must be >= 1");
        if (l.len[k] > 1) dims.push_back({l.stride[k], l.len[k]});
    }
    if (l.batch > 1) {
        if (l.dist < 1) throw std::invalid_argument(std::string(side) + " distance must be >= 1");
        dims.push_back({l.dist, l.batch});
    }
    long double span = 0;  // largest offset, in long double so huge strides cannot wrap
    for (auto& d : dims) span += static_cast<long double>(d.first) * static_cast<long double>(d.second - 1);
    if (span >= static_cast<long double>(INT64_MAX / 16))
        throw std::invalid_argument(std::string(side) + " layout exceeds the addressable range");
    if (!output) return;
    std::sort(dims.begin(), dims.end());
    int64_t reach = 0;  // largest offset reachable by the dimensions so far
    for (auto& d : dims) {
        if (d.first <= reach) throw std::invalid_argument("output layout overlaps itself");
        reach += d.first * (d.second - 1);
    }
}

DevicePlan* create_strided_plan(const syclfft_b200_plan_config_v1& cfg, const syclfft_b200_layout_v1& lay,
                                uint32_t flags) {
    if (cfg.rank == 0 || cfg.rank > 3) throw std::invalid_argument("FFT rank must be between 1 and 3");
    for (uint32_t k = 0; k < cfg.rank; ++k)
        if (cfg.lengths[k] == 0) throw std::invalid_argument("FFT dimensions must be non-zero");
    if (cfg.batch_count == 0) throw std::invalid_argument("FFT batch count must be non-zero");
    const Layout in = make_layout(cfg, lay.in_strides, lay.in_distance);
    const Layout out = make_layout(cfg, lay.out_strides, lay.out_distance);
    check_layout(in, false);
    check_layout(out, true);
    if (cfg.in_place && !layout_same(in, out))
        throw std::invalid_argument("an in-place plan needs equal input and output layouts");
    const bool ic = layout_contiguous(in), oc = layout_contiguous(out);
    if (ic && oc) return create_plan(cfg, flags);
    if (cfg.rank < 3 && cfg.batch_count > 1 && layout_same(in, out) && layout_interleaved(in)) {
        // The batch is the innermost index of a dense array [L.., batch]: plan that array with
        // its last axis left untransformed, so the axis passes read and write it in place of a
        // gather / scatter (transforms down the columns of a row-major matrix, FFTW's
        // stride = batch, distance = 1).
        syclfft_b200_plan_config_v1 c = cfg;
        c.rank = cfg.rank + 1;
        c.lengths[cfg.rank] = cfg.batch_count;
        c.batch_count = 1;
        std::unique_ptr<DevicePlan> inner(create_plan(c, flags | SYCLFFT_B200_CREATE_SYNC, 1u << cfg.rank));
        auto plan = std::make_unique<DevicePlan>();
        plan->device = inner->device;
        plan->sms = inner->sms;
        plan->spec.req = inner->spec.req;
        plan->spec.req.shape.assign(cfg.lengths, cfg.lengths + cfg.rank);
        plan->spec.req.batch = cfg.batch_count;
        plan->spec.req.skip_axes = 0;
        plan->spec.transform_size = inner->spec.transform_size;
        plan->spec.elements = inner->spec.elements;
        plan->spec.scratch_elements = inner->spec.scratch_elements;
        plan->status = inner->status;
        plan->strided = true;
        plan->interleaved = true;
        plan->in_layout = in;
        plan->out_layout = out;
        plan->in_contig = plan->out_contig = false;
        DeviceGuard guard(plan->device);
        check(cudaEventCreateWithFlags(&plan->done, cudaEventDisableTiming), "cudaEventCreate");
        plan->inner = std::move(inner);
        return plan.release();
    }
    syclfft_b200_plan_config_v1 c = cfg;
    c.in_place = (!ic && !oc) ? 1 : 0;  // both strided: transform the gathered copy in place
    std::unique_ptr<DevicePlan> inner(create_plan(c, flags | SYCLFFT_B200_CREATE_SYNC));
    auto plan = std::make_unique<DevicePlan>();
    plan->device = inner->device;
    plan->sms = inner->sms;
    plan->spec.req = inner->spec.req;
    plan->spec.req.in_place = cfg.in_place != 0;
    plan->spec.transform_size = inner->spec.transform_size;
    plan->spec.elements = inner->spec.elements;
    plan->status = inner->status;
    plan->strided = true;
    plan->in_layout = in;
    plan->out_layout = out;
    plan->in_contig = ic;
    plan->out_contig = oc;
    const size_t cs = plan->spec.req.dbl ? 16 : 8;
    plan->spec.scratch_elements = inner->spec.scratch_elements + inner->spec.elements;
    DeviceGuard guard(plan->device);
    cudaStream_t ms = memory_stream(plan->device);
    check(cudaMallocAsync(&plan->pack_buf, inner->spec.elements * cs, ms), "cudaMallocAsync(layout scratch)");
    check(cudaStreamSynchronize(ms), "layout scratch");
    check(cudaEventCreateWithFlags(&plan->done, cudaEventDisableTiming), "cudaEventCreate");
    plan->inner = std::move(inner);
    return plan.release();
}

void execute_strided(DevicePlan* plan, const void* in, void* out, cudaStream_t stream, uint64_t batch, int direction,
                     int normalization) {
    const uint64_t planned = plan->spec.req.batch;
    if (batch == 0) batch = planned;
    if (batch > planned) throw std::invalid_argument("batch exceeds the plan's batch count");
    if (plan->spec.req.in_place ? in != out : in == out)
        throw std::invalid_argument(plan->spec.req.in_place ? "In-place plan must be executed with execute(inout)"
                                                            : "Out-of-place plan requires distinct allocations");
    std::lock_guard<std::mutex> lock(plan->mu);
    DeviceGuard guard(plan->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
    const bool dbl = plan->spec.req.dbl;
    Layout li = plan->in_layout, lo = plan->out_layout;
    li.batch = lo.batch = static_cast<int64_t>(batch);
    DevicePlan* inner = plan->inner.get();
    if (plan->interleaved) {
        if (batch != planned)
            throw std::invalid_argument("a plan over an interleaved batch (distance 1) runs its whole batch");
        execute_plan(inner, in, out, stream, 0, direction, normalization);
    } else if (!plan->in_contig && !plan->out_contig) {
        check(launch_layout_gather(dbl, in, li, plan->pack_buf, stream), "layout gather");
        execute_plan(inner, plan->pack_buf, plan->pack_buf, stream, batch, direction, normalization);
        check(launch_layout_scatter(dbl, plan->pack_buf, out, lo, stream), "layout scatter");
    } else if (!plan->in_contig) {
        check(launch_layout_gather(dbl, in, li, plan->pack_buf, stream), "layout gather");
        execute_plan(inner, plan->pack_buf, out, stream, batch, direction, normalization);
    } else {
        execute_plan(inner, in, plan->pack_buf, stream, batch, direction, normalization);
        check(launch_layout_scatter(dbl, plan->pack_buf, out, lo, stream), "layout scatter");
    }
    check(cap != cudaStreamCaptureStatusNone ? cudaEventRecordWithFlags(plan->done, stream, cudaEventRecordExternal)
                                             : cudaEventRecord(plan->done, stream),
          "cudaEventRecord");
}

void execute_real(DevicePlan* plan, const void* in, void* out, cudaStream_t stream, uint64_t batch, int direction,
                  int normalization) {
    const uint64_t planned = plan->spec.req.batch;
    if (batch == 0) batch = planned;
    if (batch > planned) throw std::invalid_argument("batch exceeds the plan's batch count");
    if (in == out) throw std::invalid_argument("Out-of-place plan requires distinct allocations");
    const int dir = plan->spec.req.direction;
    if (direction != 0 && direction != dir) throw std::invalid_argument("a real plan runs in its own direction");
    if (plan->real_md) {
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceGuard guard(plan->device);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        check(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
        const uint64_t lines = batch * static_cast<uint64_t>(plan->real_outer);
        if (plan->real_kind == SYCLFFT_B200_REAL_R2C) {
            execute_real(plan->inner.get(), in, out, stream, lines, 0, normalization);
            execute_plan(plan->outer.get(), out, out, stream, batch, 0, -1);
        } else {
            execute_plan(plan->outer.get(), in, plan->md_buf, stream, batch, 0, -1);
            execute_real(plan->inner.get(), plan->md_buf, out, stream, lines, 0, normalization);
        }
        check(cap != cudaStreamCaptureStatusNone ? cudaEventRecordWithFlags(plan->done, stream, cudaEventRecordExternal)
                                                 : cudaEventRecord(plan->done, stream),
              "cudaEventRecord");
        return;
    }
    const int norm = normalization < 0 ? plan->spec.req.normalization : normalization;
    const double scale = normalization_scale(norm, dir, plan->spec.transform_size);
    std::lock_guard<std::mutex> lock(plan->mu);
    DeviceGuard guard(plan->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
    const bool dbl = plan->spec.req.dbl;
    const int64_t h = plan->real_n / 2;
    const int64_t lines = static_cast<int64_t>(batch);
    // the real side is read / written as complex pairs
    const uintptr_t align = dbl ? 16 : 8;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) % align)
        throw std::invalid_argument("real-transform buffers must be aligned to the complex element size");
    if (plan->real_fused) {
        const void* base = static_cast<const unsigned char*>(plan->real_tw) + plan->real_base_off * (dbl ? 16 : 8);
        check(launch_real_fused(*plan->real_fused, plan->real_kind == SYCLFFT_B200_REAL_R2C, in, out, lines,
                                plan->real_tw, base, scale, stream),
              "fused real transform");
    } else if (plan->real_kind == SYCLFFT_B200_REAL_R2C) {
        execute_plan(plan->inner.get(), in, plan->real_buf, stream, batch, 0, -1);
        check(launch_r2c_post(dbl, plan->real_buf, out, h, lines, plan->real_tw, scale, stream), "R2C post-process");
    } else {
        check(launch_c2r_pre(dbl, in, plan->real_buf, h, lines, plan->real_tw, scale, stream), "C2R pre-process");
        execute_plan(plan->inner.get(), plan->real_buf, out, stream, batch, 0, -1);
    }
    check(cap != cudaStreamCaptureStatusNone ? cudaEventRecordWithFlags(plan->done, stream, cudaEventRecordExternal)
                                             : cudaEventRecord(plan->done, stream),
          "cudaEventRecord");
}

// TMA-staged four-step column pass; false when the tensor map cannot describe the buffer
// (the caller then runs the plain size-specialised kernel).
bool launch_tma(DevicePlan* plan, const BoundPass& bp, void* src, void* dst, cudaStream_t stream) {
    const PassParams& p = bp.p;
    const FixedParams& f = bp.fp;
    TmaColParams q;
    q.col_tiles = static_cast<int>((p.n_cols + f.w - 1) / f.w);
    q.n2 = static_cast<int>(p.n_cols);
    q.tiles = p.n_outer * q.col_tiles;
    q.out_hi = p.out.hi;
    q.out_ks = p.out.ks;
    q.tw = f.tw;
    q.tw4_hi = f.tw4_hi;
    q.tw4_lo = f.tw4_lo;
    q.tw4_shift = f.tw4_shift;
    q.conj_in = f.conj_in;
    q.conj_out = f.conj_out;
    q.scale = f.scale;
    q.status = plan->status;
    q.wait_polls = plan->wait_polls;
    const cudaError_t e = launch_tma_cols(bp.spec_ref().fixed_id, src, dst, p.n_outer, q, stream);
    if (e == cudaErrorInvalidValue) return false;
    check(e, "FFT TMA column pass launch");
    return true;
}

// Parameters of the contiguous runtime-length kernel for a bound pass (after its batch and
// direction / normalization overrides): the pass's geometry, the stage sequence with a
// multiply-shift quotient per stage (exact for the butterfly indices, j < 2^31), and the
// four-step twiddle.
LeanParams to_lean(const PassParams& p) {
    LeanParams L;
    L.n = p.n;
    L.tpl = p.tpl;
    L.w = p.w;
    while ((1 << L.w_shift) < p.w) ++L.w_shift;
    L.pitch = p.pitch;
    L.nstages = p.fft1.nstages;
    for (int s = 0; s < L.nstages; ++s) {
        L.radix[s] = p.fft1.radix[s];
        L.ns[s] = p.fft1.ns[s];
        L.tw_off[s] = p.fft1.tw_off[s];
        const uint32_t d = static_cast<uint32_t>(p.fft1.ns[s]);
        int l = 0;
        while ((uint64_t(2) << l) <= d) ++l;  // floor(log2 d)
        if ((d & (d - 1)) == 0) {
            L.ns_magic[s] = 0;
            L.ns_shift[s] = l;
        } else {
            // ceil(2^(32+l) / d) < 2^32: floor(j * m / 2^(32+l)) = floor(j / d) for j < 2^31
            L.ns_magic[s] = static_cast<uint32_t>(((uint64_t(1) << (32 + l)) + d - 1) / d);
            L.ns_shift[s] = l;
        }
    }
    L.tw = p.fft1.tw;
    L.n_cols = p.n_cols;
    L.col_tiles = p.col_tiles;
    L.in_hi = p.in.hi;
    L.in_cs = p.in.cs;
    L.out_hi = p.out.hi;
    L.out_cs = p.out.cs;
    L.in_ks = static_cast<int>(p.in.ks);
    L.out_ks = static_cast<int>(p.out.ks);
    L.conj_in = p.conj_in;
    L.conj_out = p.conj_out;
    L.scale = p.scale;
    L.tw4_hi = p.tw4_hi;
    L.tw4_lo = p.tw4_lo;
    L.tw4_shift = p.tw4_shift;
    L.tw4_conj = p.tw4_sign > 0 ? 1 : 0;
    return L;
}

// Launches one bound pass of a plan on its kernel family.
void launch_bound_pass(DevicePlan* plan, const BoundPass& bp, void* src, void* dst, cudaStream_t stream) {
    const bool aligned = (reinterpret_cast<uintptr_t>(src) % 16 == 0) && (reinterpret_cast<uintptr_t>(dst) % 16 == 0);
    const PassSpec& ps = bp.spec_ref();
    if (ps.blue_id >= 0) {
        check(launch_blue(ps.blue_id, plan->spec.req.dbl, ps.blue_kind, ps.rader, bp.fp, ps.threads,
                          static_cast<size_t>(ps.smem_bytes), bp.p.tiles, src, dst, stream),
              "FFT Bluestein pass launch");
    } else if (ps.tc_id >= 0) {
        check(launch_tc(ps.tc_id, bp.tp, src, dst, stream), "FFT tensor-core pass launch");
    } else if (ps.piped_id >= 0 && aligned) {
        const int64_t lines = bp.pp.lines;
        const int grid = static_cast<int>(lines < plan->sms ? lines : plan->sms);
        check(launch_piped(ps.piped_id, bp.pp, grid, src, dst, stream), "FFT pipelined pass launch");
    } else if (ps.cluster_pipe && aligned) {
        check(launch_cluster_pipe(bp.kp, src, dst, stream), "FFT pipelined cluster pass launch");
    } else if (ps.cluster_id >= 0) {
        check(launch_cluster(ps.cluster_id, bp.cp, src, dst, stream), "FFT cluster pass launch");
    } else if (ps.tma && aligned && launch_tma(plan, bp, src, dst, stream)) {
        // launched on the TMA-staged kernel
    } else if (ps.fixed_id >= 0) {
        check(launch_fixed(ps.fixed_id, plan->spec.req.dbl, bp.p.mode == kModeC, bp.fp, ps.threads,
                           static_cast<size_t>(ps.smem_bytes), bp.p.tiles, src, dst, stream),
              "FFT pass launch");
    } else if (ps.lean) {
        // lean passes may hold radix-15 stages, which the general kernel does not have
        if (!has_lean_variant(plan->spec.req.dbl, ps.kc.maxv, ps.kc.maxt))
            throw std::runtime_error("runtime-length pass has no lean kernel instantiation");
        check(launch_lean(to_lean(bp.p), plan->spec.req.dbl, ps.kc.maxv, ps.kc.maxt, bp.p.mode == kModeC, ps.lean_feat,
                          ps.threads, static_cast<size_t>(ps.smem_bytes), bp.p.tiles, src, dst, stream),
              "FFT pass launch");
    } else {
        check(launch_pass(bp.p, plan->spec.req.dbl, ps.kc.maxv, ps.kc.maxt, ps.threads, static_cast<size_t>(ps.smem_bytes),
                          src, dst, stream),
              "FFT pass launch");
    }
}

void execute_plan(DevicePlan* plan, const void* in, void* out, cudaStream_t stream, uint64_t batch,
                  int direction, int normalization) {
    if (!plan || !in || !out) throw std::invalid_argument("invalid B200 execution argument");
    // The kernels move whole float2 / double2 elements; a misaligned address would fault
    // on the device (a sticky error for the whole context), so it is refused here.
    if (!plan->real_kind &&
        (reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) % (plan->spec.req.dbl ? 16 : 8))
        throw std::invalid_argument("buffers must be aligned to the complex element size");
    if (plan->real_kind) {
        execute_real(plan, in, out, stream, batch, direction, normalization);
        return;
    }
    if (plan->strided) {
        execute_strided(plan, in, out, stream, batch, direction, normalization);
        return;
    }
    const uint64_t planned = plan->spec.req.batch;
    if (batch == 0) batch = planned;
    if (batch > planned) throw std::invalid_argument("batch exceeds the plan's batch count");
    const bool in_place = plan->spec.req.in_place;
    if (in_place && in != out) throw std::invalid_argument("In-place plan must be executed with in == out");
    if (!in_place && in == out) throw std::invalid_argument("Out-of-place plan requires distinct allocations");
    std::lock_guard<std::mutex> lock(plan->mu);
    DeviceGuard guard(plan->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    if (plan->ready && !plan->ready_done) {
        if (!capturing) {
            // no event query during a capture: it would invalidate the capture
            if (cudaEventQuery(plan->ready) == cudaSuccess) {
                plan->ready_done = true;  // the tables are complete: no further waits
            } else {
                cudaGetLastError();  // cudaErrorNotReady is not an error here
                check(cudaStreamWaitEvent(stream, plan->ready, 0), "cudaStreamWaitEvent");
            }
        } else {
            // A graph cannot depend on work outside its capture: finish the plan's tables on
            // the host now (relaxed mode lets this thread synchronize while a capture is open),
            // so every replay finds them complete.
            cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
            check(cudaThreadExchangeStreamCaptureMode(&mode), "cudaThreadExchangeStreamCaptureMode");
            const cudaError_t e = cudaEventSynchronize(plan->ready);
            cudaThreadExchangeStreamCaptureMode(&mode);
            check(e, "cudaEventSynchronize(tables)");
        }
    }
    void* scratch = plan->scratch;
    if (plan->stream_scratch && plan->spec.scratch_elements) {
        const size_t need = plan->spec.scratch_elements / planned * batch * (plan->spec.req.dbl ? 16 : 8) + 256;
        scratch = stream_arena(plan->device, stream, need, capturing);
    }
    const int dir = direction == 0 ? plan->spec.req.direction : direction;
    const int norm = normalization < 0 ? plan->spec.req.normalization : normalization;
    const bool flip = dir != plan->spec.req.direction;
    const bool set_scale = flip || norm != plan->spec.req.normalization;
    const double scale = normalization_scale(norm, dir, plan->spec.transform_size);
    auto buf = [&](Buf b) -> void* {
        if (b == Buf::Input) return const_cast<void*>(in);
        if (b == Buf::Output) return out;
        return scratch;
    };
    const size_t np = plan->passes.size();
    for (size_t i = 0; i < np; ++i) {
        BoundPass bp = rescale(plan->passes[i], batch, planned);
        bp.pp.wait_polls = plan->wait_polls;
        bp.tp.wait_polls = plan->wait_polls;
        if (flip || set_scale) apply_override(bp, i == 0, i + 1 == np, flip, scale, set_scale);
        if (bp.fused4 && i + 1 < np && bp.p.n_outer >= 3) {
            BoundPass bq = rescale(plan->passes[i + 1], batch, planned);
            if (flip || set_scale) apply_override(bq, false, i + 2 == np, flip, scale, set_scale);
            Fused4Params f;
            f.lines = bp.p.n_outer;
            f.tw1 = bp.fp.tw;
            f.tw2 = bq.fp.tw;
            f.tw4_hi = bp.fp.tw4_hi;
            f.tw4_lo = bp.fp.tw4_lo;
            f.tw4_shift = bp.fp.tw4_shift;
            f.conj_in = bp.fp.conj_in;
            f.conj_out = bq.fp.conj_out;
            f.scale = bq.fp.scale;
            f.wait_polls = plan->wait_polls;
            f.status = plan->status;
            check(launch_fused4(*bp.fused4, f, buf(bp.spec_ref().src), buf(bq.spec_ref().dst), scratch, stream),
                  "FFT fused four-step launch");
            ++i;
            continue;
        }
        if (bp.fusedblue && i + 2 < np && bp.p.n_outer >= 4) {
            BoundPass bq = rescale(plan->passes[i + 1], batch, planned);
            BoundPass br = rescale(plan->passes[i + 2], batch, planned);
            if (flip || set_scale) {
                apply_override(bq, false, false, flip, scale, set_scale);
                apply_override(br, false, i + 3 == np, flip, scale, set_scale);
            }
            FusedBlueParams f;
            f.lines = bp.p.n_outer;
            f.wait_polls = plan->wait_polls;
            f.status = plan->status;
            f.a = bp.fp;
            f.b = bq.fp;
            f.c = br.fp;
            check(launch_fusedblue(*bp.fusedblue, f, buf(bp.spec_ref().src), buf(br.spec_ref().dst), scratch, stream),
                  "FFT fused Bluestein launch");
            i += 2;
            continue;
        }
        if (bp.spec_ref().rader_dc && i > 0 && i + 1 < np) {
            // Rader convolution pass: X[0] of each line, from x[0] of the axis input, with the
            // flips and scale that the column passes around it apply to the other outputs
            BoundPass ba = rescale(plan->passes[i - 1], batch, planned);
            BoundPass bc = rescale(plan->passes[i + 1], batch, planned);
            if (flip || set_scale) {
                apply_override(ba, i - 1 == 0, false, flip, scale, set_scale);
                apply_override(bc, false, i + 2 == np, flip, scale, set_scale);
            }
            bp.fp.dc_x = buf(bp.spec_ref().rader_src);
            bp.fp.dc_y = buf(bc.spec_ref().dst);
            bp.fp.dc_x_pitch = ba.p.in.hi;
            bp.fp.dc_y_pitch = bc.p.out.hi;
            bp.fp.dc_scale = bc.fp.scale;
            bp.fp.dc_flip_in = ba.fp.flip_in;
            bp.fp.dc_flip_out = bc.fp.flip_out;
        }
        launch_bound_pass(plan, bp, buf(bp.spec_ref().src), buf(bp.spec_ref().dst), stream);
    }
    // Under capture the record becomes a node of the graph, so destroying the plan still
    // waits for the last replay that used its tables and scratch.
    check(capturing ? cudaEventRecordWithFlags(plan->done, stream, cudaEventRecordExternal)
                    : cudaEventRecord(plan->done, stream),
          "cudaEventRecord");
}

// ---------------------------------------------------------------- host buffers
// Transforms of page-locked host buffers (syclfft_b200_execute_host). The batch is cut into
// chunks that flow through device staging slots in a three-stage pipeline: copy in on one
// stream, the stages' transforms on the caller's stream, copy out on another. The two PCIe
// directions and the kernels then overlap, so a chunked call costs about the slower copy
// direction plus one chunk, not the sum of both copies and the kernels.
constexpr int kHostSlots = 4;

struct HostStaging {
    std::mutex mu;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    unsigned char* mem = nullptr;  // kHostSlots x 2 buffers of slot_bytes
    size_t slot_bytes = 0;
    cudaEvent_t start = nullptr;
    cudaEvent_t loaded[kHostSlots] = {}, computed[kHostSlots] = {}, freed[kHostSlots] = {};
    bool pending[kHostSlots] = {};  // freed[i] guards a copy-out still to be waited for
    unsigned next = 0;              // slot of the next chunk (rotates across calls)
};

HostStaging& host_staging(int device) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<HostStaging>> all;
    std::lock_guard<std::mutex> lock(mu);
    auto& h = all[device];
    if (!h) {
        auto fresh = std::make_unique<HostStaging>();
        check(cudaStreamCreateWithFlags(&fresh->h2d, cudaStreamNonBlocking), "cudaStreamCreate(copy in)");
        check(cudaStreamCreateWithFlags(&fresh->d2h, cudaStreamNonBlocking), "cudaStreamCreate(copy out)");
        check(cudaEventCreateWithFlags(&fresh->start, cudaEventDisableTiming), "cudaEventCreate");
        for (int i = 0; i < kHostSlots; ++i) {
            check(cudaEventCreateWithFlags(&fresh->loaded[i], cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&fresh->computed[i], cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&fresh->freed[i], cudaEventDisableTiming), "cudaEventCreate");
        }
        h = std::move(fresh);
    }
    return *h;
}

size_t host_chunk_bytes() {
    static const size_t bytes = [] {
        const char* v = std::getenv("SYCLFFT_B200_HOST_CHUNK_MB");
        const long mb = v ? std::strtol(v, nullptr, 10) : 0;
        return static_cast<size_t>(mb > 0 ? mb : 64) << 20;
    }();
    return bytes;
}

bool is_host_memory(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

void execute_host(const syclfft_b200_host_stage_v1* stages, uint32_t count, const void* in, void* out, uint64_t batch,
                  cudaStream_t stream) {
    if (!stages || count == 0) throw std::invalid_argument("at least one stage is needed");
    if (!in || !out) throw std::invalid_argument("input and output must be non-null");
    auto* first = static_cast<DevicePlan*>(stages[0].plan);
    if (!first) throw std::invalid_argument("invalid B200 execution argument");
    const bool dbl = first->spec.req.dbl;
    const uint64_t line = first->spec.transform_size;
    if (batch == 0) batch = first->spec.req.batch;
    for (uint32_t i = 0; i < count; ++i) {
        auto* p = static_cast<DevicePlan*>(stages[i].plan);
        if (!p) throw std::invalid_argument("invalid B200 execution argument");
        if (p->real_kind || p->strided)
            throw std::invalid_argument("host-buffer execution takes complex plans of contiguous layout");
        if (p->spec.req.dbl != dbl || p->spec.transform_size != line || p->device != first->device)
            throw std::invalid_argument("host-buffer stages need one precision, transform size and device");
        if (batch > p->spec.req.batch) throw std::invalid_argument("batch exceeds the plan's batch count");
        if (stages[i].direction != 0 && stages[i].direction != -1 && stages[i].direction != 1)
            throw std::invalid_argument("Invalid FFT direction");
        if (stages[i].normalization > 3) throw std::invalid_argument("Invalid normalization");
    }
    const size_t cs = dbl ? 16 : 8;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) % cs)
        throw std::invalid_argument("buffers must be aligned to the complex element size");
    if (!is_host_memory(in) || !is_host_memory(out))
        throw std::invalid_argument("host buffers must be page-locked (cudaHostAlloc / cudaHostRegister)");
    DeviceGuard guard(first->device);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(stream, &cap), "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
        throw std::invalid_argument("host-buffer execution cannot be captured in a CUDA graph");

    const size_t line_bytes = static_cast<size_t>(line) * cs;
    const uint64_t chunk_lines = std::max<uint64_t>(1, host_chunk_bytes() / line_bytes);
    const size_t need = static_cast<size_t>(std::min<uint64_t>(chunk_lines, batch)) * line_bytes;
    HostStaging& hs = host_staging(first->device);
    std::lock_guard<std::mutex> lock(hs.mu);
    if (hs.slot_bytes < need) {
        // every earlier chunk's copy-out is done before the staging memory is replaced
        check(cudaStreamSynchronize(hs.d2h), "staging");
        if (hs.mem) check(cudaFree(hs.mem), "cudaFree(staging)");
        hs.mem = nullptr;
        hs.slot_bytes = 0;
        for (bool& b : hs.pending) b = false;
        check(cudaMalloc(&hs.mem, need * 2 * kHostSlots), "cudaMalloc(staging)");
        hs.slot_bytes = need;
    }
    // the copies start after the caller's earlier work on `stream`
    check(cudaEventRecord(hs.start, stream), "cudaEventRecord");
    check(cudaStreamWaitEvent(hs.h2d, hs.start, 0), "cudaStreamWaitEvent");
    const auto* src = static_cast<const unsigned char*>(in);
    auto* dst = static_cast<unsigned char*>(out);
    int last = -1;
    for (uint64_t l0 = 0; l0 < batch; l0 += chunk_lines) {
        const uint64_t nl = std::min<uint64_t>(chunk_lines, batch - l0);
        const size_t bytes = static_cast<size_t>(nl) * line_bytes;
        const int slot = static_cast<int>(hs.next++ % kHostSlots);
        unsigned char* a = hs.mem + static_cast<size_t>(slot) * 2 * hs.slot_bytes;
        unsigned char* b = a + hs.slot_bytes;
        if (hs.pending[slot]) check(cudaStreamWaitEvent(hs.h2d, hs.freed[slot], 0), "cudaStreamWaitEvent");
        check(cudaMemcpyAsync(a, src + l0 * line_bytes, bytes, cudaMemcpyHostToDevice, hs.h2d), "copy in");
        check(cudaEventRecord(hs.loaded[slot], hs.h2d), "cudaEventRecord");
        check(cudaStreamWaitEvent(stream, hs.loaded[slot], 0), "cudaStreamWaitEvent");
        unsigned char* cur = a;
        for (uint32_t i = 0; i < count; ++i) {
            auto* p = static_cast<DevicePlan*>(stages[i].plan);
            if (p->spec.req.in_place) {
                execute_plan(p, cur, cur, stream, nl, stages[i].direction, stages[i].normalization);
            } else {
                unsigned char* other = cur == a ? b : a;
                execute_plan(p, cur, other, stream, nl, stages[i].direction, stages[i].normalization);
                cur = other;
            }
        }
        check(cudaEventRecord(hs.computed[slot], stream), "cudaEventRecord");
        check(cudaStreamWaitEvent(hs.d2h, hs.computed[slot], 0), "cudaStreamWaitEvent");
        check(cudaMemcpyAsync(dst + l0 * line_bytes, cur, bytes, cudaMemcpyDeviceToHost, hs.d2h), "copy out");
        check(cudaEventRecord(hs.freed[slot], hs.d2h), "cudaEventRecord");
        hs.pending[slot] = true;
        last = slot;
    }
    // the caller's stream completes after the last copy-out (copy-outs run in order)
    if (last >= 0) check(cudaStreamWaitEvent(stream, hs.freed[last], 0), "cudaStreamWaitEvent");
}

// ---------------------------------------------------------------- autotuner
struct Knobs {
    const char* name;
    bool no_fixed, no_piped, no_cluster;
    int cluster_p, force_w, force_maxv;
    bool use_tma;
    int force_n1;
};

std::string tune_key(const PlanRequest& r, int device) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    std::ostringstream k;
    k << prop.name << "|" << (r.dbl ? "z" : (r.split_bf16 ? "c-tc" : "c")) << "|" << (r.in_place ? "ip" : "oop")
      << "|b" << r.batch;
    for (auto v : r.shape) k << "|" << v;
    if (r.skip_axes) k << "|skip" << r.skip_axes;
    if (r.cluster_pipe) k << "|cpipe";
    return k.str();
}

// Decisions survive the process when SYCLFFT_B200_TUNE_CACHE names a file (one line per key).
std::map<std::string, std::string>& tune_cache() {
    static std::map<std::string, std::string> cache;
    static bool loaded = false;
    if (!loaded) {
        loaded = true;
        if (const char* path = std::getenv("SYCLFFT_B200_TUNE_CACHE")) {
            std::ifstream in(path);
            std::string key, value;
            while (std::getline(in, key, '\t') && std::getline(in, value)) cache[key] = value;
        }
    }
    return cache;
}

// Device time of one execute of a candidate plan on the tuning stream `s` (best of 3 x 3).
float time_candidate(DevicePlan* plan, int64_t batch, void* a, void* b, cudaStream_t s) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    void* out = plan->spec.req.in_place ? a : b;
    float best = 1e30f;
    try {
        for (int i = 0; i < 2; ++i) execute_plan(plan, a, out, s, static_cast<uint64_t>(batch));
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0, s);
            for (int i = 0; i < 3; ++i) execute_plan(plan, a, out, s, static_cast<uint64_t>(batch));
            cudaEventRecord(e1, s);
            check(cudaEventSynchronize(e1), "autotune timing");
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            best = std::min(best, ms / 3);
        }
    } catch (...) {
        best = 1e30f;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

PlanRequest apply(PlanRequest r, const Knobs& k) {
    r.no_fixed = k.no_fixed;
    r.no_piped = k.no_piped;
    r.no_cluster = k.no_cluster;
    r.cluster_p = k.cluster_p;
    r.force_w = k.force_w;
    r.force_maxv = k.force_maxv;
    r.use_tma = k.use_tma || r.use_tma;
    if (k.force_n1) r.force_n1 = k.force_n1;
    return r;
}

PlanRequest tune(const PlanRequest& req, int device, std::string* report) {
    static const Knobs kCandidates[] = {
        {"default", false, false, false, 0, 0, 0, false},    {"generic", true, false, false, 0, 0, 0, false},
        {"no_pipeline", false, true, false, 0, 0, 0, false}, {"cluster8", false, false, false, 8, 0, 0, false},
        {"cluster16", false, false, false, 16, 0, 0, false}, {"w1", false, false, false, 0, 1, 0, false},
        {"w2", false, false, false, 0, 2, 0, false},         {"w4", false, false, false, 0, 4, 0, false},
        {"maxv16", true, false, false, 0, 0, 16, false},     {"tma", false, false, false, 0, 0, 0, true},
        {"split64", false, false, false, 0, 0, 0, false, 64},   {"split128", false, false, false, 0, 0, 0, false, 128},
        {"split256", false, false, false, 0, 0, 0, false, 256}, {"split512", false, false, false, 0, 0, 0, false, 512},
        {"split1024", false, false, false, 0, 0, 0, false, 1024},
    };
    // one tuner at a time in the process: the cache is shared, and concurrent timings would
    // measure each other
    static std::mutex tune_mu;
    std::lock_guard<std::mutex> tune_lock(tune_mu);
    const std::string key = tune_key(req, device);
    auto& cache = tune_cache();
    auto hit = cache.find(key);
    if (hit != cache.end()) {
        for (const auto& k : kCandidates)
            if (hit->second == k.name) {
                *report = std::string("{\"choice\":\"") + k.name + "\",\"cached\":true}";
                return apply(req, k);
            }
    }
    const size_t cs = req.dbl ? 16 : 8;
    const uint64_t elements = checked_element_count(req.shape, req.batch);
    const uint64_t per = elements / req.batch;
    // time on at most ~256 MB per buffer: a sub-batch has the same per-line kernel behaviour
    const int64_t batch = static_cast<int64_t>(std::max<uint64_t>(1, std::min<uint64_t>(req.batch, (uint64_t(256) << 20) / (per * cs))));
    // Everything runs on a private stream, stream-ordered (cudaMallocAsync, cudaFreeAsync): a
    // tuning plan made inside a busy process waits for its own work, not for the device.
    cudaStream_t ts = nullptr;
    check(cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking), "cudaStreamCreate(autotune)");
    void *a = nullptr, *b = nullptr;
    cudaError_t ae = cudaMallocAsync(&a, batch * per * cs, ts);
    if (ae == cudaSuccess) ae = cudaMallocAsync(&b, batch * per * cs, ts);
    if (ae == cudaSuccess) ae = cudaMemsetAsync(a, 0, batch * per * cs, ts);
    if (ae != cudaSuccess) {
        if (a) cudaFreeAsync(a, ts);
        if (b) cudaFreeAsync(b, ts);
        cudaStreamSynchronize(ts);
        cudaStreamDestroy(ts);
        throw std::runtime_error(std::string("autotune buffers: ") + cudaGetErrorString(ae));
    }
    std::ostringstream rep;
    rep << "{\"timed_batch\":" << batch << ",\"candidates\":{";
    std::string best_name = "default";
    float best = 1e30f;
    std::vector<std::string> seen;
    bool first = true;
    for (const auto& k : kCandidates) {
        PlanRequest r = apply(req, k);
        std::string desc;
        try {
            PlanRequest rd = r;
            rd.device_spectrum = true;  // the description does not need the chirp spectra
            desc = describe_plan(make_plan(rd));
        } catch (...) {
            continue;
        }
        if (std::find(seen.begin(), seen.end(), desc) != seen.end()) continue;  // same kernels as an earlier one
        seen.push_back(desc);
        std::unique_ptr<DevicePlan> p;
        try {
            p.reset(build_plan(r, device, SYCLFFT_B200_CREATE_SYNC, ""));
        } catch (...) {
            continue;
        }
        const float ms = time_candidate(p.get(), batch, a, b, ts);
        rep << (first ? "" : ",") << "\"" << k.name << "\":" << ms;
        first = false;
        if (ms < best) {
            best = ms;
            best_name = k.name;
        }
    }
    cudaFreeAsync(a, ts);
    cudaFreeAsync(b, ts);
    cudaStreamSynchronize(ts);
    cudaStreamDestroy(ts);
    rep << "},\"choice\":\"" << best_name << "\"}";
    *report = rep.str();
    cache[key] = best_name;
    if (const char* path = std::getenv("SYCLFFT_B200_TUNE_CACHE")) {
        std::ofstream out(path, std::ios::app);
        out << key << '\t' << best_name << '\n';
    }
    for (const auto& k : kCandidates)
        if (best_name == k.name) return apply(req, k);
    return req;
}

int p_supports(int32_t device, char* err, size_t cap) {
    try {
        int count = 0;
        check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        if (device < 0) check(cudaGetDevice(&device), "cudaGetDevice");
        if (device >= count) throw std::runtime_error("CUDA device ordinal out of range");
        cudaDeviceProp prop{};
        check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        if (prop.major != 10 || prop.minor != 0)
            throw std::runtime_error(std::string("B200 provider needs an sm_100 device, found ") + prop.name);
        return 1;
    } catch (const std::exception& e) {
        set_error(err, cap, e.what());
        return 0;
    }
}

void* p_create(const syclfft_b200_plan_config_v1* cfg, char* err, size_t cap) {
    try {
        if (!cfg) throw std::invalid_argument("null plan configuration");
        return create_plan(*cfg, SYCLFFT_B200_CREATE_SYNC);
    } catch (const std::exception& e) {
        set_error(err, cap, e.what());
        return nullptr;
    }
}

void p_destroy(void* plan) { delete static_cast<DevicePlan*>(plan); }

int p_execute(void* plan, const void* in, void* out, void* stream, char* err, size_t cap) {
    try {
        execute_plan(static_cast<DevicePlan*>(plan), in, out, static_cast<cudaStream_t>(stream));
        return 0;
    } catch (const std::exception& e) {
        set_error(err, cap, e.what());
        return 1;
    }
}

uint64_t p_scratch_bytes(const void* plan) {
    const auto* p = static_cast<const DevicePlan*>(plan);
    return p ? p->spec.scratch_elements * (p->spec.req.dbl ? 16u : 8u) : 0;
}

const syclfft_b200_provider_v1 kProvider{
    SYCLFFT_B200_PROVIDER_ABI_VERSION, "b200", &p_supports, &p_create, &p_destroy, &p_execute, &p_scratch_bytes,
};

}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT const syclfft_b200_provider_v1* syclfft_b200_get_provider_v1(void) { return &sfb::kProvider; }

SYCLFFT_B200_EXPORT int syclfft_b200_describe_plan(const void* plan, char* buf, size_t cap) {
    const auto* p = static_cast<const sfb::DevicePlan*>(plan);
    if (!p || !buf || cap == 0) return -1;
    std::string s;
    if (p && p->real_md) {
        std::string shape;
        for (size_t k = 0; k < p->spec.req.shape.size(); ++k)
            shape += (k ? "," : "") + std::to_string(p->spec.req.shape[k]);
        const sfb::DevicePlan* last = p->inner.get();
        s = std::string("{\"real\":\"") + (p->real_kind == SYCLFFT_B200_REAL_R2C ? "r2c" : "c2r") +
            "\",\"n\":" + std::to_string(p->real_n) + ",\"shape\":[" + shape + "],\"fused\":" +
            (last->real_fused ? "1" : "0") + ",\"inner\":" + sfb::describe_plan(last->inner->spec) +
            ",\"outer\":" + sfb::describe_plan(p->outer->spec) + "}";
    } else if (p->real_kind) {
        // a real plan: its complex plan of half the length and the pre-/post-process pass
        s = std::string("{\"real\":\"") + (p->real_kind == SYCLFFT_B200_REAL_R2C ? "r2c" : "c2r") +
            "\",\"n\":" + std::to_string(p->real_n) + ",\"fused\":" + (p->real_fused ? "1" : "0") +
            ",\"inner\":" + sfb::describe_plan(p->inner->spec) + "}";
    } else if (p->strided) {
        auto side = [](const sfb::Layout& l, bool contig) {
            std::string r = "{\"strides\":[";
            for (int k = 0; k < l.rank; ++k) r += (k ? "," : "") + std::to_string(l.stride[k]);
            return r + "],\"distance\":" + std::to_string(l.dist) + ",\"contiguous\":" + (contig ? "1" : "0") + "}";
        };
        s = "{\"layout\":{\"in\":" + side(p->in_layout, p->in_contig) + ",\"out\":" +
            side(p->out_layout, p->out_contig) + ",\"interleaved\":" + (p->interleaved ? "1" : "0") +
            "},\"inner\":" + sfb::describe_plan(p->inner->spec) + "}";
    } else {
        s = sfb::describe_plan(p->spec);
        int fused = 0, fusedblue = 0;
        for (size_t i = 0; i + 1 < p->passes.size(); ++i) fused += p->passes[i].fused4 ? 1 : 0;
        for (size_t i = 0; i + 2 < p->passes.size(); ++i) fusedblue += p->passes[i].fusedblue ? 1 : 0;
        if (fused && !s.empty() && s.back() == '}')
            s = s.substr(0, s.size() - 1) + ",\"fused_fourstep\":" + std::to_string(fused) + "}";
        if (fusedblue && !s.empty() && s.back() == '}')
            s = s.substr(0, s.size() - 1) + ",\"fused_bluestein\":" + std::to_string(fusedblue) + "}";
    }
    if (s.size() + 1 > cap) return -1;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return static_cast<int>(s.size());
}

namespace sfb {
namespace {
// Kernel launches of one execute of a complex plan (a fused four-step runs two passes in one).
int pass_launches(const DevicePlan* p) {
    int n = static_cast<int>(p->passes.size());
    for (size_t i = 0; i + 1 < p->passes.size(); ++i) n -= p->passes[i].fused4 ? 1 : 0;
    for (size_t i = 0; i + 2 < p->passes.size(); ++i) n -= p->passes[i].fusedblue ? 2 : 0;
    return n;
}
}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT int syclfft_b200_plan_launches(const void* plan) {
    const auto* p = static_cast<const sfb::DevicePlan*>(plan);
    if (!p) return -1;
    if (p->real_md) {
        const sfb::DevicePlan* last = p->inner.get();
        return (last->real_fused ? 1 : sfb::pass_launches(last->inner.get()) + 1) + sfb::pass_launches(p->outer.get());
    }
    if (p->real_kind) return p->real_fused ? 1 : sfb::pass_launches(p->inner.get()) + 1;
    if (p->strided)
        return sfb::pass_launches(p->inner.get()) +
               (p->interleaved ? 0 : (p->in_contig ? 0 : 1) + (p->out_contig ? 0 : 1));
    return sfb::pass_launches(p);
}

SYCLFFT_B200_EXPORT const char* syclfft_b200_version(void) { return "syclfft-b200 0.1"; }

SYCLFFT_B200_EXPORT void* syclfft_b200_create_ex(const syclfft_b200_plan_config_v1* cfg, uint32_t flags, char* err,
                                                 size_t cap) {
    try {
        if (!cfg) throw std::invalid_argument("null plan configuration");
        return sfb::create_plan(*cfg, flags);
    } catch (const std::exception& e) {
        sfb::set_error(err, cap, e.what());
        return nullptr;
    }
}

SYCLFFT_B200_EXPORT void* syclfft_b200_create_real(const syclfft_b200_plan_config_v1* cfg, int32_t kind, uint32_t flags,
                                                   char* err, size_t cap) {
    try {
        if (!cfg) throw std::invalid_argument("null plan configuration");
        return sfb::create_real_plan(*cfg, kind, flags);
    } catch (const std::exception& e) {
        sfb::set_error(err, cap, e.what());
        return nullptr;
    }
}

SYCLFFT_B200_EXPORT void* syclfft_b200_create_strided(const syclfft_b200_plan_config_v1* cfg,
                                                      const syclfft_b200_layout_v1* layout, uint32_t flags, char* err,
                                                      size_t cap) {
    try {
        if (!cfg || !layout) throw std::invalid_argument("null plan configuration or layout");
        return sfb::create_strided_plan(*cfg, *layout, flags);
    } catch (const std::exception& e) {
        sfb::set_error(err, cap, e.what());
        return nullptr;
    }
}

SYCLFFT_B200_EXPORT int syclfft_b200_execute_batch(void* plan, const void* in, void* out, uint64_t batch, void* stream,
                                                   char* err, size_t cap) {
    try {
        if (batch == 0) throw std::invalid_argument("batch must be non-zero");
        sfb::execute_plan(static_cast<sfb::DevicePlan*>(plan), in, out, static_cast<cudaStream_t>(stream), batch);
        return 0;
    } catch (const std::exception& e) {
        sfb::set_error(err, cap, e.what());
        return 1;
    }
}

SYCLFFT_B200_EXPORT int syclfft_b200_execute_ex(void* plan, const void* in, void* out, uint64_t batch,
                                                int32_t direction, int32_t normalization, void* stream, char* err,
                                                size_t cap) {
    try {
        if (direction != 0 && direction != -1 && direction != 1) throw std::invalid_argument("Invalid FFT direction");
        if (normalization > 3) throw std::invalid_argument("Invalid normalization");
        sfb::execute_plan(static_cast<sfb::DevicePlan*>(plan), in, out, static_cast<cudaStream_t>(stream), batch,
                          direction, normalization);
        return 0;
    } catch (const std::exception& e) {
        sfb::set_error(err, cap, e.what());
        return 1;
    }
}

SYCLFFT_B200_EXPORT void syclfft_b200_release_stream_scratch(void* stream, int32_t device) {
    std::lock_guard<std::mutex> lock(sfb::g_arena_mu);
    auto it = sfb::g_arenas.find({device, static_cast<cudaStream_t>(stream)});
    if (it == sfb::g_arenas.end()) return;
    if (it->second.ptr) {
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != device) cudaSetDevice(device);
        cudaFreeAsync(it->second.ptr, static_cast<cudaStream_t>(stream));  // after the stream's work
        if (prev != device) cudaSetDevice(prev);
    }
    sfb::g_arenas.erase(it);
}

SYCLFFT_B200_EXPORT int syclfft_b200_execute_many(const syclfft_b200_exec_item_v1* items, uint32_t count, void* stream,
                                                  char* err, size_t cap) {
    if (count && !items) {
        sfb::set_error(err, cap, "execute items must be non-null");
        return 1;
    }
    for (uint32_t i = 0; i < count; ++i) {
        const syclfft_b200_exec_item_v1& it = items[i];
        try {
            if (it.direction != 0 && it.direction != -1 && it.direction != 1)
                throw std::invalid_argument("Invalid FFT direction");
            if (it.normalization > 3) throw std::invalid_argument("Invalid normalization");
            sfb::execute_plan(static_cast<sfb::DevicePlan*>(it.plan), it.in, it.out, static_cast<cudaStream_t>(stream),
                              it.batch, it.direction, it.normalization);
        } catch (const std::exception& e) {
            sfb::set_error(err, cap, "execute item " + std::to_string(i) + ": " + e.what());
            return 1;
        }
    }
    return 0;
}

namespace sfb {
namespace {
// Every plan of a plan tree (a real or strided plan holds its complex plans in inner / outer).
template <class F>
void for_each_plan(DevicePlan* p, F&& f) {
    if (!p) return;
    f(p);
    for_each_plan(p->inner.get(), f);
    for_each_plan(p->outer.get(), f);
}

// First non-zero status word of the tree; with `clear`, every word is reset to 0.
int read_status(DevicePlan* p, bool clear) {
    int value = 0;
    for_each_plan(p, [&](DevicePlan* q) {
        if (!q->status) return;
        const int v = clear ? __atomic_exchange_n(q->status, 0, __ATOMIC_SEQ_CST)
                            : __atomic_load_n(q->status, __ATOMIC_SEQ_CST);
        if (!value) value = v;
    });
    return value;
}
}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT int syclfft_b200_execute_host(const syclfft_b200_host_stage_v1* stages, uint32_t count,
                                                  const void* in, void* out, uint64_t batch, void* stream, char* err,
                                                  size_t cap) {
    try {
        sfb::execute_host(stages, count, in, out, batch, static_cast<cudaStream_t>(stream));
        return 0;
    } catch (const std::exception& e) {
        sfb::set_error(err, cap, e.what());
        return 1;
    }
}

SYCLFFT_B200_EXPORT uint64_t syclfft_b200_plan_device_bytes(const void* plan) {
    auto* p = const_cast<sfb::DevicePlan*>(static_cast<const sfb::DevicePlan*>(plan));
    if (!p) return 0;
    uint64_t bytes = 0;
    sfb::for_each_plan(p, [&](sfb::DevicePlan* q) {
        const size_t cs = q->spec.req.dbl ? 16 : 8;
        bytes += q->table_bytes;
        if (q->scratch) bytes += q->spec.scratch_elements * cs;
    });
    return bytes;
}

SYCLFFT_B200_EXPORT int syclfft_b200_plan_status(const void* plan) {
    auto* p = const_cast<sfb::DevicePlan*>(static_cast<const sfb::DevicePlan*>(plan));
    if (!p || !p->status) return -1;
    return sfb::read_status(p, false);
}

SYCLFFT_B200_EXPORT int syclfft_b200_plan_take_status(void* plan) {
    auto* p = static_cast<sfb::DevicePlan*>(plan);
    if (!p || !p->status) return -1;
    return sfb::read_status(p, true);
}

SYCLFFT_B200_EXPORT int syclfft_b200_plan_set_wait_limit(void* plan, int64_t polls) {
    auto* p = static_cast<sfb::DevicePlan*>(plan);
    if (!p) return -1;
    const long long v = polls < 0 ? sfb::kSpinLimit : static_cast<long long>(polls);
    sfb::for_each_plan(p, [&](sfb::DevicePlan* q) {
        std::lock_guard<std::mutex> lock(q->mu);
        q->wait_polls = v;
    });
    return 0;
}
