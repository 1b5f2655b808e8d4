// Long-line complex<float> FFT that allocates nothing.
//
// Some callers cannot allocate device memory when they need a transform: a framework
// whose memory planner owns every byte of the device and hands out only the buffers it
// planned, a real-time loop that must not call cudaMalloc (it can synchronize the whole
// device), or a process that gave all free memory to its own pool. The plan API
// allocates its twiddle tables and four-step scratch at plan creation; this entry point
// instead keeps both in file-scope device arrays of fixed size that every GPU loading
// the library holds until the process exits.
//
// It runs the same two size-specialised four-step passes as a plan for these lengths:
// a column pass (input -> scratch, four-step twiddle fused) and a row pass (scratch ->
// output, transposed store, normalization fused), preceded by a small kernel that writes
// this length's twiddles into the table array. Limits: lengths 2^15 .. 2^20 and at most
// kNoAllocMaxElements (4 Mi complex<float>, 32 MiB) elements per call.
//
// Every call shares the two arrays and they keep the last call's contents. The column
// pass overwrites every scratch element the row pass reads, so nothing has to start at
// zero. Calls that overlap on the GPU (different streams, no ordering between them) race
// on the arrays. The first call on a device looks up the arrays' device addresses
// (cudaGetSymbolAddress, with that device current) and the device's shared-memory limit;
// make that first call before any stream capture (a first call made while the stream is
// capturing is refused with an error, and a later call retries the lookup).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/syclfft_b200_provider.h"
#include "fixed_launch.hpp"
#include "planner.hpp"

namespace sfb {
namespace {

constexpr int64_t kNoAllocMaxElements = int64_t(1) << 22;  // 32 MiB of complex<float>
constexpr int kNoAllocMaxTable = 8192;                      // complex<float> twiddle entries
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocMaxElements];
static __device__ __align__(256) float2 g_noalloc_tables[kNoAllocMaxTable];

struct DeviceArrays {
    float2* scratch = nullptr;
    float2* tables = nullptr;
    int smem_optin = 0;  // cudaDevAttrMaxSharedMemoryPerBlockOptin
    bool ready = false;
};
DeviceArrays g_arrays[kMaxDevices];
std::mutex g_arrays_mu[kMaxDevices];

// Device addresses of the two arrays and the shared-memory limit of the current device
// `dev`, looked up on the first successful call and kept; a failed lookup is not kept, so
// a later call tries again.
cudaError_t device_arrays(int dev, cudaStream_t st, DeviceArrays* out, std::string* why) {
    std::lock_guard<std::mutex> lock(g_arrays_mu[dev]);
    DeviceArrays& a = g_arrays[dev];
    if (!a.ready) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cudaError_t e = cudaStreamIsCapturing(st, &cap);
        if (e != cudaSuccess) {
            *why = "cudaStreamIsCapturing";
            return e;
        }
        if (cap != cudaStreamCaptureStatusNone) {
            *why = "the first no-allocation call on a device must not be made while its stream is capturing";
            return cudaErrorStreamCaptureUnsupported;
        }
        DeviceArrays t;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&t.scratch), g_noalloc_scratch);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(reinterpret_cast<void**>(&t.tables), g_noalloc_tables);
        if (e != cudaSuccess) {
            *why = "cudaGetSymbolAddress";
            return e;
        }
        e = cudaDeviceGetAttribute(&t.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) {
            *why = "cudaDeviceGetAttribute";
            return e;
        }
        t.ready = true;
        a = t;
    }
    *out = a;
    return cudaSuccess;
}

// exp(-2 pi i num / den) in double, stored as float.
__device__ float2 cis_neg_f(long long num, long long den) {
    long long m = num % den;
    if (m < 0) m += den;
    double s, c;
    sincospi(2.0 * static_cast<double>(m) / static_cast<double>(den), &s, &c);
    return make_float2(static_cast<float>(c), static_cast<float>(-s));
}

struct TableJob {
    int n1, n2, nr1, nr2;
    int r1[kMaxStages], r2[kMaxStages];
    int off2, off_hi, off_lo;  // offsets of the row-stage table and the four-step tables
    int nhi, nlo, shift;
    long long n;
};

// One thread per table entry: stage twiddles of the column FFT, of the row FFT, then the
// two-level four-step twiddle W_N^m = hi[m >> shift] * lo[m & (2^shift - 1)].
__global__ void noalloc_fill_tables(const __grid_constant__ TableJob job, float2* tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    // base twiddles of the size-specialised kernels: per stage, W_(ns*R)^jm for jm < ns
    auto stage_entry = [](int idx, const int* r, int nr, float2* out) -> bool {
        int ns = 1, off = 0;
        for (int s = 0; s < nr; ++s) {
            const int R = r[s];
            if (idx < off + ns) {
                *out = cis_neg_f(idx - off, static_cast<long long>(ns) * R);
                return true;
            }
            off += ns;
            ns *= R;
        }
        return false;
    };
    float2 v;
    if (i < job.off2) {
        if (stage_entry(i, job.r1, job.nr1, &v)) tab[i] = v;
    } else if (i < job.off_hi) {
        if (stage_entry(i - job.off2, job.r2, job.nr2, &v)) tab[i] = v;
    } else if (i < job.off_lo) {
        const int q = i - job.off_hi;
        if (q < job.nhi) tab[i] = cis_neg_f(static_cast<long long>(q) << job.shift, job.n);
    } else if (i < job.off_lo + job.nlo) {
        tab[i] = cis_neg_f(i - job.off_lo, job.n);
    }
}

void set_error(char* err, size_t cap, const std::string& msg) {
    if (!err || cap == 0) return;
    const size_t n = msg.size() < cap - 1 ? msg.size() : cap - 1;
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

int stage_table_size(const FixedEntry& e) {
    int ns = 1, off = 0;
    for (int s = 0; s < e.nstages; ++s) {
        off += ns;
        ns *= e.radices[s];
    }
    return off;
}

int pitch_k(int n) {
    int p = n + (n >> 4);
    return (p & 1) ? p : p + 1;
}

}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT int syclfft_b200_execute_noalloc_c2c_f32(const void* in, void* out, uint64_t n, uint64_t batch,
                                                             int32_t direction, uint32_t normalization,
                                                             void* stream, char* err, size_t cap) {
    using namespace sfb;
    if (!in || !out) {
        set_error(err, cap, "input and output must be non-null device pointers");
        return 1;
    }
    // The kernels move whole float2 elements: an address off an 8-byte boundary would fault
    // on the device and leave the caller's context unusable, so it is refused here.
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) % sizeof(float2)) {
        set_error(err, cap, "input and output must be aligned to 8 bytes (one complex<float>)");
        return 1;
    }
    if (direction != -1 && direction != 1) {
        set_error(err, cap, "Invalid FFT direction");
        return 1;
    }
    if (normalization > 3) {
        set_error(err, cap, "Invalid normalization");
        return 1;
    }
    if (batch == 0 || n == 0) {
        set_error(err, cap, "FFT length and batch count must be non-zero");
        return 1;
    }
    if (n < (1u << 15) || n > (1u << 20) || (n & (n - 1))) {
        set_error(err, cap, "no-allocation FFT supports power-of-two lengths 2^15 .. 2^20, got " + std::to_string(n));
        return 1;
    }
    if (batch > static_cast<uint64_t>(kNoAllocMaxElements) / n) {
        set_error(err, cap, "no-allocation FFT is limited to " + std::to_string(kNoAllocMaxElements) +
                                " complex<float> elements per call (n * batch)");
        return 1;
    }
    // Split n = n1 * n2 over the size-specialised column (twiddle fused) and row
    // (transposed store) kernels; the most balanced split wins.
    const FixedEntry *ec = nullptr, *er = nullptr;
    for (int64_t n1 = 2; n1 * n1 <= static_cast<int64_t>(n); n1 *= 2) {
        if (n % n1) continue;
        const FixedEntry* c = find_fixed(false, kModeC, static_cast<int>(n1), kFixedTw4);
        const FixedEntry* r = find_fixed(false, kModeK, static_cast<int>(n / n1), kFixedTStore);
        if (c && r && n1 % r->w == 0) {
            ec = c;
            er = r;
        }
    }
    if (!ec || !er) {
        set_error(err, cap, "no-allocation FFT has no kernel split for length " + std::to_string(n));
        return 1;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(err, cap, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return 1;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(err, cap, "no-allocation FFT supports device ordinals below " + std::to_string(kMaxDevices) +
                                ", got " + std::to_string(dev));
        return 1;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceArrays arr;
    std::string why;
    e = device_arrays(dev, st, &arr, &why);
    if (e != cudaSuccess) {
        set_error(err, cap, why + ": " + cudaGetErrorString(e));
        return 1;
    }
    const int n1 = ec->n, n2 = er->n;
    const size_t smem_cols = static_cast<size_t>(ec->w) * n1 * sizeof(float2);
    const size_t smem_rows = static_cast<size_t>(er->w) * pitch_k(n2) * sizeof(float2);
    if (smem_cols > static_cast<size_t>(arr.smem_optin) || smem_rows > static_cast<size_t>(arr.smem_optin)) {
        set_error(err, cap, "no-allocation FFT of length " + std::to_string(n) + " needs " +
                                std::to_string(smem_cols > smem_rows ? smem_cols : smem_rows) +
                                " bytes of shared memory per block; this device allows " +
                                std::to_string(arr.smem_optin));
        return 1;
    }
    TableJob job{};
    job.n1 = n1;
    job.n2 = n2;
    job.nr1 = ec->nstages;
    job.nr2 = er->nstages;
    for (int i = 0; i < ec->nstages; ++i) job.r1[i] = ec->radices[i];
    for (int i = 0; i < er->nstages; ++i) job.r2[i] = er->radices[i];
    job.n = static_cast<long long>(n);
    int shift = 0;
    while ((int64_t(1) << (2 * shift)) < static_cast<int64_t>(n)) ++shift;
    job.shift = shift;
    job.nhi = static_cast<int>((n + (uint64_t(1) << shift) - 1) >> shift) + 1;
    job.nlo = 1 << shift;
    auto align64 = [](int v) { return (v + 63) / 64 * 64; };
    job.off2 = align64(stage_table_size(*ec));
    job.off_hi = job.off2 + align64(stage_table_size(*er));
    job.off_lo = job.off_hi + align64(job.nhi);
    const int total = job.off_lo + job.nlo;
    if (total > kNoAllocMaxTable) {
        set_error(err, cap, "no-allocation FFT twiddle table overflow");
        return 1;
    }
    noalloc_fill_tables<<<(total + 255) / 256, 256, 0, st>>>(job, arr.tables);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(err, cap, std::string("table kernel: ") + cudaGetErrorString(e));
        return 1;
    }
    const int64_t N = static_cast<int64_t>(n), B = static_cast<int64_t>(batch);
    const double scale = normalization_scale(static_cast<int>(normalization), direction, n);
    // column pass: in -> scratch, FFT over n1 (stride n2), W_N^(n2*k1) fused
    FixedParams a;
    a.n_cols = n2;
    a.col_tiles = (n2 + ec->w - 1) / ec->w;
    a.w = ec->w;
    a.in_hi = N;
    a.out_hi = N;
    a.in_ks = n2;
    a.out_ks = n2;
    a.tw = arr.tables;
    a.conj_in = direction == 1;
    a.tw4_hi = arr.tables + job.off_hi;
    a.tw4_lo = arr.tables + job.off_lo;
    a.tw4_shift = shift;
    e = launch_fixed(ec->id, false, true, a, ec->w * ec->tpl, smem_cols, B * a.col_tiles, in, arr.scratch, st);
    if (e != cudaSuccess) {
        set_error(err, cap, std::string("column pass: ") + cudaGetErrorString(e));
        return 1;
    }
    // row pass: scratch -> out, FFT over n2, stored transposed at k1 + n1 * k2
    FixedParams b;
    b.n_cols = B * n1;
    b.w = er->w;
    b.col_tiles = (b.n_cols + b.w - 1) / b.w;
    b.in_pitch = n2;
    b.out_pitch = n2;
    b.tw = arr.tables + job.off2;
    b.conj_out = direction == 1;
    b.scale = scale;
    b.rows = n1;
    b.line = N;
    e = launch_fixed(er->id, false, false, b, er->w * er->tpl, smem_rows, b.col_tiles, arr.scratch, out, st);
    if (e != cudaSuccess) {
        set_error(err, cap, std::string("row pass: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}
