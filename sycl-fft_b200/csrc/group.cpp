// Grouped execution API: one launch for many requests of a length family
// (include/syclfft_b200_provider.h, syclfft_b200_group_*).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/syclfft_b200_provider.h"
#include "grouped_launch.hpp"
#include "planner.hpp"

namespace sfb {
namespace {

struct DeviceGroup {
    int device = 0;
    bool dbl = false;
    int n = 0;
    const FixedEntry* entry = nullptr;
    int w = 1;
    int threads = 0;
    size_t smem = 0;
    void* tw = nullptr;
    ~DeviceGroup() {
        if (tw) cudaFree(tw);
    }
};

void set_error(char* err, size_t cap, const std::string& msg) {
    if (!err || cap == 0) return;
    const size_t n = std::min(cap - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

int kpitch_of(int n, bool dbl) {
    int p = n + (n >> (dbl ? 3 : 4));
    return (p & 1) ? p : p + 1;
}

}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT int syclfft_b200_group_supports(uint32_t scalar, uint64_t n) {
    return sfb::find_fixed(scalar == SYCLFFT_B200_SCALAR_DOUBLE, sfb::kModeK, static_cast<int>(std::min<uint64_t>(n, 1u << 30)),
                           sfb::kFixedPlain) != nullptr
               ? 1
               : 0;
}

SYCLFFT_B200_EXPORT void* syclfft_b200_group_create(uint32_t scalar, uint64_t n, int32_t device, char* err,
                                                    size_t cap) {
    using namespace sfb;
    try {
        if (scalar != SYCLFFT_B200_SCALAR_FLOAT && scalar != SYCLFFT_B200_SCALAR_DOUBLE)
            throw std::invalid_argument("unsupported scalar type");
        auto g = std::make_unique<DeviceGroup>();
        g->dbl = scalar == SYCLFFT_B200_SCALAR_DOUBLE;
        g->n = static_cast<int>(n);
        g->entry = find_fixed(g->dbl, kModeK, g->n, kFixedPlain);
        if (!g->entry || n > (1u << 20)) throw std::invalid_argument("no grouped kernel for this length");
        int prev = 0;
        check(cudaGetDevice(&prev), "cudaGetDevice");
        g->device = device < 0 ? prev : device;
        if (g->device != prev) check(cudaSetDevice(g->device), "cudaSetDevice");
        const int cs = g->dbl ? 16 : 8;
        const int tpl = g->entry->tpl;
        int w = std::max(1, 256 / tpl);
        while (w > 1 && (w * tpl > g->entry->maxt || static_cast<int64_t>(w) * kpitch_of(g->n, g->dbl) * cs > 227 * 1024))
            --w;
        g->w = w;
        g->threads = (w * tpl + 31) / 32 * 32;
        g->smem = static_cast<size_t>(w) * kpitch_of(g->n, g->dbl) * cs;
        // base twiddles of the family's radix sequence, generated in FP64
        std::vector<unsigned char> blob;
        int64_t ns = 1;
        for (int s = 0; s < g->entry->nstages; ++s) {
            const int R = g->entry->radices[s];
            for (int64_t jm = 0; jm < ns; ++jm) {
                const auto v = cis_neg(jm, ns * R);
                if (g->dbl) {
                    double d[2] = {v.real(), v.imag()};
                    blob.insert(blob.end(), reinterpret_cast<unsigned char*>(d), reinterpret_cast<unsigned char*>(d) + 16);
                } else {
                    float f[2] = {static_cast<float>(v.real()), static_cast<float>(v.imag())};
                    blob.insert(blob.end(), reinterpret_cast<unsigned char*>(f), reinterpret_cast<unsigned char*>(f) + 8);
                }
            }
            ns *= R;
        }
        if (blob.empty()) blob.resize(16, 0);
        // The copy is waited for on a stream of its own: a synchronous cudaMemcpy from pageable
        // memory can return before its DMA reaches the device, and the launches that read these
        // tables run on non-blocking streams, which are not ordered after it.
        cudaError_t e = cudaMalloc(&g->tw, blob.size());
        cudaStream_t up = nullptr;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMemcpyAsync(g->tw, blob.data(), blob.size(), cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess) e = cudaStreamSynchronize(up);
        if (up) cudaStreamDestroy(up);
        if (g->device != prev) cudaSetDevice(prev);
        check(e, "group tables");
        return g.release();
    } catch (const std::exception& ex) {
        set_error(err, cap, ex.what());
        return nullptr;
    }
}

SYCLFFT_B200_EXPORT void syclfft_b200_group_destroy(void* group) {
    auto* g = static_cast<sfb::DeviceGroup*>(group);
    if (!g) return;
    const int device = g->device;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    cudaDeviceSynchronize();  // the group's table may still be read by queued launches
    delete g;
    if (prev != device) cudaSetDevice(prev);
}

SYCLFFT_B200_EXPORT int syclfft_b200_group_execute(void* group, const syclfft_b200_group_item_v1* items,
                                                   uint32_t count, void* stream, char* err, size_t cap) {
    using namespace sfb;
    try {
        auto* g = static_cast<DeviceGroup*>(group);
        if (!g || (!items && count)) throw std::invalid_argument("invalid grouped execution argument");
        int prev = 0;
        check(cudaGetDevice(&prev), "cudaGetDevice");
        if (prev != g->device) check(cudaSetDevice(g->device), "cudaSetDevice");
        uint32_t done = 0;
        cudaError_t e = cudaSuccess;
        while (done < count && e == cudaSuccess) {
            GroupParams p{};
            p.tw = g->tw;
            p.w = g->w;
            p.pitch = g->n;
            int64_t tiles = 0;
            int k = 0;
            for (; k < kGroupMaxItems && done + k < count; ++k) {
                const auto& it = items[done + k];
                if (!it.in || !it.out || it.batch == 0 || (it.direction != -1 && it.direction != 1) ||
                    it.normalization > 3)
                    throw std::invalid_argument("invalid grouped request " + std::to_string(done + k));
                GroupItem& d = p.items[k];
                d.in = it.in;
                d.out = it.out;
                d.lines = static_cast<int64_t>(it.batch);
                d.tile_begin = tiles;
                d.scale = normalization_scale(static_cast<int>(it.normalization), it.direction,
                                              static_cast<uint64_t>(g->n));
                d.conj = it.direction == 1 ? 1 : 0;
                tiles += (d.lines + g->w - 1) / g->w;
            }
            p.count = k;
            e = launch_grouped(g->entry->id, p, tiles, g->threads, g->smem, static_cast<cudaStream_t>(stream));
            done += k;
        }
        if (prev != g->device) cudaSetDevice(prev);
        check(e, "grouped launch");
        return 0;
    } catch (const std::exception& ex) {
        set_error(err, cap, ex.what());
        return 1;
    }
}
