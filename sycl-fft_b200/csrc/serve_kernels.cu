// Serving helpers: deterministic uniform fill of many request buffers in one launch.
//
// A request's synthetic input is 2 * elements reals uniform in [-1, 1) drawn from its seed:
// value i is a function of (seed, i) alone (the SplitMix64 output function of Steele, Lea and
// Flood applied to seed * K1 + i * K2), so the values do not depend on the launch shape and a
// server can fill every request of an admission round with one launch.
#include <climits>
#include <cstdint>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/syclfft_b200_provider.h"

namespace sfb {
namespace {

constexpr int kFillMaxItems = 256;
constexpr int kFillThreads = 256;
constexpr int kFillPerThread = 8;
constexpr int64_t kFillTile = int64_t(kFillThreads) * kFillPerThread;  // reals per block

struct FillItem {
    void* data;
    int64_t count;
    uint64_t seed;
    int64_t tile_begin;
    int dbl;
};

struct FillParams {
    int count;
    FillItem items[kFillMaxItems];
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ull;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(kFillThreads) fill_uniform_kernel(const __grid_constant__ FillParams P) {
    const int64_t tile = blockIdx.x;
    int lo = 0, hi = P.count - 1;  // last item with tile_begin <= tile
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (P.items[mid].tile_begin <= tile) lo = mid;
        else hi = mid - 1;
    }
    const FillItem& it = P.items[lo];
    const int64_t base = (tile - it.tile_begin) * kFillTile;
    const uint64_t s = it.seed * 0xd1b54a32d192ed03ull + 0x632be59bd9b4e019ull;
#pragma unroll
    for (int e = 0; e < kFillPerThread; ++e) {
        const int64_t i = base + int64_t(e) * kFillThreads + threadIdx.x;
        if (i >= it.count) break;
        const uint64_t h = mix64(s + static_cast<uint64_t>(i) * 0x9e3779b97f4a7c15ull);
        if (it.dbl) {
            static_cast<double*>(it.data)[i] = static_cast<double>(h >> 11) * 0x1.0p-52 - 1.0;
        } else {
            static_cast<float*>(it.data)[i] = static_cast<float>(h >> 40) * 0x1.0p-23f - 1.0f;
        }
    }
}

void set_error(char* err, size_t cap, const std::string& m) {
    if (!err || !cap) return;
    const size_t n = m.size() < cap - 1 ? m.size() : cap - 1;
    std::memcpy(err, m.data(), n);
    err[n] = 0;
}

}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT int syclfft_b200_fill_uniform(const syclfft_b200_fill_item_v1* items, uint32_t count,
                                                  void* stream, char* err, size_t cap) {
    using namespace sfb;
    if (count == 0) return 0;
    if (!items) {
        set_error(err, cap, "fill items must be non-null");
        return 1;
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (items[i].count && !items[i].data) {
            set_error(err, cap, "fill item " + std::to_string(i) + ": data must be non-null");
            return 1;
        }
        if (items[i].scalar != SYCLFFT_B200_SCALAR_FLOAT && items[i].scalar != SYCLFFT_B200_SCALAR_DOUBLE) {
            set_error(err, cap, "fill item " + std::to_string(i) + ": scalar must be float or double");
            return 1;
        }
    }
    FillParams P;
    uint32_t i = 0;
    while (i < count) {
        P.count = 0;
        int64_t tiles = 0;
        for (; i < count && P.count < kFillMaxItems; ++i) {
            if (items[i].count == 0) continue;
            FillItem& f = P.items[P.count++];
            f.data = items[i].data;
            f.count = static_cast<int64_t>(items[i].count);
            f.seed = items[i].seed;
            f.dbl = items[i].scalar == SYCLFFT_B200_SCALAR_DOUBLE;
            f.tile_begin = tiles;
            tiles += (f.count + kFillTile - 1) / kFillTile;
        }
        if (P.count == 0) continue;
        if (tiles > INT_MAX) {
            set_error(err, cap, "fill request too large for one launch");
            return 1;
        }
        fill_uniform_kernel<<<static_cast<unsigned>(tiles), kFillThreads, 0, static_cast<cudaStream_t>(stream)>>>(P);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            set_error(err, cap, std::string("fill launch: ") + cudaGetErrorString(e));
            return 1;
        }
    }
    return 0;
}
