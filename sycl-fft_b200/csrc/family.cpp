// Radix-family execution API: one launch for requests of several lengths of one radix family
// (include/syclfft_b200_provider.h, syclfft_b200_family_*).
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/syclfft_b200_provider.h"
#include "family_launch.hpp"
#include "planner.hpp"

namespace sfb {
namespace {

struct DeviceFamily {
    int device = 0;
    bool dbl = false;
    void* tw = nullptr;                // base twiddles of every length, concatenated
    std::vector<size_t> tw_off;        // byte offset of length 2^(6+k)
    ~DeviceFamily() {
        if (tw) cudaFree(tw);
    }
};

void set_error(char* err, size_t cap, const std::string& msg) {
    if (!err || cap == 0) return;
    const size_t n = msg.size() < cap - 1 ? msg.size() : cap - 1;
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

int family_log2(bool dbl, uint64_t n) {
    if (n < 64 || (n & (n - 1))) return -1;
    int l = 0;
    while ((uint64_t(1) << l) < n) ++l;
    return l <= (dbl ? 11 : 12) ? l : -1;
}

}  // namespace
}  // namespace sfb

SYCLFFT_B200_EXPORT int syclfft_b200_family_supports(uint32_t scalar, uint64_t n) {
    if (scalar != SYCLFFT_B200_SCALAR_FLOAT && scalar != SYCLFFT_B200_SCALAR_DOUBLE) return 0;
    return sfb::family_log2(scalar == SYCLFFT_B200_SCALAR_DOUBLE, n) >= 0 ? 1 : 0;
}

SYCLFFT_B200_EXPORT void* syclfft_b200_family_create(uint32_t scalar, int32_t device, char* err, size_t cap) {
    using namespace sfb;
    try {
        if (scalar != SYCLFFT_B200_SCALAR_FLOAT && scalar != SYCLFFT_B200_SCALAR_DOUBLE)
            throw std::invalid_argument("unsupported scalar type");
        auto f = std::make_unique<DeviceFamily>();
        f->dbl = scalar == SYCLFFT_B200_SCALAR_DOUBLE;
        int prev = 0;
        check(cudaGetDevice(&prev), "cudaGetDevice");
        f->device = device < 0 ? prev : device;
        // base twiddles W_(ns*R)^jm of every length's stages, generated in FP64
        std::vector<unsigned char> blob;
        for (int l = 6; l <= (f->dbl ? 11 : 12); ++l) {
            blob.resize((blob.size() + 255) / 256 * 256, 0);
            f->tw_off.push_back(blob.size());
            int r[kMaxStages];
            const int ns_count = family_radices(f->dbl, l, r);
            int64_t ns = 1;
            for (int s = 0; s < ns_count; ++s) {
                for (int64_t jm = 0; jm < ns; ++jm) {
                    const auto v = cis_neg(jm, ns * r[s]);
                    if (f->dbl) {
                        double d[2] = {v.real(), v.imag()};
                        blob.insert(blob.end(), reinterpret_cast<unsigned char*>(d),
                                    reinterpret_cast<unsigned char*>(d) + 16);
                    } else {
                        float x[2] = {static_cast<float>(v.real()), static_cast<float>(v.imag())};
                        blob.insert(blob.end(), reinterpret_cast<unsigned char*>(x),
                                    reinterpret_cast<unsigned char*>(x) + 8);
                    }
                }
                ns *= r[s];
            }
        }
        if (f->device != prev) check(cudaSetDevice(f->device), "cudaSetDevice");
        // The copy is waited for on a stream of its own: a synchronous cudaMemcpy from pageable
        // memory can return before its DMA reaches the device, and the launches that read these
        // tables run on non-blocking streams, which are not ordered after it.
        cudaError_t e = cudaMalloc(&f->tw, blob.size());
        cudaStream_t up = nullptr;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMemcpyAsync(f->tw, blob.data(), blob.size(), cudaMemcpyHostToDevice, up);
        if (e == cudaSuccess) e = cudaStreamSynchronize(up);
        if (up) cudaStreamDestroy(up);
        if (f->device != prev) cudaSetDevice(prev);
        check(e, "family tables");
        return f.release();
    } catch (const std::exception& ex) {
        set_error(err, cap, ex.what());
        return nullptr;
    }
}

SYCLFFT_B200_EXPORT void syclfft_b200_family_destroy(void* family) {
    auto* f = static_cast<sfb::DeviceFamily*>(family);
    if (!f) return;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != f->device) cudaSetDevice(f->device);
    cudaDeviceSynchronize();  // queued launches may still read the tables
    const int device = f->device;
    delete f;
    if (prev != device) cudaSetDevice(prev);
}

SYCLFFT_B200_EXPORT int syclfft_b200_family_execute(void* family, const syclfft_b200_family_item_v1* items,
                                                    uint32_t count, void* stream, char* err, size_t cap) {
    using namespace sfb;
    try {
        auto* f = static_cast<DeviceFamily*>(family);
        if (!f || (!items && count)) throw std::invalid_argument("invalid family execution argument");
        const size_t cs = f->dbl ? 16 : 8;
        for (uint32_t i = 0; i < count; ++i) {
            const auto& it = items[i];
            if (!it.in || !it.out || it.batch == 0 || (it.direction != -1 && it.direction != 1) ||
                it.normalization > 3 || family_log2(f->dbl, it.n) < 0)
                throw std::invalid_argument("invalid family request " + std::to_string(i));
            if ((reinterpret_cast<uintptr_t>(it.in) | reinterpret_cast<uintptr_t>(it.out)) % cs)
                throw std::invalid_argument("buffers must be aligned to the complex element size");
        }
        int prev = 0;
        check(cudaGetDevice(&prev), "cudaGetDevice");
        if (prev != f->device) check(cudaSetDevice(f->device), "cudaSetDevice");
        const int per = f->dbl ? 8 : 16;
        uint32_t done = 0;
        cudaError_t e = cudaSuccess;
        while (done < count && e == cudaSuccess) {
            auto p = std::make_unique<FamilyParams>();
            int64_t tiles = 0;
            int k = 0;
            for (; k < kFamilyMaxItems && done + k < count; ++k) {
                const auto& it = items[done + k];
                const int l = family_log2(f->dbl, it.n);
                const int w = kFamilyThreads / static_cast<int>(it.n / per);
                FamilyItem& d = p->items[k];
                d.in = it.in;
                d.out = it.out;
                d.tw = static_cast<const unsigned char*>(f->tw) + f->tw_off[l - 6];
                d.lines = static_cast<int64_t>(it.batch);
                d.tile_begin = tiles;
                d.scale = normalization_scale(static_cast<int>(it.normalization), it.direction, it.n);
                d.conj = it.direction == 1 ? 1 : 0;
                d.log2n = l;
                tiles += (d.lines + w - 1) / w;
            }
            p->count = k;
            e = launch_family(f->dbl, *p, tiles, static_cast<cudaStream_t>(stream));
            done += k;
        }
        if (prev != f->device) cudaSetDevice(prev);
        check(e, "family launch");
        return 0;
    } catch (const std::exception& ex) {
        set_error(err, cap, ex.what());
        return 1;
    }
}
