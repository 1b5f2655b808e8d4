// Dispatch from a planned pass to the kernel instantiation that runs it.
#include "launch.hpp"

namespace sfb {

cudaError_t launch_f32_plain(const PassParams&, int, int, int, size_t, const void*, void*, cudaStream_t);
cudaError_t launch_f32_full(const PassParams&, int, int, int, size_t, const void*, void*, cudaStream_t);
cudaError_t launch_f64_plain(const PassParams&, int, int, int, size_t, const void*, void*, cudaStream_t);
cudaError_t launch_f64_full(const PassParams&, int, int, int, size_t, const void*, void*, cudaStream_t);

bool needs_full(const PassParams& p) {
    return p.premul || p.pointwise || p.postmul || p.tw4_sign != 0 || p.fft2.nstages > 0 || p.store_via_smem ||
           p.in_len < p.n || p.out_len < p.n || p.g_k != 1 || p.sel_mode != kSelNone;
}

bool has_variant(bool dbl, int maxv, int maxt) {
    if (maxt != 256 && maxt != 512 && maxt != 1024) return false;
    if (!dbl) return maxv == 16;
    if (maxv == 8) return true;
    return maxv == 16 && maxt <= 512;
}

cudaError_t launch_pass(const PassParams& p, bool dbl, int maxv, int maxt, int threads, size_t smem,
                        const void* in, void* out, cudaStream_t stream) {
    const bool full = needs_full(p);
    if (!dbl) {
        return full ? launch_f32_full(p, maxv, maxt, threads, smem, in, out, stream)
                    : launch_f32_plain(p, maxv, maxt, threads, smem, in, out, stream);
    }
    return full ? launch_f64_full(p, maxv, maxt, threads, smem, in, out, stream)
                : launch_f64_plain(p, maxv, maxt, threads, smem, in, out, stream);
}

}  // namespace sfb
