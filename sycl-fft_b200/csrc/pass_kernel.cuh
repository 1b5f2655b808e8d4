// The FFT pass kernel: a tile of lines, loaded once from HBM straight into
// registers, transformed by a Stockham sequence of register butterflies that
// exchange through shared memory, and stored once.
//
// Stockham radix-R stage (Ns = product of earlier radices, nr = n / R), for every
// butterfly j in [0, nr):
//     v_r  = x[j + r * nr] * exp(-2 pi i r (j mod Ns) / (Ns R)),   r = 0..R-1
//     v    = DFT_R(v)
//     y[(j - j mod Ns) * R + (j mod Ns) + r * Ns] = v_r
// The first stage reads x[j + r*nr] and the last stage writes y[j + r*nr]: both
// are unit-stride in j, so the first stage loads directly from HBM and the last
// stage stores directly to HBM with coalesced accesses (consecutive threads walk
// j in kModeK, or consecutive columns in kModeC). Only the inner exchanges touch
// shared memory.
#pragma once

#include <cuda_runtime.h>

#include "butterfly.cuh"
#include "pass_params.h"

namespace sfb {

template <class C>
__device__ __forceinline__ C ldg_c(const C* p) {
    return __ldg(p);
}

template <class T>
struct TileCtx {
    using C = cplx<T>;
    C* sm;
    const C* in;
    C* out;
    int w, t;
    bool active;     // thread maps to a (line, lane) of this tile
    bool line_ok;    // the line exists (ragged last tile)
    int64_t in_base, out_base, sel;
    T scale;
};

__device__ __forceinline__ int smem_index(const PassParams& P, int w, int k) {
    return P.mode == kModeK ? w * P.pitch + k + (k >> P.pad_shift) : k * P.w + w;
}

__device__ __forceinline__ int64_t line_base(const LineLayout& L, int64_t o, int64_t c) {
    return (L.d == 1 ? o * L.hi : (o / L.d) * L.hi + (o % L.d) * L.lo) + c * L.cs;
}

// FULL = false compiles the plain-FFT flavour: no zero padding, tables or four-step
// twiddle on load/store (single passes of 7-smooth axes, the common case).
template <class T, bool FULL>
__device__ __forceinline__ cplx<T> load_elem(const PassParams& P, const TileCtx<T>& X, int k) {
    using C = cplx<T>;
    C a = cmake<C>(T(0), T(0));
    if constexpr (FULL) {
        const int64_t g = (int64_t)k * P.g_k + X.sel;
        if (X.line_ok && g < P.in_len) {
            a = X.in[X.in_base + (int64_t)k * P.in.ks];
            if (P.flip_in) a.y = -a.y;
            if (P.premul) a = cmul(a, ldg_c(static_cast<const C*>(P.premul) + g));
            if (P.conj_in) a.y = -a.y;
        }
    } else {
        if (X.line_ok) {
            a = X.in[X.in_base + (int64_t)k * P.in.ks];
            if (P.conj_in) a.y = -a.y;
        }
    }
    return a;
}

template <class T, bool FULL>
__device__ __forceinline__ void store_elem(const PassParams& P, const TileCtx<T>& X, int64_t base,
                                           int64_t sel, int k, cplx<T> v) {
    using C = cplx<T>;
    if constexpr (!FULL) {
        if (P.conj_out) v.y = -v.y;
        v.x *= X.scale;
        v.y *= X.scale;
        X.out[base + (int64_t)k * P.out.ks] = v;
        return;
    }
    const int64_t g = (int64_t)k * P.g_k + sel;
    if (g >= P.out_len) return;
    if (P.conj_out) v.y = -v.y;
    if (P.tw4_sign != 0) {
        const int64_t m = (int64_t)k * sel;
        const C* hi = static_cast<const C*>(P.tw4_hi);
        const C* lo = static_cast<const C*>(P.tw4_lo);
        C w = cmul(ldg_c(hi + (m >> P.tw4_shift)), ldg_c(lo + (m & ((int64_t(1) << P.tw4_shift) - 1))));
        if (P.tw4_sign > 0) w.y = -w.y;
        v = cmul(v, w);
    }
    if (P.postmul) v = cmul(v, ldg_c(static_cast<const C*>(P.postmul) + g));
    v.x *= X.scale;
    v.y *= X.scale;
    if (P.flip_out) v.y = -v.y;
    X.out[base + (int64_t)k * P.out.ks] = v;
}

template <class T>
__device__ __forceinline__ cplx<T> apply_mid(const PassParams& P, const TileCtx<T>& X, int k, cplx<T> v) {
    using C = cplx<T>;
    if (P.pointwise) v = cmul(v, ldg_c(static_cast<const C*>(P.pointwise) + k + X.sel * P.pw_stride));
    if (P.conj_mid) v.y = -v.y;
    return v;
}

enum : int { kSrcSmem = 0, kSrcGlobal = 1 };
enum : int { kDstSmem = 0, kDstSmemMid = 1, kDstGlobal = 2 };

template <int R, class T, int MAXV, bool FULL>
__device__ __forceinline__ void run_stage(const PassParams& P, const StageSeq& S, int s, TileCtx<T>& X,
                                          int src, int dst) {
    using C = cplx<T>;
    constexpr int NB = MAXV / R;
    const int nr = P.n / R;
    const int Ns = S.ns[s];
    C v[NB * R];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = X.t + i * P.tpl;
        if (X.active && j < nr) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int k = j + r * nr;
                v[i * R + r] = (src == kSrcGlobal) ? load_elem<T, FULL>(P, X, k) : X.sm[smem_index(P, X.w, k)];
            }
        }
    }
    if (src == kSrcSmem) __syncthreads();
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = X.t + i * P.tpl;
        if (X.active && j < nr) {
            C* u = &v[i * R];
            const int jm = j % Ns;
            if (R > 1 && Ns > 1) {
                const C* tw = static_cast<const C*>(S.tw) + S.tw_off[s] + jm * (R - 1);
#pragma unroll
                for (int r = 1; r < R; ++r) u[r] = cmul(u[r], ldg_c(tw + (r - 1)));
            }
            dft<R, T>(u);
            const int base = (j - jm) * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int k = base + r * Ns;
                if (dst == kDstGlobal) {
                    if (X.line_ok) store_elem<T, FULL>(P, X, X.out_base, X.sel, k, u[r]);
                } else {
                    if constexpr (FULL) {
                        X.sm[smem_index(P, X.w, k)] = (dst == kDstSmemMid) ? apply_mid<T>(P, X, k, u[r]) : u[r];
                    } else {
                        X.sm[smem_index(P, X.w, k)] = u[r];
                    }
                }
            }
        }
    }
    if (dst != kDstGlobal) __syncthreads();
}

template <int R, class T, int MAXV, bool FULL>
__device__ __forceinline__ void run_group(const PassParams& P, const StageSeq& S, TileCtx<T>& X, bool from_global,
                                          int last_dst, int& s) {
    while (s < S.nstages && S.radix[s] == R) {
        const int src = (s == 0 && from_global) ? kSrcGlobal : kSrcSmem;
        const int dst = (s == S.nstages - 1) ? last_dst : kDstSmem;
        run_stage<R, T, MAXV, FULL>(P, S, s, X, src, dst);
        ++s;
    }
}

// Stages run grouped by radix (16, 8, 4, 2, 3, 5, 7, 1): a Stockham sequence may use its
// radices in any order, and straight-line per-radix loops keep register allocation local
// (a loop over a radix switch does not).
template <class T, int MAXV, bool FULL>
__device__ __forceinline__ void run_seq(const PassParams& P, const StageSeq& S, TileCtx<T>& X, bool from_global,
                                        int last_dst) {
    int s = 0;
    if constexpr (MAXV >= 16) run_group<16, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<8, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<4, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<2, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<3, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<5, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<7, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
    run_group<1, T, MAXV, FULL>(P, S, X, from_global, last_dst, s);
}

// Registers per thread the instantiation is compiled for: the register arrays of a stage
// hold MAXV complex values; 64 registers suffice for 16 float or 8 double values.
template <class T, int MAXV>
constexpr int reg_target() {
    return (sizeof(T) * MAXV > 64) ? 128 : 64;
}

template <class T, int MAXV, int MAXT, bool FULL>
__global__ void __launch_bounds__(MAXT, 65536 / (MAXT * reg_target<T, MAXV>()))
    fft_pass_kernel(const __grid_constant__ PassParams P, const cplx<T>* in, cplx<T>* out) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileCtx<T> X;
    X.sm = reinterpret_cast<C*>(smem_raw);
    X.in = in;
    X.out = out;
    X.scale = static_cast<T>(P.scale);
    const int tid = threadIdx.x;
    if (P.mode == kModeK) {
        X.w = tid / P.tpl;
        X.t = tid - X.w * P.tpl;
        X.active = X.w < P.w;
    } else {
        X.t = tid / P.w;
        X.w = tid - X.t * P.w;
        X.active = X.t < P.tpl;
    }
    // One tile per CTA (a grid-stride tile loop keeps every stage's addressing live across
    // iterations and costs more registers than it saves in launch overhead).
    const int64_t tile = blockIdx.x;
    const int64_t o = tile / P.col_tiles;
    const int64_t c0 = (tile - o * P.col_tiles) * P.w;
    const int64_t c = c0 + X.w;
    X.line_ok = X.active && c < P.n_cols;
    X.in_base = line_base(P.in, o, c);
    X.out_base = line_base(P.out, o, c);
    X.sel = P.sel_mode == kSelCol ? c
            : P.sel_mode == kSelOuterLo ? o % P.sel_d
            : P.sel_mode == kSelColMod  ? c % P.sel_d
                                        : 0;
    if constexpr (!FULL) {
        run_seq<T, MAXV, false>(P, P.fft1, X, true, kDstGlobal);
        return;
    }
    const bool two = P.fft2.nstages > 0;
    const int last1 = two ? kDstSmemMid : (P.store_via_smem ? kDstSmem : kDstGlobal);
    run_seq<T, MAXV, FULL>(P, P.fft1, X, true, last1);
    if (two) run_seq<T, MAXV, FULL>(P, P.fft2, X, false, P.store_via_smem ? kDstSmem : kDstGlobal);
    if (P.store_via_smem) {
        // Transposed store: walk the tile in the output's coalesced order.
        const int total = P.w * P.n;
        const bool col_fast = P.out.cs == 1;
        for (int idx = tid; idx < total; idx += blockDim.x) {
            int w, k;
            if (col_fast) {
                k = idx / P.w;
                w = idx - k * P.w;
            } else {
                w = idx / P.n;
                k = idx - w * P.n;
            }
            const int64_t cc = c0 + w;
            if (cc >= P.n_cols) continue;
            const int64_t sel = P.sel_mode == kSelCol ? cc
                                : P.sel_mode == kSelOuterLo ? o % P.sel_d
                                : P.sel_mode == kSelColMod  ? cc % P.sel_d
                                                            : 0;
            store_elem<T, FULL>(P, X, line_base(P.out, o, cc), sel, k, X.sm[smem_index(P, w, k)]);
        }
    }
}

}  // namespace sfb
