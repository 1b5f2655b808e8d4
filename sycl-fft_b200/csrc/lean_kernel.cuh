// Runtime-length pass kernel for contiguous layouts ("lean"): the same Stockham register /
// shared-memory scheme as pass_kernel.cuh for lengths the size-specialised catalog does not
// have (7-smooth lengths with factors 3, 5, 7; a 3 and a 5 stage run as one prime-factor radix
// 15 where 16 values a thread fit), with the layout and the fused feature fixed at
// compile time and the per-element work cut to what the three contiguous cases need:
//   kLeanPlain, kModeK: whole lines, conjugation and scale on load / store;
//   kLeanTw4,   kModeC: four-step column pass, W_L^(k*c) twiddle on the store;
//   kLeanPlain, kModeC: four-step row pass as a column tile (lanes walk adjacent rows, element
//                       stride 1 on load and the transposed element stride on store).
// Element offsets within a line are 32-bit, the butterfly index j mod Ns uses a precomputed
// multiply-shift quotient (ns_magic / ns_shift), each butterfly's R - 1 twiddles are read from
// the stage's table (L1-resident; forming them as powers of one base twiddle in registers
// measured 15-30% slower here, the kernel being bound by its FMA and ALU issue), and no
// padding or second-FFT branch is compiled in.
// Strided layouts and the Bluestein extras stay on fft_pass_kernel.
#pragma once

#include <cuda_runtime.h>

#include "butterfly.cuh"
#include "pass_params.h"

namespace sfb {

enum : int { kLeanPlain = 0, kLeanTw4 = 1 };

struct LeanParams {
    int n = 0, tpl = 1, w = 1, w_shift = 0;  // w: lines per tile, a power of two (w = 1 << w_shift)
    int pitch = 0;                          // kModeK shared-memory line pitch (padding: kLeanPad)
    int nstages = 0;
    int radix[kMaxStages] = {};
    int ns[kMaxStages] = {};
    int tw_off[kMaxStages] = {};
    // j / ns[s] = umulhi(j, ns_magic[s]) >> ns_shift[s]; ns_magic 0: ns[s] = 1 << ns_shift[s]
    uint32_t ns_magic[kMaxStages] = {};
    int ns_shift[kMaxStages] = {};
    const void* tw = nullptr;  // per stage [ns][radix - 1] of W_(ns*radix)^(r*jm)
    int64_t n_cols = 1, col_tiles = 1;
    int64_t in_hi = 0, in_cs = 0, out_hi = 0, out_cs = 0;  // line (o, c) starts at o*hi + c*cs
    int in_ks = 1, out_ks = 1;                             // element stride within a line
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    const void* tw4_hi = nullptr;  // kLeanTw4: W^m = hi[m >> tw4_shift] * lo[m & mask], m = k*c
    const void* tw4_lo = nullptr;
    int tw4_shift = 0, tw4_conj = 0;
};

template <class T>
struct LeanCtx {
    cplx<T>* sm;  // kModeK: this line's row of shared memory; kModeC: this column's base
    const cplx<T>* gin;
    cplx<T>* gout;
    int t, w, c;  // lane within the line, line within the tile, column index (kLeanTw4)
    bool active, line_ok;
};

__device__ __forceinline__ int lean_quot(const LeanParams& P, int s, int j) {
    const uint32_t m = P.ns_magic[s];
    return m ? static_cast<int>(__umulhi(static_cast<uint32_t>(j), m) >> P.ns_shift[s]) : (j >> P.ns_shift[s]);
}

// kModeK rows hold one padding element per 2^kLeanPad (the planner's pad for the precision).
template <class T>
constexpr int kLeanPad = sizeof(T) == 4 ? 4 : 3;

// Four-step twiddle W_L^m = tw4_hi[m >> tw4_shift] * tw4_lo[m & mask] (m = k * c < L).
template <class C>
__device__ __forceinline__ C lean_tw4(const LeanParams& P, int m) {
    return cmul(__ldg(static_cast<const C*>(P.tw4_hi) + (m >> P.tw4_shift)),
                __ldg(static_cast<const C*>(P.tw4_lo) + (m & ((1 << P.tw4_shift) - 1))));
}

template <class T, bool MODEC>
__device__ __forceinline__ int lean_sidx(const LeanParams& P, int k) {
    if constexpr (MODEC) return k << P.w_shift;
    else return k + (k >> kLeanPad<T>);
}

// One radix-R Stockham stage over the tile: first stage loads from HBM, the last stores to HBM,
// inner stages exchange through shared memory.
// Global and column-tile addresses advance by a per-stage step (one add per element; a second
// path for padded line rows whose step is a multiple of the padding unit cost more registers
// than it saved), and the first stage (Ns = 1) and the last (j < Ns) need no quotient.
template <int R, class T, int MAXV, bool MODEC, int FEAT, bool FIRST, bool LAST>
__device__ __forceinline__ void lean_stage(const LeanParams& P, int s, LeanCtx<T>& X) {
    using C = cplx<T>;
    constexpr int NB = MAXV / R;
    const int nr = P.n / R;
    const int Ns = P.ns[s];
    C v[NB * R];
    // loads: element k = j + r * nr
    constexpr bool lin_in = MODEC;
    const int in_step = FIRST ? (MODEC ? nr * P.in_ks : nr) : (MODEC ? nr << P.w_shift : 0);
    [[maybe_unused]] const T in_sy = P.conj_in ? T(-1) : T(1);  // conjugated input: im * -1
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = X.t + i * P.tpl;
        if (X.active && j < nr) {
            if constexpr (FIRST) {
                const C* g = X.gin + (MODEC ? j * P.in_ks : j);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    C a = cmake<C>(T(0), T(0));
                    if (X.line_ok) {
                        a = g[r * in_step];
                        a.y *= in_sy;
                    }
                    v[i * R + r] = a;
                }
            } else if constexpr (lin_in) {
                const C* p = X.sm + lean_sidx<T, MODEC>(P, j);
#pragma unroll
                for (int r = 0; r < R; ++r) v[i * R + r] = p[r * in_step];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) v[i * R + r] = X.sm[lean_sidx<T, MODEC>(P, j + r * nr)];
            }
        }
    }
    if constexpr (!FIRST) __syncthreads();
    constexpr bool to_global = LAST;
    // stores: element k = base + r * Ns (base = j in the last stage)
    constexpr bool lin_out = MODEC;
    const int out_step = to_global ? (MODEC ? nr * P.out_ks : nr) : (MODEC ? Ns << P.w_shift : 0);
    // Output conjugation folded into the scale (and, with the four-step twiddle, into that
    // twiddle's sign: conj(u) * w = conj(u * conj(w))), so the store has no select.
    [[maybe_unused]] const T out_sx = static_cast<T>(P.scale);
    [[maybe_unused]] const T out_sy = P.conj_out ? -out_sx : out_sx;
    [[maybe_unused]] const T tw4_sy = (P.tw4_conj != P.conj_out) ? T(-1) : T(1);
    // The four-step twiddles of one butterfly's outputs k = j + r * nr form a geometric
    // sequence, W^(k*c) = W^(j*c) * (W^(nr*c))^r: one table lookup per butterfly, the step once
    // per thread, then one product per output (at most 14 deep; the last radix is at most 15).
    [[maybe_unused]] C tw4_step = cmake<C>(T(1), T(0));
    if constexpr (LAST && FEAT == kLeanTw4) {
        if (X.line_ok) {
            tw4_step = lean_tw4<C>(P, nr * X.c);
            tw4_step.y *= tw4_sy;
        }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = X.t + i * P.tpl;
        if (X.active && j < nr) {
            C* u = &v[i * R];
            int q, jm;
            if constexpr (FIRST) {
                q = j;
                jm = 0;
            } else if constexpr (LAST) {
                q = 0;
                jm = j;
            } else {
                q = lean_quot(P, s, j);
                jm = j - q * Ns;
            }
            if (R > 1 && !FIRST && Ns > 1) {
                const C* tw = static_cast<const C*>(P.tw) + P.tw_off[s] + jm * (R - 1);
#pragma unroll
                for (int r = 1; r < R; ++r) u[r] = cmul(u[r], __ldg(tw + (r - 1)));
            }
            dft<R, T>(u);
            const int base = q * Ns * R + jm;
            if constexpr (to_global) {
                if (X.line_ok) {
                    C* g = X.gout + (MODEC ? j * P.out_ks : j);
                    [[maybe_unused]] C w;
                    if constexpr (FEAT == kLeanTw4) {
                        w = lean_tw4<C>(P, j * X.c);
                        w.y *= tw4_sy;
                    }
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        C a = u[r];
                        if constexpr (FEAT == kLeanTw4) {
                            if (r > 0) w = cmul(w, tw4_step);
                            a = cmul(a, w);
                        }
                        a.x *= out_sx;
                        a.y *= out_sy;
                        g[r * out_step] = a;
                    }
                }
            } else if constexpr (lin_out) {
                C* p = X.sm + lean_sidx<T, MODEC>(P, base);
#pragma unroll
                for (int r = 0; r < R; ++r) p[r * out_step] = u[r];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) X.sm[lean_sidx<T, MODEC>(P, base + r * Ns)] = u[r];
            }
        }
    }
    if constexpr (!to_global) __syncthreads();
}

// The first and the last stage touch HBM and are compiled apart from the inner stages, which
// run grouped by radix (16, 8, 4, 2, 15, 3, 5, 7, the order the planner gives them), so no stage
// carries the register cost of both kinds of access. At least two stages.
template <class T, int MAXV, bool MODEC, int FEAT, bool FIRST, bool LAST>
__device__ __forceinline__ void lean_edge(const LeanParams& P, int s, LeanCtx<T>& X) {
    switch (P.radix[s]) {
        case 16:
            if constexpr (MAXV >= 16) lean_stage<16, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X);
            break;
        case 15:
            if constexpr (MAXV >= 16) lean_stage<15, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X);
            break;
        case 8: lean_stage<8, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X); break;
        case 4: lean_stage<4, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X); break;
        case 2: lean_stage<2, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X); break;
        case 3: lean_stage<3, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X); break;
        case 5: lean_stage<5, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X); break;
        default: lean_stage<7, T, MAXV, MODEC, FEAT, FIRST, LAST>(P, s, X); break;
    }
}

template <int R, class T, int MAXV, bool MODEC, int FEAT>
__device__ __forceinline__ void lean_group(const LeanParams& P, LeanCtx<T>& X, int& s) {
    while (s < P.nstages - 1 && P.radix[s] == R) {
        lean_stage<R, T, MAXV, MODEC, FEAT, false, false>(P, s, X);
        ++s;
    }
}

template <class T, int MAXV>
constexpr int lean_regs() {
    return (sizeof(T) * MAXV > 64) ? 128 : 64;
}

// grid = n_outer * col_tiles tiles; block >= w * tpl; dynamic smem: kModeK w * pitch, kModeC
// w * n complex values.
template <class T, int MAXV, int MAXT, bool MODEC, int FEAT>
__global__ void __launch_bounds__(MAXT, 65536 / (MAXT * lean_regs<T, MAXV>()))
    fft_lean_kernel(const __grid_constant__ LeanParams P, const cplx<T>* in, cplx<T>* out) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    LeanCtx<T> X;
    const int tid = threadIdx.x;
    if constexpr (MODEC) {
        X.w = tid & (P.w - 1);
        X.t = tid >> P.w_shift;
        X.active = X.t < P.tpl;
    } else {
        X.w = tid / P.tpl;
        X.t = tid - X.w * P.tpl;
        X.active = X.w < P.w;
    }
    const int64_t tile = blockIdx.x;
    const int64_t o = tile / P.col_tiles;
    const int64_t c0 = (tile - o * P.col_tiles) << P.w_shift;
    const int64_t c = c0 + X.w;
    X.c = static_cast<int>(c);
    X.line_ok = X.active && c < P.n_cols;
    X.gin = in + o * P.in_hi + c * P.in_cs;
    X.gout = out + o * P.out_hi + c * P.out_cs;
    X.sm = MODEC ? sm + X.w : sm + X.w * P.pitch;
    lean_edge<T, MAXV, MODEC, FEAT, true, false>(P, 0, X);
    int s = 1;
    if constexpr (MAXV >= 16) lean_group<16, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_group<8, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_group<4, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_group<2, T, MAXV, MODEC, FEAT>(P, X, s);
    if constexpr (MAXV >= 16) lean_group<15, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_group<3, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_group<5, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_group<7, T, MAXV, MODEC, FEAT>(P, X, s);
    lean_edge<T, MAXV, MODEC, FEAT, false, true>(P, P.nstages - 1, X);
}

}  // namespace sfb
