// Size-specialised pass kernels: the same Stockham register/shared-memory scheme as
// pass_kernel.cuh, with the FFT length, radix sequence, threads per line and the
// shared-memory layout fixed at compile time. Every stage's strides, twiddle-table
// offsets and shared-memory offsets then fold into immediates, so a thread's work is
// loads, butterflies and stores with almost no index arithmetic.
//
// Plain passes use them (a whole line per CTA row, conjugation for inverse transforms and
// the normalization scale fused into the store), the four-step column and row passes
// (twiddle fused into the store, transposed store), the Bluestein passes (a zero-padded
// chirp pre-multiply on the first load, a spectrum multiply between two FFTs held in
// shared memory, and a chirp post-multiply with truncation on the last store) and the Rader
// passes of prime lengths (a permuted gather on the first load, the same spectrum multiply
// with the x[0] term, a permuted scatter on the last store).
//   kModeK: lines are contiguous (line pitch `in_pitch`), threads walk elements;
//   kModeC: lines are strided columns (element stride `in_ks`, columns contiguous),
//           threads walk W adjacent columns so every access is a W-wide segment.
#pragma once

#include <cuda_runtime.h>

#include "butterfly.cuh"

namespace sfb {

struct FixedParams {
    int64_t n_cols = 1;     // lines (kModeK) or columns per outer index (kModeC)
    int64_t col_tiles = 1;  // ceil(n_cols / w)
    int w = 1;              // lines per CTA (kModeK; kModeC uses the compile-time W)
    int64_t in_hi = 0, out_hi = 0;      // outer stride (kModeC)
    int64_t in_pitch = 0, out_pitch = 0;  // line pitch (kModeK)
    int64_t in_ks = 1, out_ks = 1;      // element stride (kModeC)
    const void* tw = nullptr;           // base twiddles: per stage, W_(ns*R)^jm for jm < ns, concatenated
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    // kFeatTw4 (kModeC column pass of a four-step): multiply output k of column c by
    // W_L^(k*c) = tw4_hi[m >> tw4_shift] * tw4_lo[m & mask], m = k * c.
    const void* tw4_hi = nullptr;
    const void* tw4_lo = nullptr;
    int tw4_shift = 0;
    // kFeatTStore (kModeK row pass of a four-step): row l = o*rows + k1 of length N is
    // stored transposed at o * line + k1 + k2 * rows (coalesced over consecutive rows).
    int64_t rows = 1, line = 0;
    // Bluestein features. Element index g = k * g_k + sel (sel: the column in kModeC, 0 in
    // kModeK); kFeatPremul loads x[g] * premul[g] for g < in_len and 0 beyond; kFeatConv
    // multiplies the first FFT's output k by pointwise[k + sel * pw_stride] (sel: the row
    // index modulo `rows` in kModeK), conjugates it when conj_mid, and runs the FFT again;
    // kFeatPostmul stores v * postmul[g] for g < out_len only. flip_in / flip_out conjugate
    // the raw input and the final value (a direction override of the whole plan).
    const void* premul = nullptr;
    const void* postmul = nullptr;
    const void* pointwise = nullptr;
    int g_k = 1;
    int in_len = 0, out_len = 0;
    int pw_stride = 0;
    int conj_mid = 0;
    int flip_in = 0, flip_out = 0;
    // Rader features (a prime length L whose convolution length M = L - 1 the catalog covers:
    // with g a primitive root mod L, X[g^-q] = x[0] + sum_p x[g^p] W^(g^(p-q)), a cyclic
    // convolution of length M). kFeatGather loads element g as x[perm_in[g]] from the start
    // of the line (g < in_len); kFeatScatter stores element g to y[perm_out[g]] (g < out_len);
    // kFeatRaderDC (the convolution pass): bin 0 of the first FFT is A0 = sum over the
    // gathered line, so X[0] = x[0] + A0 is stored at y[0], and x[0] is added to bin 0 of the
    // spectrum product, which adds it to every convolution output. dc_x / dc_y are the line
    // starts of x and y for the three-pass row kernel (line o = row / rows), dc_scale and
    // dc_flip_in / dc_flip_out the scale and direction flips of the outputs around it.
    const int* perm_in = nullptr;
    const int* perm_out = nullptr;
    const void* dc_x = nullptr;
    void* dc_y = nullptr;
    int64_t dc_x_pitch = 0, dc_y_pitch = 0;
    double dc_scale = 1.0;
    int dc_flip_in = 0, dc_flip_out = 0;
};

// Features (bits): kFeatTw4 four-step twiddle on the last store, kFeatTStore transposed
// row store, kFeatPremul / kFeatConv / kFeatPostmul the Bluestein hooks above,
// kFeatTw4Conj the conjugate twiddle (inverse four-step), kFeatMid (internal) the first
// FFT of a kFeatConv pass storing its spectrum product to shared memory.
enum : int {
    kFeatPlain = 0,
    kFeatTw4 = 1,
    kFeatTStore = 2,
    kFeatPremul = 4,
    kFeatMid = 8,
    kFeatPostmul = 16,
    kFeatTw4Conj = 32,
    kFeatConv = 64,
    kFeatSmemIn = 128,  // the first stage reads the tile from shared memory (TMA-staged passes)
    // Real transforms of length 2N over this length-N FFT (kModeK only; the W_2N^k table of
    // N+1 entries in `postmul` / `premul`):
    kFeatRealPost = 512,  // R2C: the spectrum Z goes to shared memory, then X[k] for k = 0..N from
                          // the pairs (Z[k], Z[N-k]), N+1 bins per line stored
    kFeatRealPre = 1024,  // C2R: the first stage forms Z[k] from the bins (X[k], X[N-k]) on load
    kFeatLoadCG = 2048,   // first-stage global loads bypass L1 (ld.global.cg): data another CTA of
                          // the same launch wrote (the fused four-step's L2-resident ring)
    kFeatLoadCS = 4096,   // first-stage global loads and last-stage global stores marked
    kFeatStoreCS = 8192,  // streaming (ld/st .cs, evicted first): data read or written once, so
                          // it does not push an L2-resident ring out of the cache
    kFeatGather = 16384,  // Rader: first-stage loads through perm_in
    kFeatScatter = 32768, // Rader: last-stage stores through perm_out
    kFeatRaderDC = 65536, // Rader: X[0] and the x[0] term at bin 0 of the convolution pass
};

// 4-byte global -> shared copy that completes asynchronously (cp.async), and its wait.
__device__ __forceinline__ void cp_async4(int* dst, const int* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit_only() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int FEAT, class C>
__device__ __forceinline__ C fixed_load(const C* p) {
    if constexpr (FEAT & kFeatLoadCG) return __ldcg(p);
    else if constexpr (FEAT & kFeatLoadCS) return __ldcs(p);
    else return *p;
}

// X[k] = 1/2 [(Z[k] + conj Z[N-k]) - i W_2N^k (Z[k] - conj Z[N-k])] * scale; a = Z[k], c = Z[N-k]
template <class C, class T>
__device__ __forceinline__ C real_post_pair(C a, C c, C w, T half) {
    const C e = cmake<C>(a.x + c.x, a.y - c.y);
    const C d = cmake<C>(a.x - c.x, a.y + c.y);
    const T p = w.x * d.x - w.y * d.y, q = w.x * d.y + w.y * d.x;  // w * D
    return cmake<C>((e.x + q) * half, (e.y - p) * half);
}

// Z[k] = (X[k] + conj X[N-k]) + i conj(W_2N^k) (X[k] - conj X[N-k]); a = X[k], c = X[N-k]
template <class C, class T = decltype(C::x)>
__device__ __forceinline__ C real_pre_pair(C a, C c, C w) {
    const C e = cmake<C>(a.x + c.x, a.y - c.y);
    const C d = cmake<C>(a.x - c.x, a.y + c.y);
    const T p = w.x * d.x + w.y * d.y, q = w.x * d.y - w.y * d.x;  // conj(w) * D
    return cmake<C>(e.x - q, e.y + p);
}

template <class T>
struct FixedCtx {
    using C = cplx<T>;
    C* sm;           // this thread's line (kModeK) or column (kModeC) in shared memory
    const C* gin;    // this thread's line / column in the input
    C* gout;
    const C* twb;    // twiddle table base
    int t;
    bool active;
    bool line_ok;
    int64_t in_ks, out_ks;
    T scale;
    bool conj_in, conj_out;
    int sel;              // column index (kFeatTw4, Bluestein element index)
    const C *tw4_hi, *tw4_lo;
    int tw4_shift;
    const C *premul, *postmul, *pw;  // pw: pointwise table of this line (kFeatConv)
    int g_k, in_len, out_len;
    bool conj_mid, flip_in, flip_out;
    const int *perm_in, *perm_out;  // Rader permutations
    const C* gline;                  // start of this thread's input line (kFeatGather)
    C* gline_out;                    // start of its output line (kFeatScatter)
    const int* sidx;                 // kModeC kFeatScatter: this column's perm_out entries in
                                     // shared memory (element k at sidx[k * W])
    const C* rx;                     // x line and y line of the bin-0 term (kFeatRaderDC)
    C* ry;
    T dc_scale;
    bool dc_flip_in, dc_flip_out;
};

template <class T> __host__ __device__ constexpr int pad_shift_c() { return sizeof(T) == 4 ? 4 : 3; }
template <class T, int N> __host__ __device__ constexpr int kpitch() {
    constexpr int p = N + (N >> pad_shift_c<T>());
    return (p & 1) ? p : p + 1;
}

template <class T>
__device__ __forceinline__ int pidx(int k) {
    return k + (k >> pad_shift_c<T>());
}

template <class T, int N, int TPL, bool MODEC, int W, int FEAT, int NS, int TWOFF, int R, bool FIRST, bool LAST>
__device__ __forceinline__ void fixed_stage(FixedCtx<T>& X) {
    using C = cplx<T>;
    constexpr int PS = pad_shift_c<T>();
    constexpr int PAD = 1 << PS;
    constexpr int NR = N / R;
    constexpr int NB = (NR + TPL - 1) / TPL;
    constexpr bool EXACT = (NR % TPL) == 0;
    C v[NB * R];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = X.t + i * TPL;
        if (X.active && (EXACT || j < NR)) {
            if constexpr (FIRST && (FEAT & kFeatSmemIn)) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    C a = MODEC ? X.sm[(j + r * NR) * W] : X.sm[pidx<T>(j + r * NR)];
                    if (X.conj_in) a.y = -a.y;
                    v[i * R + r] = a;
                }
            } else if constexpr (FIRST && (FEAT & kFeatPremul)) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int k = j + r * NR;
                    const int g = k * X.g_k + X.sel;
                    C a = cmake<C>(T(0), T(0));
                    if (X.line_ok && g < X.in_len) {
                        a = fixed_load<FEAT>(MODEC ? X.gin + (int64_t)k * X.in_ks : X.gin + k);
                        if (X.flip_in) a.y = -a.y;
                        a = cmul(a, __ldg(X.premul + g));
                        if (X.conj_in) a.y = -a.y;
                    }
                    v[i * R + r] = a;
                }
            } else if constexpr (FIRST && (FEAT & kFeatGather)) {
                // all of this butterfly's indices first, then all its gathers: the two
                // dependent loads cost one round trip each instead of one per element
                int src[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int g = (j + r * NR) * X.g_k + X.sel;
                    src[r] = X.line_ok && g < X.in_len ? __ldg(X.perm_in + g) : -1;
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    C a = cmake<C>(T(0), T(0));
                    if (src[r] >= 0) {
                        a = X.gline[src[r]];
                        if (X.flip_in) a.y = -a.y;
                        if (X.conj_in) a.y = -a.y;
                    }
                    v[i * R + r] = a;
                }
            } else if constexpr (FIRST && (FEAT & kFeatRealPre)) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int k = j + r * NR;
                    C a = cmake<C>(T(0), T(0));
                    if (X.line_ok) {
                        C xa = X.gin[k];
                        C xc = X.gin[N - k];  // the line holds N+1 bins
                        if (k == 0) {
                            xa.y = T(0);  // bins 0 and N of a real signal are real
                            xc.y = T(0);
                        }
                        a = real_pre_pair(xa, xc, __ldg(X.premul + k));
                        if (X.conj_in) a.y = -a.y;
                    }
                    v[i * R + r] = a;
                }
            } else if constexpr (FIRST) {
                if (X.line_ok) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const C* src = MODEC ? X.gin + (int64_t)(j + r * NR) * X.in_ks : X.gin + (j + r * NR);
                        C a = fixed_load<FEAT>(src);
                        if (X.conj_in) a.y = -a.y;
                        v[i * R + r] = a;
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) v[i * R + r] = cmake<C>(T(0), T(0));
                }
            } else if constexpr (MODEC) {
#pragma unroll
                for (int r = 0; r < R; ++r) v[i * R + r] = X.sm[(j + r * NR) * W];
            } else if constexpr (NR % PAD == 0) {
                const C* p = X.sm + pidx<T>(j);
#pragma unroll
                for (int r = 0; r < R; ++r) v[i * R + r] = p[r * (NR + NR / PAD)];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) v[i * R + r] = X.sm[pidx<T>(j + r * NR)];
            }
        }
    }
    if constexpr (LAST && MODEC && (FEAT & kFeatScatter)) {
        // the scatter indices this thread's copies brought to shared memory (kernel start)
        cp_async_commit_wait_all();
        if constexpr (FIRST) __syncthreads();
    }
    if constexpr (!FIRST || (FEAT & kFeatSmemIn)) __syncthreads();
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = X.t + i * TPL;
        if (X.active && (EXACT || j < NR)) {
            C* u = &v[i * R];
            const int jm = j % NS;
            if constexpr (NS > 1 && R > 1) {
                // base-twiddle table: one W_(NS*R)^jm per butterfly, powers in registers
                if constexpr (R == 15) twiddle_powers15(u, __ldg(X.twb + TWOFF + jm));
                else twiddle_powers<R>(u, __ldg(X.twb + TWOFF + jm));
            }
            dft<R, T>(u);
            if constexpr (LAST && (FEAT & (kFeatTStore | kFeatMid | kFeatRealPost))) {
                // natural order into shared memory: the transposed store, or the second FFT
                // of a Bluestein convolution (after the spectrum multiply), follows
                if constexpr (FEAT & kFeatMid) {
                    C dc = cmake<C>(T(0), T(0));
                    if constexpr (FEAT & kFeatRaderDC) {
                        // bin 0 of this line (row 0, element 0): X[0] = x[0] + A0
                        if (X.sel == 0 && j == 0 && X.line_ok) {
                            dc = X.rx[0];
                            if (X.dc_flip_in) dc.y = -dc.y;
                            C y0 = cmake<C>(dc.x + u[0].x, dc.y + u[0].y);
                            if (X.dc_flip_out) y0.y = -y0.y;
                            y0.x *= X.dc_scale;
                            y0.y *= X.dc_scale;
                            X.ry[0] = y0;
                        }
                    }
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        u[r] = cmul(u[r], __ldg(X.pw + j + r * NR));
                        if constexpr (FEAT & kFeatRaderDC) {
                            if (r == 0) {
                                u[0].x += dc.x;
                                u[0].y += dc.y;
                            }
                        }
                        if (X.conj_mid) u[r].y = -u[r].y;
                    }
                }
                if constexpr (NR % PAD == 0) {
                    C* p = X.sm + pidx<T>(j);
#pragma unroll
                    for (int r = 0; r < R; ++r) p[r * (NR + NR / PAD)] = u[r];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) X.sm[pidx<T>(j + r * NR)] = u[r];
                }
            } else if constexpr (LAST) {
                // last stage: base == j, outputs at j + r * NR
                if (X.line_ok) {
                    // complex<double>: the four-step twiddles of this butterfly's outputs form a
                    // geometric sequence, W^((j + r*NR)*sel) = W^(j*sel) * (W^(NR*sel))^r, so the
                    // two-level table is read twice per butterfly instead of per output (R - 1
                    // products deep; float keeps the per-output lookup, its last radix being 16)
                    constexpr bool kGeo = (FEAT & kFeatTw4) && sizeof(T) == 8;
                    [[maybe_unused]] C w4, w4_step;
                    if constexpr (kGeo) {
                        const int m0 = j * X.sel, ms = NR * X.sel, mask = (1 << X.tw4_shift) - 1;
                        w4 = cmul(__ldg(X.tw4_hi + (m0 >> X.tw4_shift)), __ldg(X.tw4_lo + (m0 & mask)));
                        w4_step = cmul(__ldg(X.tw4_hi + (ms >> X.tw4_shift)), __ldg(X.tw4_lo + (ms & mask)));
                        if constexpr (FEAT & kFeatTw4Conj) {
                            w4.y = -w4.y;
                            w4_step.y = -w4_step.y;
                        }
                    }
                    // with nothing between the output conjugation and the scale, the conjugation
                    // is the sign of the imaginary part's scale (no select per output)
                    constexpr bool kFold = !(FEAT & (kFeatTw4 | kFeatPostmul));
                    [[maybe_unused]] const T sy_out = X.conj_out ? -X.scale : X.scale;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int k = j + r * NR;
                        C a = u[r];
                        if constexpr (!kFold) {
                            if (X.conj_out) a.y = -a.y;
                        }
                        if constexpr (kGeo) {
                            if (r > 0) w4 = cmul(w4, w4_step);
                            a = cmul(a, w4);
                        } else if constexpr (FEAT & kFeatTw4) {
                            const int m = k * X.sel;
                            C w = cmul(__ldg(X.tw4_hi + (m >> X.tw4_shift)),
                                       __ldg(X.tw4_lo + (m & ((1 << X.tw4_shift) - 1))));
                            if constexpr (FEAT & kFeatTw4Conj) w.y = -w.y;
                            a = cmul(a, w);
                        }
                        if constexpr (FEAT & kFeatPostmul) {
                            const int g = k * X.g_k + X.sel;
                            if (g >= X.out_len) continue;
                            a = cmul(a, __ldg(X.postmul + g));
                        }
                        [[maybe_unused]] int g = 0;
                        if constexpr (FEAT & kFeatScatter) {
                            g = k * X.g_k + X.sel;
                            if (g >= X.out_len) continue;
                        }
                        a.x *= X.scale;
                        a.y *= kFold ? sy_out : X.scale;
                        if constexpr (FEAT & (kFeatPostmul | kFeatScatter)) {
                            if (X.flip_out) a.y = -a.y;
                        }
                        C* dst;
                        if constexpr ((FEAT & kFeatScatter) && MODEC) dst = X.gline_out + X.sidx[k * W];
                        else if constexpr (FEAT & kFeatScatter) dst = X.gline_out + __ldg(X.perm_out + g);
                        else dst = MODEC ? X.gout + (int64_t)k * X.out_ks : X.gout + k;
                        if constexpr (FEAT & kFeatStoreCS) __stcs(dst, a);
                        else *dst = a;
                    }
                }
            } else {
                const int base = (j - jm) * R + jm;
                if constexpr (MODEC) {
#pragma unroll
                    for (int r = 0; r < R; ++r) X.sm[(base + r * NS) * W] = u[r];
                } else if constexpr (NS % PAD == 0 || (R * NS <= PAD && PAD % (R * NS) == 0)) {
                    C* p = X.sm + pidx<T>(base);
#pragma unroll
                    for (int r = 0; r < R; ++r) p[r * NS + (r * NS) / PAD] = u[r];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) X.sm[pidx<T>(base + r * NS)] = u[r];
                }
            }
        }
    }
    if constexpr (!LAST || (FEAT & (kFeatTStore | kFeatMid | kFeatRealPost))) __syncthreads();
}

template <class T, int N, int TPL, bool MODEC, int W, int FEAT, int NS, int TWOFF, bool FIRST, int R, int... Rest>
__device__ __forceinline__ void fixed_stages(FixedCtx<T>& X) {
    constexpr bool LAST = sizeof...(Rest) == 0;
    fixed_stage<T, N, TPL, MODEC, W, FEAT, NS, TWOFF, R, FIRST, LAST>(X);
    if constexpr (!LAST)
        fixed_stages<T, N, TPL, MODEC, W, FEAT, NS * R, TWOFF + NS, false, Rest...>(X);
}

// Register budget: 64 per thread (16 float or 8 double complex values per stage).
template <class T, int MAXT, int REGS>
__host__ __device__ constexpr int fixed_min_blocks() {
    return 65536 / (MAXT * REGS) > 0 ? 65536 / (MAXT * REGS) : 1;
}

// kModeK: grid = ceil(lines / w), block = w * TPL (<= MAXT), dynamic smem = w * kpitch<T,N>() * sizeof(C).
// kModeC: grid = n_outer * col_tiles, block = W * TPL, dynamic smem = N * W * sizeof(C).
template <class T, int N, int TPL, bool MODEC, int W, int FEAT, int MAXT, int REGS, int... Rs>
__global__ void __launch_bounds__(MAXT, fixed_min_blocks<T, MAXT, REGS>())
    fft_fixed_kernel(const __grid_constant__ FixedParams P, const cplx<T>* in, cplx<T>* out) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    FixedCtx<T> X;
    X.twb = static_cast<const C*>(P.tw);
    X.scale = static_cast<T>(P.scale);
    X.conj_in = P.conj_in != 0;
    X.conj_out = P.conj_out != 0;
    X.premul = static_cast<const C*>(P.premul);
    X.postmul = static_cast<const C*>(P.postmul);
    X.g_k = P.g_k;
    X.in_len = P.in_len;
    X.out_len = P.out_len;
    X.conj_mid = P.conj_mid != 0;
    X.flip_in = P.flip_in != 0;
    X.flip_out = P.flip_out != 0;
    X.perm_in = P.perm_in;
    X.perm_out = P.perm_out;
    const int tid = threadIdx.x;
    if constexpr (MODEC) {
        const int w = tid % W;
        X.t = tid / W;
        X.active = X.t < TPL;
        const int64_t tile = blockIdx.x;
        const int64_t o = tile / P.col_tiles;
        const int64_t c = (tile - o * P.col_tiles) * W + w;
        X.line_ok = X.active && c < P.n_cols;
        X.sel = static_cast<int>(c);
        X.tw4_hi = static_cast<const C*>(P.tw4_hi);
        X.tw4_lo = static_cast<const C*>(P.tw4_lo);
        X.tw4_shift = P.tw4_shift;
        X.sm = sm + w;
        X.gin = in + o * P.in_hi + c;
        X.gout = out + o * P.out_hi + c;
        X.gline = in + o * P.in_hi;
        X.gline_out = out + o * P.out_hi;
        X.in_ks = P.in_ks;
        X.out_ks = P.out_ks;
        if constexpr (FEAT & kFeatScatter) {
            // the tile's scatter indices perm_out[k * g_k + c] (the planner adds N * W ints of
            // shared memory after the tile) fetched asynchronously while the stages run
            int* sidx = reinterpret_cast<int*>(sm + N * W);
            const int64_t c0 = (tile - o * P.col_tiles) * W;
            for (int e = tid; e < N * W; e += blockDim.x) {
                const int k = e / W;
                const int64_t cc = c0 + (e - k * W);
                if (cc < P.n_cols) cp_async4(sidx + e, P.perm_out + (int64_t)k * P.g_k + cc);
            }
            cp_async_commit_only();
            X.sidx = sidx + w;
        }
    } else {
        const int w = tid / TPL;
        X.t = tid - w * TPL;
        X.active = w < P.w;
        const int64_t c = (int64_t)blockIdx.x * P.w + w;
        X.line_ok = X.active && c < P.n_cols;
        X.sm = sm + w * kpitch<T, N>();
        X.gin = in + c * P.in_pitch;
        X.gout = out + c * P.out_pitch;
        X.in_ks = 1;
        X.out_ks = 1;
        // row index within its line (four-step row passes: the k1 of the twiddle and of
        // the spectrum table); 0 for whole lines
        X.sel = (FEAT & (kFeatTw4 | kFeatConv)) && P.rows > 1 ? static_cast<int>(c % P.rows) : 0;
        X.tw4_hi = static_cast<const C*>(P.tw4_hi);
        X.tw4_lo = static_cast<const C*>(P.tw4_lo);
        X.tw4_shift = P.tw4_shift;
        X.gline = X.gin;
        X.gline_out = X.gout;
        if constexpr (FEAT & kFeatRaderDC) {
            if constexpr (FEAT & kFeatGather) {
                // whole line in this CTA row (fused single pass): its own line, scale and flips
                X.rx = X.gin;
                X.ry = X.gout;
                X.dc_scale = X.scale;
                X.dc_flip_in = X.flip_in;
                X.dc_flip_out = X.flip_out;
            } else {
                // three-pass row kernel: row c is row c % rows of line c / rows
                const int64_t o = c / P.rows;
                X.rx = static_cast<const C*>(P.dc_x) + o * P.dc_x_pitch;
                X.ry = static_cast<C*>(P.dc_y) + o * P.dc_y_pitch;
                X.dc_scale = static_cast<T>(P.dc_scale);
                X.dc_flip_in = P.dc_flip_in != 0;
                X.dc_flip_out = P.dc_flip_out != 0;
            }
        }
    }
    if constexpr (FEAT & kFeatConv) {
        // Bluestein convolution: FFT, spectrum multiply (to shared memory), FFT again
        X.pw = static_cast<const C*>(P.pointwise) + (int64_t)X.sel * P.pw_stride;
        constexpr int kFirstOnly = kFeatPremul | kFeatGather | kFeatRaderDC;
        fixed_stages<T, N, TPL, MODEC, W, (FEAT & kFirstOnly) | kFeatMid, 1, 0, true, Rs...>(X);
        fixed_stages<T, N, TPL, MODEC, W, FEAT & ~(kFirstOnly | kFeatConv), 1, 0, false, Rs...>(X);
        return;
    }
    fixed_stages<T, N, TPL, MODEC, W, FEAT, 1, 0, true, Rs...>(X);
    if constexpr (FEAT & kFeatRealPost) {
        static_assert(!MODEC, "real transforms use contiguous lines");
        // pairs (k, N-k) of this line's spectrum in shared memory -> N+1 bins at X.gout
        if (X.line_ok) {
            const T half = T(0.5) * X.scale;
            for (int k = X.t; k <= N / 2; k += TPL) {
                const int kk = N - k;
                const C a = X.sm[pidx<T>(k)];
                const C c = X.sm[pidx<T>(kk == N ? 0 : kk)];
                X.gout[k] = real_post_pair(a, c, __ldg(X.postmul + k), half);
                if (kk != k) X.gout[kk] = real_post_pair(c, a, __ldg(X.postmul + kk), half);
            }
        }
    }
    if constexpr ((FEAT & kFeatTStore) && !MODEC) {
        // Rows blockIdx.x*W .. +W-1 are consecutive k1 of one line (the planner keeps
        // rows % W == 0): walk (row fastest, element) so every store is a W-wide segment.
        const int64_t row0 = (int64_t)blockIdx.x * W;
        const int64_t o = row0 / P.rows;
        C* dst = out + o * P.line + (row0 - o * P.rows);
        const int valid = static_cast<int>(P.n_cols - row0 < W ? P.n_cols - row0 : W);
        const T sc = X.scale;
        const T sy = X.conj_out ? -sc : sc;
#pragma unroll 4
        for (int idx = tid; idx < W * N; idx += blockDim.x) {
            const int k = idx / W;
            const int w = idx - k * W;
            if (w >= valid) continue;
            const C a = sm[w * kpitch<T, N>() + pidx<T>(k)];
            dst[w + (int64_t)k * P.rows] = cmake<C>(a.x * sc, a.y * sy);
        }
    }
}

}  // namespace sfb
