// Register-resident forward DFT butterflies of radix 1, 2, 3, 4, 5, 7, 8, 16.
//
// All butterflies compute X_p = sum_q v_q * exp(-2*pi*i*p*q/R) in place on an array
// of R complex values held in registers. Inverse transforms are obtained by the
// caller through conjugation (IDFT(x) = conj(DFT(conj(x)))), so only the forward
// sign is compiled. Radix 3/5/7 use the symmetric (cos on sums, sin on
// differences) form; radix 8 and 16 are split-radix products of radix 2 and 4.
//
// The functions are __host__ __device__ so the host test library can check them
// against a direct DFT without a GPU.
#pragma once

#if defined(__CUDACC__)
#define SFB_HD __host__ __device__ __forceinline__
#else
#define SFB_HD inline
#endif

#include <cstdint>
#if defined(__CUDACC__)
#include <cuda_runtime.h>
#else
struct float2 { float x, y; };
struct double2 { double x, y; };
#endif

namespace sfb {

template <class T> struct cvec;
template <> struct cvec<float> { using type = float2; };
template <> struct cvec<double> { using type = double2; };
template <class T> using cplx = typename cvec<T>::type;

template <class C> SFB_HD C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class C> SFB_HD C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <class C> SFB_HD C cmul(C a, C b) {
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <class C, class T> SFB_HD C cscale(C a, T s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
template <class C> SFB_HD C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
// multiply by -i
template <class C> SFB_HD C cmul_mi(C a) { C r; r.x = a.y; r.y = -a.x; return r; }
template <class C> SFB_HD C cmake(decltype(C::x) x, decltype(C::x) y) { C r; r.x = x; r.y = y; return r; }

// Exact decimal expansions of cos/sin at rational multiples of pi.
#define SFB_K3S 0.866025403784438646764
#define SFB_K5C1 0.309016994374947424102
#define SFB_K5C2 -0.809016994374947424102
#define SFB_K5S1 0.951056516295153572116
#define SFB_K5S2 0.587785252292473129169
#define SFB_K7C1 0.623489801858733530525
#define SFB_K7C2 -0.222520933956314404289
#define SFB_K7C3 -0.900968867902419126236
#define SFB_K7S1 0.781831482468029808708
#define SFB_K7S2 0.974927912181823607018
#define SFB_K7S3 0.433883739117558120476
#define SFB_K8 0.707106781186547524401
#define SFB_K16C 0.923879532511286756128
#define SFB_K16S 0.382683432365089771728

template <class C> SFB_HD void bfly2(C& a, C& b) {
    const C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <class C> SFB_HD void bfly4(C& v0, C& v1, C& v2, C& v3) {
    const C t0 = cadd(v0, v2), t1 = csub(v0, v2);
    const C t2 = cadd(v1, v3), t3 = cmul_mi(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

template <class T, class C> SFB_HD void bfly3(C* v) {
    const T k3s = T(SFB_K3S);
    const C s = cadd(v[1], v[2]);
    const C d = csub(v[1], v[2]);
    const C m = cmake<C>(v[0].x - T(0.5) * s.x, v[0].y - T(0.5) * s.y);
    v[0] = cadd(v[0], s);
    // X1 = m - i*k3s*d, X2 = m + i*k3s*d
    v[1] = cmake<C>(m.x + k3s * d.y, m.y - k3s * d.x);
    v[2] = cmake<C>(m.x - k3s * d.y, m.y + k3s * d.x);
}

template <class T, class C> SFB_HD void bfly5(C* v) {
    const T c1 = T(SFB_K5C1), c2 = T(SFB_K5C2), s1 = T(SFB_K5S1), s2 = T(SFB_K5S2);
    const C a1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
    const C a2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
    const C x0 = v[0];
    const C A1 = cmake<C>(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    const C A2 = cmake<C>(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    const C B1 = cmake<C>(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
    const C B2 = cmake<C>(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
    v[0] = cmake<C>(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    v[1] = cmake<C>(A1.x + B1.y, A1.y - B1.x);
    v[4] = cmake<C>(A1.x - B1.y, A1.y + B1.x);
    v[2] = cmake<C>(A2.x + B2.y, A2.y - B2.x);
    v[3] = cmake<C>(A2.x - B2.y, A2.y + B2.x);
}

template <class T, class C> SFB_HD void bfly7(C* v) {
    const T c1 = T(SFB_K7C1), c2 = T(SFB_K7C2), c3 = T(SFB_K7C3);
    const T s1 = T(SFB_K7S1), s2 = T(SFB_K7S2), s3 = T(SFB_K7S3);
    const C a1 = cadd(v[1], v[6]), d1 = csub(v[1], v[6]);
    const C a2 = cadd(v[2], v[5]), d2 = csub(v[2], v[5]);
    const C a3 = cadd(v[3], v[4]), d3 = csub(v[3], v[4]);
    const C x0 = v[0];
    // p*q mod 7 table: p=1 -> (1,2,3); p=2 -> (2,4,6); p=3 -> (3,6,2)
    const C A1 = cmake<C>(x0.x + c1 * a1.x + c2 * a2.x + c3 * a3.x,
                          x0.y + c1 * a1.y + c2 * a2.y + c3 * a3.y);
    const C A2 = cmake<C>(x0.x + c2 * a1.x + c3 * a2.x + c1 * a3.x,
                          x0.y + c2 * a1.y + c3 * a2.y + c1 * a3.y);
    const C A3 = cmake<C>(x0.x + c3 * a1.x + c1 * a2.x + c2 * a3.x,
                          x0.y + c3 * a1.y + c1 * a2.y + c2 * a3.y);
    const C B1 = cmake<C>(s1 * d1.x + s2 * d2.x + s3 * d3.x, s1 * d1.y + s2 * d2.y + s3 * d3.y);
    const C B2 = cmake<C>(s2 * d1.x - s3 * d2.x - s1 * d3.x, s2 * d1.y - s3 * d2.y - s1 * d3.y);
    const C B3 = cmake<C>(s3 * d1.x - s1 * d2.x + s2 * d3.x, s3 * d1.y - s1 * d2.y + s2 * d3.y);
    v[0] = cmake<C>(x0.x + a1.x + a2.x + a3.x, x0.y + a1.y + a2.y + a3.y);
    v[1] = cmake<C>(A1.x + B1.y, A1.y - B1.x);
    v[6] = cmake<C>(A1.x - B1.y, A1.y + B1.x);
    v[2] = cmake<C>(A2.x + B2.y, A2.y - B2.x);
    v[5] = cmake<C>(A2.x - B2.y, A2.y + B2.x);
    v[3] = cmake<C>(A3.x + B3.y, A3.y - B3.x);
    v[4] = cmake<C>(A3.x - B3.y, A3.y + B3.x);
}

template <class T, class C> SFB_HD void bfly8(C* v) {
    const T k = T(SFB_K8);
    // DIT: DFT4 of evens and odds, then combine with W8^k.
    bfly4(v[0], v[2], v[4], v[6]);
    bfly4(v[1], v[3], v[5], v[7]);
    // odds: O1 *= W8 = (k, -k), O2 *= -i, O3 *= W8^3 = (-k, -k)
    const C o1 = cmake<C>(k * (v[3].x + v[3].y), k * (v[3].y - v[3].x));
    const C o2 = cmul_mi(v[5]);
    const C o3 = cmake<C>(k * (v[7].y - v[7].x), -k * (v[7].x + v[7].y));
    const C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    const C o0 = v[1];
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
}

template <class T, class C> SFB_HD void bfly16(C* v) {
    const T c = T(SFB_K16C), s = T(SFB_K16S), k = T(SFB_K8);
    // n = n2 + 4*n1: DFT4 over n1 for each n2 (in place: v[n2 + 4*k1] = Y[n2][k1])
    bfly4(v[0], v[4], v[8], v[12]);
    bfly4(v[1], v[5], v[9], v[13]);
    bfly4(v[2], v[6], v[10], v[14]);
    bfly4(v[3], v[7], v[11], v[15]);
    // twiddles W16^(n2*k1): W1=(c,-s) W2=(k,-k) W3=(s,-c) W4=-i W6=(-k,-k) W9=(-c,s)
    v[5] = cmul(v[5], cmake<C>(c, -s));
    v[9] = cmul(v[9], cmake<C>(k, -k));
    v[13] = cmul(v[13], cmake<C>(s, -c));
    v[6] = cmul(v[6], cmake<C>(k, -k));
    v[10] = cmul_mi(v[10]);
    v[14] = cmul(v[14], cmake<C>(-k, -k));
    v[7] = cmul(v[7], cmake<C>(s, -c));
    v[11] = cmul(v[11], cmake<C>(-k, -k));
    v[15] = cmul(v[15], cmake<C>(-c, s));
    // DFT4 over n2 for each k1: X[k1 + 4*k2] from Y[.][k1] at v[4*k1 + n2]
    bfly4(v[0], v[1], v[2], v[3]);
    bfly4(v[4], v[5], v[6], v[7]);
    bfly4(v[8], v[9], v[10], v[11]);
    bfly4(v[12], v[13], v[14], v[15]);
    // now v[4*k1 + k2] = X[k1 + 4*k2]: transpose 4x4 in registers
    C t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
}

// Radix 15 as a prime-factor (Good-Thomas) DFT, 15 = 3 * 5 with coprime factors: no
// internal twiddles. Input n = (5*n1 + 3*n2) mod 15 feeds five-point DFTs over n2, then
// three-point DFTs over n1; output (k1, k2) is X[(10*k1 + 6*k2) mod 15], since
// W15^(n k) = W3^(n1 k1) * W5^(n2 k2) for those index maps.
template <class T, class C> SFB_HD void bfly15(C* v) {
    C a[3][5];
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) {
#pragma unroll
        for (int n2 = 0; n2 < 5; ++n2) a[n1][n2] = v[(5 * n1 + 3 * n2) % 15];
        bfly5<T>(a[n1]);
    }
#pragma unroll
    for (int k2 = 0; k2 < 5; ++k2) {
        C b[3] = {a[0][k2], a[1][k2], a[2][k2]};
        bfly3<T>(b);
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) v[(10 * k1 + 6 * k2) % 15] = b[k1];
    }
}

// u[r] *= w^r for r = 1..R-1, the powers formed by a balanced product tree
// (w^r = w^h * w^(r-h), h the largest power of two <= r): at most log2(R)+1 roundings deep.
template <int R, class C> SFB_HD void twiddle_powers(C* u, C w) {
    C p[R > 1 ? R : 1];
    p[0] = w;  // p[k] holds w^(k+1)
#pragma unroll
    for (int r = 2; r < R; ++r) {
        int h = 1;
        while (h * 2 <= r) h *= 2;
        p[r - 1] = (h == r) ? cmul(p[h / 2 - 1], p[h / 2 - 1]) : cmul(p[h - 1], p[r - h - 1]);
    }
#pragma unroll
    for (int r = 1; r < R; ++r) u[r] = cmul(u[r], p[r - 1]);
}

// Radix 15 twiddles u[r] *= w^r with few live registers: the powers of the balanced tree
// (w^r = w^h * w^(r-h), at most 4 roundings deep) are formed right before their use, so only
// w, w^2, w^4, w^8 and w^12 stay live instead of all fourteen.
template <class C> SFB_HD void twiddle_powers15(C* u, C w) {
    const C w2 = cmul(w, w);
    const C w4 = cmul(w2, w2);
    const C w8 = cmul(w4, w4);
    u[1] = cmul(u[1], w);
    u[2] = cmul(u[2], w2);
    u[3] = cmul(u[3], cmul(w2, w));
    u[4] = cmul(u[4], w4);
    u[5] = cmul(u[5], cmul(w4, w));
    const C w6 = cmul(w4, w2);
    u[6] = cmul(u[6], w6);
    u[7] = cmul(u[7], cmul(w6, w));
    u[8] = cmul(u[8], w8);
    u[9] = cmul(u[9], cmul(w8, w));
    const C w10 = cmul(w8, w2);
    u[10] = cmul(u[10], w10);
    u[11] = cmul(u[11], cmul(w10, w));
    const C w12 = cmul(w8, w4);
    u[12] = cmul(u[12], w12);
    u[13] = cmul(u[13], cmul(w12, w));
    u[14] = cmul(u[14], cmul(w12, w2));
}

template <int R, class T, class C> SFB_HD void dft(C* v) {
    if constexpr (R == 1) {
        (void)v;
    } else if constexpr (R == 2) {
        bfly2(v[0], v[1]);
    } else if constexpr (R == 3) {
        bfly3<T>(v);
    } else if constexpr (R == 4) {
        bfly4(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 5) {
        bfly5<T>(v);
    } else if constexpr (R == 7) {
        bfly7<T>(v);
    } else if constexpr (R == 8) {
        bfly8<T>(v);
    } else if constexpr (R == 15) {
        bfly15<T>(v);
    } else if constexpr (R == 16) {
        bfly16<T>(v);
    }
}

}  // namespace sfb
