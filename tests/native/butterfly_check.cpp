// Host-side check of the register butterflies in sycl-fft_b200/csrc/butterfly.cuh.
// Test infrastructure: compiled with g++ (no GPU) and called from tests/ via ctypes.
#include "../../sycl-fft_b200/csrc/butterfly.cuh"

template <int R, class T>
static void run(const T* in, T* out) {
    using C = sfb::cplx<T>;
    C v[R > 0 ? R : 1];
    for (int i = 0; i < R; ++i) { v[i].x = in[2 * i]; v[i].y = in[2 * i + 1]; }
    sfb::dft<R, T>(v);
    for (int i = 0; i < R; ++i) { out[2 * i] = v[i].x; out[2 * i + 1] = v[i].y; }
}

template <class T>
static int dispatch(int radix, const T* in, T* out) {
    switch (radix) {
        case 1: run<1, T>(in, out); return 0;
        case 2: run<2, T>(in, out); return 0;
        case 3: run<3, T>(in, out); return 0;
        case 4: run<4, T>(in, out); return 0;
        case 5: run<5, T>(in, out); return 0;
        case 7: run<7, T>(in, out); return 0;
        case 8: run<8, T>(in, out); return 0;
        case 15: run<15, T>(in, out); return 0;
        case 16: run<16, T>(in, out); return 0;
        default: return 1;
    }
}

extern "C" int sfb_check_dft_f64(int radix, const double* in, double* out) { return dispatch<double>(radix, in, out); }
extern "C" int sfb_check_dft_f32(int radix, const float* in, float* out) { return dispatch<float>(radix, in, out); }

// u[r] *= w^r, r = 1..radix-1, through the size-specialised kernels' twiddle_powers
// (balanced product tree; mode 0, the only mode).
template <int R, class T>
static void powers(int mode, T wr, T wi, const T* in, T* out) {
    using C = sfb::cplx<T>;
    C v[R];
    for (int i = 0; i < R; ++i) { v[i].x = in[2 * i]; v[i].y = in[2 * i + 1]; }
    C w;
    w.x = wr;
    w.y = wi;
    if (mode != 0) return;
    sfb::twiddle_powers<R>(v, w);
    for (int i = 0; i < R; ++i) { out[2 * i] = v[i].x; out[2 * i + 1] = v[i].y; }
}

template <class T>
static int powers_dispatch(int mode, int radix, T wr, T wi, const T* in, T* out) {
    switch (radix) {
        case 2: powers<2, T>(mode, wr, wi, in, out); return 0;
        case 3: powers<3, T>(mode, wr, wi, in, out); return 0;
        case 4: powers<4, T>(mode, wr, wi, in, out); return 0;
        case 5: powers<5, T>(mode, wr, wi, in, out); return 0;
        case 7: powers<7, T>(mode, wr, wi, in, out); return 0;
        case 8: powers<8, T>(mode, wr, wi, in, out); return 0;
        case 16: powers<16, T>(mode, wr, wi, in, out); return 0;
        default: return 1;
    }
}

extern "C" int sfb_check_powers_f64(int mode, int radix, double wr, double wi, const double* in, double* out) {
    return powers_dispatch<double>(mode, radix, wr, wi, in, out);
}
extern "C" int sfb_check_powers_f32(int mode, int radix, float wr, float wi, const float* in, float* out) {
    return powers_dispatch<float>(mode, radix, wr, wi, in, out);
}
