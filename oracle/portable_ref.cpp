// CPU restatement of the syclfft portable provider -- TEST INFRASTRUCTURE ONLY.
//
// This file is the oracle for the B200 provider's parity tests and the timed CPU
// baseline in bench.py. It is never linked into, loaded by, or called from the
// product library (sycl-fft_b200/). It restates, kernel for kernel, the
// portable SYCL provider of Vaskozlov/sycl-fft:
//
//   src/sycl/sycl.cpp:34-46    next_power_of_two           -> next_pow2()
//   src/sycl/sycl.cpp:48-61    supported_factors           -> smooth_factors()
//   src/sycl/sycl.cpp:63-70    axis_stride                 -> stride_after()
//   src/sycl/sycl.cpp:87-98    enqueue_copy_scaled   (K1)  -> k1_scale_copy()
//   src/sycl/sycl.cpp:100-173  enqueue_mixed_axis (K2,K3)  -> mixed_radix_axis()
//   src/sycl/sycl.cpp:175-234  enqueue_radix2_axis (K4,K5) -> pow2_axis()
//   src/sycl/sycl.cpp:236-266  host_radix2_fft             -> host_pow2_fft()
//   src/sycl/sycl.cpp:268-339  enqueue_bluestein_axis(K6-8)-> bluestein_axis()
//   src/sycl/sycl.cpp:509-569  plan-time table generation  -> OraclePlan ctor
//   src/sycl/sycl.cpp:688-775  impl::execute axis loop     -> OraclePlan::run()
//   src/core/provider_loader.cpp:112-132 checked_element_count
//   src/core/provider_loader.cpp:134-147 normalization_scale
//
// Arithmetic follows the reference: tables are generated with angles formed in
// the plan's Scalar type (float or double) with std::cos/std::sin, complex
// multiply is (ac-bd, ad+bc) as in third_party/syclcplx/sycl_ext_complex.hpp:569-580
// (the Annex-G NaN/Inf recovery branch there only fires on non-finite products,
// which the parity inputs never produce), and every SYCL parallel_for becomes an
// OpenMP parallel loop over the same index space. Work items inside one SYCL
// kernel are independent, so results are those of the SYCL kernels up to
// floating-point contraction (this file is built with -ffp-contract=off).
//
// C ABI (for ctypes): oracle_plan_create / oracle_plan_execute /
// oracle_plan_destroy / oracle_set_threads, see oracle/portable_ref.h.

#include "portable_ref.h"

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

template <class T>
struct cx {
    T re, im;
};

template <class T>
inline cx<T> mul(cx<T> a, cx<T> b) {
    // syclcplx operator* (finite branch): (ac - bd, ad + bc)
    const T ac = a.re * b.re;
    const T bd = a.im * b.im;
    const T ad = a.re * b.im;
    const T bc = a.im * b.re;
    return {ac - bd, ad + bc};
}
template <class T>
inline cx<T> add(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <class T>
inline cx<T> sub(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <class T>
inline cx<T> scale_by(cx<T> a, T s) { return {a.re * s, a.im * s}; }

template <class T>
constexpr T kPi = static_cast<T>(3.141592653589793238462643383279502884L);

struct OracleError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// sycl.cpp:34-46
std::size_t next_pow2(std::size_t v) {
    std::size_t r = 1;
    while (r < v) {
        if (r > std::numeric_limits<std::size_t>::max() / 2) {
            throw OracleError("Bluestein convolution size overflows size_t");
        }
        r *= 2;
    }
    return r;
}

// sycl.cpp:48-61: factors in the order 2..., 3..., 5..., 7...; empty if not 7-smooth.
std::vector<std::size_t> smooth_factors(std::size_t v) {
    std::vector<std::size_t> out;
    const std::size_t primes[4] = {2, 3, 5, 7};
    for (std::size_t p : primes) {
        while (v % p == 0) {
            out.push_back(p);
            v /= p;
        }
    }
    if (v != 1) out.clear();
    return out;
}

// sycl.cpp:63-70
std::size_t stride_after(const std::vector<std::size_t>& shape, std::size_t axis) {
    std::size_t s = 1;
    for (std::size_t i = axis + 1; i < shape.size(); ++i) s *= shape[i];
    return s;
}

bool is_pow2(std::size_t v) { return v != 0 && (v & (v - 1)) == 0; }

// provider_loader.cpp:134-147; mode: 0 none, 1 forward, 2 backward, 3 orthogonal
double norm_scale(int mode, int dir, std::size_t n) {
    switch (mode) {
        case 0: return 1.0;
        case 1: return dir == -1 ? 1.0 / static_cast<double>(n) : 1.0;
        case 2: return dir == 1 ? 1.0 / static_cast<double>(n) : 1.0;
        case 3: return 1.0 / std::sqrt(static_cast<double>(n));
        default: return 1.0;
    }
}

// K1, sycl.cpp:87-98
template <class T>
void k1_scale_copy(const cx<T>* in, cx<T>* out, std::size_t count, T s) {
#pragma omp parallel for schedule(static)
    for (std::int64_t i = 0; i < static_cast<std::int64_t>(count); ++i) out[i] = scale_by(in[i], s);
}

// K2 + K3, sycl.cpp:100-173
template <class T>
void mixed_radix_axis(const cx<T>* in, cx<T>* out, std::size_t total, std::size_t len,
                      std::size_t stride, const cx<T>* tw, const std::vector<std::size_t>& factors) {
    if (factors.size() > 64) throw OracleError("Too many mixed-radix stages");
    const std::size_t nf = factors.size();
    // K2: digit-reversal gather (radices consumed in factor order).
#pragma omp parallel for schedule(static)
    for (std::int64_t li = 0; li < static_cast<std::int64_t>(total); ++li) {
        const std::size_t linear = static_cast<std::size_t>(li);
        const std::size_t coord = (linear / stride) % len;
        const std::size_t base = linear - coord * stride;
        std::size_t src = 0, rem = len, digits = coord;
        for (std::size_t s = 0; s < nf; ++s) {
            const std::size_t r = factors[s];
            rem /= r;
            src += (digits % r) * rem;
            digits /= r;
        }
        out[linear] = in[base + src * stride];
    }
    // K3: one O(r^2) butterfly kernel per factor.
    const std::size_t lines = total / len;
    std::size_t stage = 1;
    for (std::size_t r : factors) {
        const std::size_t prev = stage;
        stage *= r;
        const std::size_t per_line = len / r;
        const std::int64_t work = static_cast<std::int64_t>(lines * per_line);
#pragma omp parallel for schedule(static)
        for (std::int64_t bi = 0; bi < work; ++bi) {
            const std::size_t b = static_cast<std::size_t>(bi);
            const std::size_t line = b / per_line;
            const std::size_t in_line = b % per_line;
            const std::size_t group = in_line / prev;
            const std::size_t j = in_line % prev;
            const std::size_t outer = line / stride;
            const std::size_t inner = line % stride;
            const std::size_t base =
                outer * len * stride + inner + group * stage * stride + j * stride;
            cx<T> v[7];
            for (std::size_t q = 0; q < r; ++q) {
                v[q] = mul(out[base + q * prev * stride], tw[(q * j * (len / stage)) % len]);
            }
            for (std::size_t p = 0; p < r; ++p) {
                cx<T> acc{T(0), T(0)};
                for (std::size_t q = 0; q < r; ++q) {
                    acc = add(acc, mul(v[q], tw[(q * p * (len / r)) % len]));
                }
                out[base + p * prev * stride] = acc;
            }
        }
    }
}

// K4 + K5, sycl.cpp:175-234
template <class T>
void pow2_axis(const cx<T>* in, cx<T>* out, std::size_t total, std::size_t len, std::size_t stride,
               const cx<T>* tw, bool conj_tw) {
    unsigned bits = 0;
    for (std::size_t v = len; v > 1; v >>= 1) ++bits;
#pragma omp parallel for schedule(static)
    for (std::int64_t li = 0; li < static_cast<std::int64_t>(total); ++li) {
        const std::size_t linear = static_cast<std::size_t>(li);
        const std::size_t coord = (linear / stride) % len;
        std::size_t rev = 0, v = coord;
        for (unsigned b = 0; b < bits; ++b) {
            rev = (rev << 1) | (v & 1);
            v >>= 1;
        }
        const std::size_t base = linear - coord * stride;
        out[linear] = in[base + rev * stride];
    }
    const std::size_t lines = total / len;
    for (std::size_t stage = 2; stage <= len; stage <<= 1) {
        const std::size_t half = stage / 2;
        const std::int64_t work = static_cast<std::int64_t>(lines * (len / 2));
#pragma omp parallel for schedule(static)
        for (std::int64_t pi = 0; pi < work; ++pi) {
            const std::size_t pair = static_cast<std::size_t>(pi);
            const std::size_t line = pair / (len / 2);
            const std::size_t pin = pair % (len / 2);
            const std::size_t group = pin / half;
            const std::size_t j = pin % half;
            const std::size_t outer = line / stride;
            const std::size_t inner = line % stride;
            const std::size_t base = outer * len * stride + inner;
            const std::size_t first = base + (group * stage + j) * stride;
            const std::size_t second = first + half * stride;
            cx<T> w = tw[j * (len / stage)];
            if (conj_tw) w.im = -w.im;
            const cx<T> lhs = out[first];
            const cx<T> rhs = mul(out[second], w);
            out[first] = add(lhs, rhs);
            out[second] = sub(lhs, rhs);
        }
    }
}

// sycl.cpp:236-266: in-place iterative radix-2 DIT, per-butterfly cos/sin in T.
template <class T>
void host_pow2_fft(std::vector<cx<T>>& a, int dir) {
    const std::size_t n = a.size();
    for (std::size_t i = 1, rev = 0; i < n; ++i) {
        std::size_t bit = n >> 1;
        while (rev & bit) {
            rev ^= bit;
            bit >>= 1;
        }
        rev ^= bit;
        if (i < rev) std::swap(a[i], a[rev]);
    }
    const T sgn = dir == -1 ? T(-1) : T(1);
    const T two_pi = T(2) * kPi<T>;
    for (std::size_t stage = 2; stage <= n; stage *= 2) {
        for (std::size_t base = 0; base < n; base += stage) {
            for (std::size_t j = 0; j < stage / 2; ++j) {
                const T ang = sgn * two_pi * static_cast<T>(j) / static_cast<T>(stage);
                const cx<T> w{std::cos(ang), std::sin(ang)};
                const cx<T> lhs = a[base + j];
                const cx<T> rhs = mul(a[base + j + stage / 2], w);
                a[base + j] = add(lhs, rhs);
                a[base + j + stage / 2] = sub(lhs, rhs);
            }
        }
    }
}

// K6, radix-2 FFT_M, K7, radix-2 IFFT_M (conjugated twiddles), K8; sycl.cpp:268-339
template <class T>
void bluestein_axis(const cx<T>* in, cx<T>* first, cx<T>* second, std::size_t total,
                    std::size_t len, std::size_t stride, std::size_t m, const cx<T>* chirp,
                    const cx<T>* spectrum, const cx<T>* conv_tw) {
    const std::size_t lines = total / len;
    const std::size_t expanded = lines * m;
#pragma omp parallel for schedule(static)
    for (std::int64_t ei = 0; ei < static_cast<std::int64_t>(expanded); ++ei) {
        const std::size_t e = static_cast<std::size_t>(ei);
        const std::size_t line = e / m;
        const std::size_t c = e % m;
        if (c < len) {
            const std::size_t outer = line / stride;
            const std::size_t inner = line % stride;
            first[e] = mul(in[outer * len * stride + inner + c * stride], chirp[c]);
        } else {
            first[e] = {T(0), T(0)};
        }
    }
    pow2_axis(first, second, expanded, m, 1, conv_tw, false);
#pragma omp parallel for schedule(static)
    for (std::int64_t ei = 0; ei < static_cast<std::int64_t>(expanded); ++ei) {
        const std::size_t e = static_cast<std::size_t>(ei);
        second[e] = mul(second[e], spectrum[e % m]);
    }
    pow2_axis(second, first, expanded, m, 1, conv_tw, true);
    const T inv = T(1) / static_cast<T>(m);
#pragma omp parallel for schedule(static)
    for (std::int64_t li = 0; li < static_cast<std::int64_t>(total); ++li) {
        const std::size_t linear = static_cast<std::size_t>(li);
        const std::size_t c = (linear / stride) % len;
        const std::size_t line = (linear / (len * stride)) * stride + linear % stride;
        const cx<T> ch{chirp[c].re * inv, chirp[c].im * inv};
        second[linear] = mul(first[line * m + c], ch);
    }
}

struct AxisTables {
    bool bluestein = false;
    std::size_t m = 0;
    std::vector<std::size_t> factors;
    // untyped storage; reinterpreted as cx<T>
    std::vector<unsigned char> twiddles, chirp, spectrum, conv_tw;
};

template <class T>
std::vector<unsigned char> to_bytes(const std::vector<cx<T>>& v) {
    std::vector<unsigned char> b(v.size() * sizeof(cx<T>));
    if (!b.empty()) std::memcpy(b.data(), v.data(), b.size());
    return b;
}

template <class T>
std::vector<cx<T>> make_twiddles(std::size_t len, T sgn) {
    // sycl.cpp:509-518: angle formed in T
    std::vector<cx<T>> t(len);
    const T two_pi = T(2) * kPi<T>;
    for (std::size_t i = 0; i < len; ++i) {
        const T ang = sgn * two_pi * static_cast<T>(i) / static_cast<T>(len);
        t[i] = {std::cos(ang), std::sin(ang)};
    }
    return t;
}

struct OraclePlan {
    bool dbl = false;
    int dir = -1;
    int norm = 0;
    std::vector<std::size_t> shape;
    std::size_t batch = 0, elements = 0, transform = 0, scratch_elems = 0;
    std::vector<AxisTables> axes;
    std::vector<unsigned char> scratch_a, scratch_b;

    template <class T>
    void build() {
        const T sgn = dir == -1 ? T(-1) : T(1);
        scratch_elems = elements;
        for (std::size_t axis = 0; axis < shape.size(); ++axis) {
            AxisTables at;
            const std::size_t len = shape[axis];
            at.factors = smooth_factors(len);
            if (!at.factors.empty() || len == 1) {
                at.twiddles = to_bytes(make_twiddles<T>(len, sgn));
                axes.push_back(std::move(at));
                continue;
            }
            // sycl.cpp:530-568
            if (len > std::numeric_limits<std::size_t>::max() / 2 + 1) {
                throw OracleError("Bluestein convolution size overflows size_t");
            }
            at.bluestein = true;
            at.m = next_pow2(2 * len - 1);
            const std::size_t lines = elements / len;
            if (lines > std::numeric_limits<std::size_t>::max() / at.m) {
                throw OracleError("Bluestein scratch size overflows size_t");
            }
            scratch_elems = std::max(scratch_elems, lines * at.m);
            std::vector<cx<T>> kern(at.m, cx<T>{T(0), T(0)});
            std::vector<cx<T>> chirp(len);
            const T pi = kPi<T>;
            for (std::size_t i = 0; i < len; ++i) {
                const T sq = static_cast<T>(i) * static_cast<T>(i);
                const T ang = -sgn * pi * sq / static_cast<T>(len);
                const cx<T> v{std::cos(ang), std::sin(ang)};
                kern[i] = v;
                if (i != 0) kern[at.m - i] = v;
                chirp[i] = {v.re, -v.im};
            }
            host_pow2_fft(kern, -1);
            at.chirp = to_bytes(chirp);
            at.spectrum = to_bytes(kern);
            at.conv_tw = to_bytes(make_twiddles<T>(at.m, T(-1)));
            axes.push_back(std::move(at));
        }
        scratch_a.assign(scratch_elems * sizeof(cx<T>), 0);
        scratch_b.assign(scratch_elems * sizeof(cx<T>), 0);
    }

    template <class T>
    void run(const void* input, void* output) {
        cx<T>* sa = reinterpret_cast<cx<T>*>(scratch_a.data());
        cx<T>* sb = reinterpret_cast<cx<T>*>(scratch_b.data());
        const cx<T>* cur_in = static_cast<const cx<T>*>(input);
        cx<T>* cur_out = sa;
        for (std::size_t axis = 0; axis < shape.size(); ++axis) {
            const AxisTables& at = axes[axis];
            const std::size_t len = shape[axis];
            const std::size_t stride = stride_after(shape, axis);
            if (!at.bluestein) {
                cur_out = (cur_in == sa) ? sb : sa;
                const cx<T>* tw = reinterpret_cast<const cx<T>*>(at.twiddles.data());
                if (is_pow2(len)) {
                    pow2_axis(cur_in, cur_out, elements, len, stride, tw, false);
                } else {
                    mixed_radix_axis(cur_in, cur_out, elements, len, stride, tw, at.factors);
                }
            } else {
                cx<T>* first = (cur_in == sa) ? sb : sa;
                cx<T>* second = (first == sa) ? sb : sa;
                bluestein_axis(cur_in, first, second, elements, len, stride, at.m,
                               reinterpret_cast<const cx<T>*>(at.chirp.data()),
                               reinterpret_cast<const cx<T>*>(at.spectrum.data()),
                               reinterpret_cast<const cx<T>*>(at.conv_tw.data()));
                cur_out = second;
            }
            cur_in = cur_out;
        }
        const T s = static_cast<T>(norm_scale(norm, dir, transform));
        k1_scale_copy(cur_in, static_cast<cx<T>*>(output), elements, s);
    }
};

void set_err(char* err, std::size_t cap, const char* msg) {
    if (!err || cap == 0) return;
    std::size_t n = std::strlen(msg);
    if (n > cap - 1) n = cap - 1;
    std::memcpy(err, msg, n);
    err[n] = '\0';
}

}  // namespace

extern "C" {

void* oracle_plan_create(int double_precision, int direction, int normalization, unsigned rank,
                         const uint64_t* lengths, uint64_t batch, char* err, size_t cap) {
    try {
        // provider_loader.cpp:112-132 checked_element_count
        if (rank == 0 || rank > 3) throw OracleError("FFT rank must be between 1 and 3");
        if (batch == 0) throw OracleError("FFT batch count must be non-zero");
        if (direction != -1 && direction != 1) throw OracleError("Invalid FFT direction");
        auto* p = new OraclePlan();
        p->dbl = double_precision != 0;
        p->dir = direction;
        p->norm = normalization;
        p->batch = batch;
        std::size_t count = batch, tsize = 1;
        for (unsigned i = 0; i < rank; ++i) {
            const std::size_t len = lengths[i];
            if (len == 0) {
                delete p;
                throw OracleError("FFT dimensions must be non-zero");
            }
            if (count > std::numeric_limits<std::size_t>::max() / len) {
                delete p;
                throw OracleError("FFT element count overflows size_t");
            }
            count *= len;
            tsize *= len;
            p->shape.push_back(len);
        }
        p->elements = count;
        p->transform = tsize;
        try {
            if (p->dbl) p->build<double>(); else p->build<float>();
        } catch (...) {
            delete p;
            throw;
        }
        return p;
    } catch (const std::exception& e) {
        set_err(err, cap, e.what());
        return nullptr;
    }
}

int oracle_plan_execute(void* plan, const void* in, void* out, char* err, size_t cap) {
    try {
        auto* p = static_cast<OraclePlan*>(plan);
        if (!p || !in || !out) throw OracleError("invalid oracle execution argument");
        if (p->dbl) p->run<double>(in, out); else p->run<float>(in, out);
        return 0;
    } catch (const std::exception& e) {
        set_err(err, cap, e.what());
        return 1;
    }
}

void oracle_plan_destroy(void* plan) { delete static_cast<OraclePlan*>(plan); }

uint64_t oracle_plan_scratch_bytes(const void* plan) {
    const auto* p = static_cast<const OraclePlan*>(plan);
    return p ? 2ull * p->scratch_elems * (p->dbl ? 16ull : 8ull) : 0ull;
}

void oracle_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
