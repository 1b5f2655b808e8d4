// syclfft B200: C++ front end.
//
// A headless mirror of the reference's SYCL front end for builds without a SYCL
// compiler: the same plan surface (include/syclfft/syclfft.hpp:45-130), the same enums,
// options, error codes and exception (include/syclfft/common.hpp:34-128), the same
// validation and serialisation rules (src/sycl/sycl.cpp:424-491, 615-641, 818-907), and the
// same provider-module loading rules (src/core/provider_loader.cpp:168-232): the B200
// provider module syclfft_provider_b200 is found in $SYCLFFT_PLUGIN_PATH or in
// <directory of this library>/syclfft/providers, resolved with dlsym, and rejected with
// error_code::plugin_error when its ABI version differs.
//
// The SYCL types map to CUDA: `queue` is a device ordinal plus a cudaStream_t, `event`
// wraps a cudaEvent_t recorded after the transform. complex<Scalar> is std::complex
// (interleaved re, im -- the layout syclcplx uses).
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#define SYCLFFT_B200_CXX_EXPORT __attribute__((visibility("default")))

struct CUstream_st;
struct CUevent_st;

namespace syclfft_b200 {

enum class direction { forward = -1, backward = 1 };
enum class placement { in_place, out_of_place };
enum class normalization { none, forward, backward, orthogonal };
enum class planning_mode { estimate, measure };
// common.hpp:56-64 plus the slot of this provider.
enum class provider { automatic, portable_sycl, fftw, cufft, rocfft, onemkl, b200 };

struct plan_options {
    syclfft_b200::placement placement = syclfft_b200::placement::out_of_place;
    syclfft_b200::normalization normalization = syclfft_b200::normalization::none;
    planning_mode planning = planning_mode::estimate;
    provider preferred_provider = provider::automatic;
    // B200 extension, no counterpart in syclfft::plan_options: complex<float> plans run the
    // radix-16 butterflies of eligible axes (256 / 4096 points) as BF16 hi/lo products with
    // FP32 accumulation on the tensor cores (about 1e-5 relative L2); ignored for double.
    bool split_precision = false;
};

// B200 extension (the reference's plans read and write contiguous batch-major arrays only):
// element (b, i0, .., i_{rank-1}) of the input is at b * in_distance + sum_k i_k * in_strides[k]
// complex elements from the input pointer, and likewise for the output. One stride per axis,
// strides >= 1, distances >= 1 when batch_count > 1; the output layout must not overlap
// itself and an in-place plan needs equal layouts (invalid_argument otherwise).
struct data_layout {
    std::vector<std::ptrdiff_t> in_strides;
    std::ptrdiff_t in_distance = 0;
    std::vector<std::ptrdiff_t> out_strides;
    std::ptrdiff_t out_distance = 0;
};

// B200 extension: kind of a real transform (real_plan).
enum class real_kind { r2c, c2r };

struct provider_status {
    provider id{};
    std::string name;
    bool built{};
    bool available{};
    std::string reason;
};

enum class error_code {
    invalid_argument,
    invalid_state,
    invalid_pointer,
    unsupported_precision,
    provider_unavailable,
    planning_failed,
    execution_failed,
    plugin_error,
};

class SYCLFFT_B200_CXX_EXPORT exception : public std::runtime_error {
public:
    exception(error_code code, const std::string& message) : std::runtime_error(message), code_(code) {}
    [[nodiscard]] error_code code() const noexcept { return code_; }

private:
    error_code code_;
};

// Stand-in for sycl::queue: where work runs and is ordered.
struct queue {
    int device = -1;                    // CUDA ordinal, -1 = current device
    CUstream_st* stream = nullptr;      // cudaStream_t; nullptr = legacy default stream
};

// Stand-in for sycl::event: completion of one execution. wait_and_throw() also reports a
// failed device wait of that execution (a bounded wait in one of the plan's kernels gave up,
// so its output is incomplete) as error_code::execution_failed, the code the reference gives
// a failed provider execution (src/sycl/sycl.cpp:671-676); each failure is reported once.
class SYCLFFT_B200_CXX_EXPORT event {
public:
    event() = default;
    void wait_and_throw() const;
    [[nodiscard]] bool valid() const noexcept { return static_cast<bool>(ev_); }
    [[nodiscard]] CUevent_st* native() const noexcept { return ev_ ? ev_.get() : nullptr; }
    static event record(CUstream_st* stream);
    // An event whose wait_and_throw() also reads and clears the status word of the provider
    // plan `plan` through `take_status`; `owner` keeps that plan alive as long as the event.
    static event record(CUstream_st* stream, std::shared_ptr<void> owner, void* plan, int (*take_status)(void*));

private:
    std::shared_ptr<CUevent_st> ev_;
    std::shared_ptr<void> owner_;
    void* plan_ = nullptr;
    int (*take_status_)(void*) = nullptr;
};

template <class Scalar>
using complex = std::complex<Scalar>;

template <class Scalar>
class SYCLFFT_B200_CXX_EXPORT plan {
    static_assert(std::is_same_v<Scalar, float> || std::is_same_v<Scalar, double>,
                  "syclfft supports float and double precision");

public:
    using scalar_type = Scalar;
    using complex_type = complex<Scalar>;

    plan(const plan&) = delete;
    plan& operator=(const plan&) = delete;
    plan(plan&&) noexcept;
    plan& operator=(plan&&) noexcept;
    ~plan();

    event execute(complex_type* inout);
    event execute(complex_type* inout, const event& dependency);
    event execute(complex_type* inout, const std::vector<event>& dependencies);

    event execute(const complex_type* input, complex_type* output);
    event execute(const complex_type* input, complex_type* output, const event& dependency);
    event execute(const complex_type* input, complex_type* output, const std::vector<event>& dependencies);

    [[nodiscard]] std::vector<std::size_t> shape() const;
    [[nodiscard]] std::size_t batch_count() const noexcept;
    [[nodiscard]] syclfft_b200::direction direction() const noexcept;
    [[nodiscard]] provider selected_provider() const noexcept;
    [[nodiscard]] std::size_t scratch_size_bytes() const noexcept;

    plan(queue q, std::vector<std::size_t> lengths, std::size_t batch_count, syclfft_b200::direction dir,
         plan_options options);
    // B200 extension: strided input / output (data_layout)
    plan(queue q, std::vector<std::size_t> lengths, std::size_t batch_count, syclfft_b200::direction dir,
         plan_options options, const data_layout& layout);

private:
    class impl;
    std::unique_ptr<impl> impl_;
};

// B200 extension, no counterpart in the reference (its v0.1 scope is complex-to-complex):
// batched real transforms of rank 1-3 with an even last length n, out of place, in numpy's
// rfftn / irfftn layouts. r2c (forward): prod(shape) reals per transform in,
// prod(shape[0..rank-2]) x (n/2 + 1) complex out. c2r (backward): the reverse (the imaginary
// parts of bins 0 and n/2 of every last-axis line are ignored). plan_options::normalization
// scales relative to prod(shape) as for a complex plan of that shape; placement must be
// out_of_place.
template <class Scalar>
class SYCLFFT_B200_CXX_EXPORT real_plan {
    static_assert(std::is_same_v<Scalar, float> || std::is_same_v<Scalar, double>,
                  "syclfft supports float and double precision");

public:
    using scalar_type = Scalar;
    using complex_type = complex<Scalar>;

    real_plan(const real_plan&) = delete;
    real_plan& operator=(const real_plan&) = delete;
    real_plan(real_plan&&) noexcept;
    real_plan& operator=(real_plan&&) noexcept;
    ~real_plan();

    // r2c plans (invalid_argument on a c2r plan)
    event execute(const Scalar* input, complex_type* output, const std::vector<event>& dependencies = {});
    // c2r plans (invalid_argument on an r2c plan)
    event execute(const complex_type* input, Scalar* output, const std::vector<event>& dependencies = {});

    [[nodiscard]] std::size_t length() const noexcept;  // the last (real) length n
    [[nodiscard]] std::vector<std::size_t> shape() const;
    [[nodiscard]] std::size_t batch_count() const noexcept;
    [[nodiscard]] real_kind kind() const noexcept;

    real_plan(queue q, std::size_t n, std::size_t batch_count, real_kind kind, plan_options options);
    real_plan(queue q, std::vector<std::size_t> lengths, std::size_t batch_count, real_kind kind,
              plan_options options);

private:
    class impl;
    std::unique_ptr<impl> impl_;
};

SYCLFFT_B200_CXX_EXPORT std::vector<provider_status> query_providers(const queue& q);

template <class Scalar>
plan<Scalar> plan_many_dft(queue q, const std::vector<std::size_t>& lengths, std::size_t batch_count,
                           direction dir, plan_options options = {}) {
    return plan<Scalar>(q, lengths, batch_count, dir, options);
}

template <class Scalar>
plan<Scalar> plan_many_dft(queue q, std::initializer_list<std::size_t> lengths, std::size_t batch_count,
                           direction dir, plan_options options = {}) {
    return plan<Scalar>(q, {lengths.begin(), lengths.end()}, batch_count, dir, options);
}

// B200 extension: strided layouts (data_layout)
template <class Scalar>
plan<Scalar> plan_many_dft(queue q, const std::vector<std::size_t>& lengths, std::size_t batch_count,
                           direction dir, plan_options options, const data_layout& layout) {
    return plan<Scalar>(q, lengths, batch_count, dir, options, layout);
}

template <class Scalar>
real_plan<Scalar> plan_dft_r2c_1d(queue q, std::size_t n, std::size_t batch_count = 1, plan_options options = {}) {
    return real_plan<Scalar>(q, n, batch_count, real_kind::r2c, options);
}

template <class Scalar>
real_plan<Scalar> plan_dft_c2r_1d(queue q, std::size_t n, std::size_t batch_count = 1, plan_options options = {}) {
    return real_plan<Scalar>(q, n, batch_count, real_kind::c2r, options);
}

template <class Scalar>
real_plan<Scalar> plan_dft_r2c(queue q, const std::vector<std::size_t>& lengths, std::size_t batch_count = 1,
                               plan_options options = {}) {
    return real_plan<Scalar>(q, lengths, batch_count, real_kind::r2c, options);
}

template <class Scalar>
real_plan<Scalar> plan_dft_c2r(queue q, const std::vector<std::size_t>& lengths, std::size_t batch_count = 1,
                               plan_options options = {}) {
    return real_plan<Scalar>(q, lengths, batch_count, real_kind::c2r, options);
}

template <class Scalar>
plan<Scalar> plan_dft_1d(queue q, std::size_t n, direction dir, plan_options options = {}) {
    return plan_many_dft<Scalar>(q, {n}, 1, dir, options);
}

template <class Scalar>
plan<Scalar> plan_dft_2d(queue q, std::size_t n0, std::size_t n1, direction dir, plan_options options = {}) {
    return plan_many_dft<Scalar>(q, {n0, n1}, 1, dir, options);
}

template <class Scalar>
plan<Scalar> plan_dft_3d(queue q, std::size_t n0, std::size_t n1, std::size_t n2, direction dir,
                         plan_options options = {}) {
    return plan_many_dft<Scalar>(q, {n0, n1, n2}, 1, dir, options);
}

namespace detail {
// provider_loader.cpp:112-147
SYCLFFT_B200_CXX_EXPORT std::size_t checked_element_count(const std::vector<std::size_t>& lengths,
                                                          std::size_t batch_count);
SYCLFFT_B200_CXX_EXPORT double normalization_scale(normalization mode, direction dir, std::size_t transform_size);
SYCLFFT_B200_CXX_EXPORT const char* provider_name(provider value) noexcept;
// provider_loader.cpp:168-176: $SYCLFFT_PLUGIN_PATH entries, then <libdir>/syclfft/providers.
SYCLFFT_B200_CXX_EXPORT std::vector<std::string> provider_search_paths();
}  // namespace detail

extern template class plan<float>;
extern template class plan<double>;
extern template class real_plan<float>;
extern template class real_plan<double>;

}  // namespace syclfft_b200
