// The reference's portable-provider test program (tests/sycl_tests.cpp), restated for the
// C++ front end of the B200 provider (include/syclfft_b200.hpp). Same cases, inputs,
// direct-DFT oracles, tolerances and error-code checks; device buffers come from
// cudaMalloc instead of SYCL USM, events are CUDA events. Needs a GPU; run by
// tests/test_frontend.py. Exit status 0 = every check passed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/syclfft_b200.hpp"

namespace sf = syclfft_b200;

namespace {

void check(bool condition, const std::string& message) {
    if (!condition) throw std::runtime_error(message);
}

sf::plan_options make_plan_options(sf::placement placement = sf::placement::out_of_place,
                                   sf::normalization normalization = sf::normalization::none,
                                   sf::provider provider = sf::provider::automatic) {
    sf::plan_options o;
    o.placement = placement;
    o.normalization = normalization;
    o.preferred_provider = provider;
    return o;
}

template <class F>
void expect_error(sf::error_code code, F&& fn) {
    try {
        fn();
    } catch (const sf::exception& ex) {
        check(ex.code() == code, std::string("wrong exception code: ") + ex.what());
        return;
    }
    throw std::runtime_error("expected syclfft_b200::exception");
}

template <class T>
class device_buffer {
public:
    explicit device_buffer(std::size_t count) : count_(count) {
        if (cudaMalloc(&ptr_, count * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    }
    ~device_buffer() { cudaFree(ptr_); }
    device_buffer(const device_buffer&) = delete;
    device_buffer& operator=(const device_buffer&) = delete;
    T* get() const { return static_cast<T*>(ptr_); }
    void write(const std::vector<T>& v) {
        check(v.size() == count_, "upload size mismatch");
        check(cudaMemcpy(ptr_, v.data(), count_ * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess, "upload");
    }
    std::vector<T> read() const {
        std::vector<T> v(count_);
        check(cudaMemcpy(v.data(), ptr_, count_ * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess, "download");
        return v;
    }

private:
    std::size_t count_;
    void* ptr_ = nullptr;
};

// sycl_tests.cpp:91-112
template <class Scalar>
std::vector<std::complex<Scalar>> direct_dft(const std::vector<std::complex<Scalar>>& input, sf::direction dir,
                                             sf::normalization norm) {
    const auto count = input.size();
    std::vector<std::complex<Scalar>> output(count);
    const auto sign = dir == sf::direction::forward ? Scalar{-1} : Scalar{1};
    const auto pi = std::acos(Scalar{-1});
    for (std::size_t k = 0; k < count; ++k)
        for (std::size_t n = 0; n < count; ++n) {
            const auto angle = sign * Scalar{2} * pi * static_cast<Scalar>(k * n) / static_cast<Scalar>(count);
            output[k] += input[n] * std::complex<Scalar>{std::cos(angle), std::sin(angle)};
        }
    const auto scale = static_cast<Scalar>(sf::detail::normalization_scale(norm, dir, count));
    for (auto& v : output) v *= scale;
    return output;
}

// sycl_tests.cpp:115-151
template <class Scalar>
std::vector<std::complex<Scalar>> reference_many(std::vector<std::complex<Scalar>> values,
                                                 const std::vector<std::size_t>& shape, std::size_t batch,
                                                 sf::direction dir) {
    std::size_t transform = 1;
    for (auto n : shape) transform *= n;
    const auto sign = dir == sf::direction::forward ? Scalar{-1} : Scalar{1};
    const auto pi = std::acos(Scalar{-1});
    for (std::size_t axis = 0; axis < shape.size(); ++axis) {
        auto output = values;
        std::size_t stride = 1;
        for (std::size_t i = axis + 1; i < shape.size(); ++i) stride *= shape[i];
        const auto length = shape[axis];
        for (std::size_t b = 0; b < batch; ++b) {
            const auto offset = b * transform;
            for (std::size_t linear = 0; linear < transform; ++linear) {
                const auto coordinate = (linear / stride) % length;
                const auto base = linear - coordinate * stride;
                std::complex<Scalar> sum{};
                for (std::size_t k = 0; k < length; ++k) {
                    const auto angle = sign * Scalar{2} * pi * static_cast<Scalar>(coordinate * k) /
                                       static_cast<Scalar>(length);
                    sum += values[offset + base + k * stride] * std::complex<Scalar>{std::cos(angle), std::sin(angle)};
                }
                output[offset + linear] = sum;
            }
        }
        values = std::move(output);
    }
    return values;
}

template <class Scalar>
void run_many(const std::vector<std::size_t>& shape, std::size_t batch) {
    std::size_t count = batch;
    for (auto n : shape) count *= n;
    std::vector<std::complex<Scalar>> source(count);
    for (std::size_t i = 0; i < count; ++i)
        source[i] = {static_cast<Scalar>((i * 11 + 2) % 17) / Scalar{8}, static_cast<Scalar>((i * 3 + 1) % 13) / Scalar{7}};
    const auto expected = reference_many(source, shape, batch, sf::direction::forward);
    device_buffer<std::complex<Scalar>> input(count), output(count);
    input.write(source);
    auto fft = sf::plan_many_dft<Scalar>(sf::queue{}, shape, batch, sf::direction::forward,
                                         make_plan_options(sf::placement::out_of_place, sf::normalization::none,
                                                           sf::provider::b200));
    fft.execute(input.get(), output.get()).wait_and_throw();
    const auto actual = output.read();
    const auto tol = std::is_same_v<Scalar, float> ? Scalar{8e-4} : Scalar{5e-11};
    for (std::size_t i = 0; i < count; ++i)
        check(std::abs(actual[i] - expected[i]) <= tol * (Scalar{1} + std::abs(expected[i])),
              "multidimensional or batch mismatch at element " + std::to_string(i));
}

template <class Scalar>
void run_1d(std::size_t count, sf::direction dir, sf::normalization norm, sf::placement pl) {
    std::vector<std::complex<Scalar>> source(count);
    for (std::size_t i = 0; i < count; ++i)
        source[i] = {static_cast<Scalar>((i * 5 + 1) % 9) / Scalar{4}, static_cast<Scalar>((i * 3 + 2) % 7) / Scalar{5}};
    const auto expected = direct_dft(source, dir, norm);
    device_buffer<std::complex<Scalar>> input(count);
    std::unique_ptr<device_buffer<std::complex<Scalar>>> out_storage, repeat_storage;
    if (pl == sf::placement::out_of_place) {
        out_storage = std::make_unique<device_buffer<std::complex<Scalar>>>(count);
        repeat_storage = std::make_unique<device_buffer<std::complex<Scalar>>>(count);
    }
    input.write(source);
    auto fft = sf::plan_dft_1d<Scalar>(sf::queue{}, count, dir, make_plan_options(pl, norm, sf::provider::b200));
    auto dependency = sf::event::record(nullptr);
    auto ev = pl == sf::placement::in_place ? fft.execute(input.get(), dependency)
                                            : fft.execute(input.get(), out_storage->get(), dependency);
    sf::event repeated;
    if (repeat_storage) repeated = fft.execute(input.get(), repeat_storage->get());
    ev.wait_and_throw();
    repeated.wait_and_throw();
    const auto actual = out_storage ? out_storage->read() : input.read();
    const auto again = repeat_storage ? repeat_storage->read() : std::vector<std::complex<Scalar>>{};
    const auto tol = std::is_same_v<Scalar, float> ? Scalar{4e-4} : Scalar{2e-11};
    for (std::size_t i = 0; i < count; ++i) {
        if (std::abs(actual[i] - expected[i]) > tol * (Scalar{1} + std::abs(expected[i])))
            throw std::runtime_error("b200 mismatch at element " + std::to_string(i));
        if (repeat_storage)
            check(std::abs(again[i] - expected[i]) <= tol * (Scalar{1} + std::abs(expected[i])),
                  "serialized repeated execution mismatch");
    }
    check(fft.selected_provider() == sf::provider::b200, "wrong provider");
}

}  // namespace

int main()
try {
    static_assert(sizeof(sf::complex<float>) == 2 * sizeof(float));
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
        std::cerr << "no CUDA device\n";
        return 2;
    }
    for (auto norm : {sf::normalization::none, sf::normalization::forward, sf::normalization::backward,
                      sf::normalization::orthogonal})
        run_1d<float>(8, sf::direction::forward, norm, sf::placement::out_of_place);
    run_1d<float>(7, sf::direction::backward, sf::normalization::none, sf::placement::in_place);
    run_1d<float>(6, sf::direction::forward, sf::normalization::none, sf::placement::out_of_place);
    run_1d<float>(15, sf::direction::backward, sf::normalization::none, sf::placement::out_of_place);
    run_1d<float>(35, sf::direction::forward, sf::normalization::none, sf::placement::out_of_place);
    run_1d<float>(11, sf::direction::backward, sf::normalization::none, sf::placement::in_place);
    run_many<float>({3, 4}, 2);
    run_many<float>({2, 3, 5}, 1);
    run_many<float>({11, 3}, 1);
    run_1d<double>(11, sf::direction::forward, sf::normalization::orthogonal, sf::placement::out_of_place);

    {  // sycl_tests.cpp:367-399: N=13 round trip chained by an event
        device_buffer<std::complex<float>> input(13), spectrum(13), restored(13);
        std::vector<std::complex<float>> source(13);
        for (std::size_t i = 0; i < 13; ++i) source[i] = {static_cast<float>(i) / 7.0f, static_cast<float>(i % 3) / 5.0f};
        input.write(source);
        auto forward = sf::plan_dft_1d<float>(sf::queue{}, 13, sf::direction::forward);
        auto backward = sf::plan_dft_1d<float>(sf::queue{}, 13, sf::direction::backward,
                                               make_plan_options(sf::placement::out_of_place, sf::normalization::backward));
        const auto forward_done = forward.execute(input.get(), spectrum.get());
        backward.execute(spectrum.get(), restored.get(), forward_done).wait_and_throw();
        const auto actual = restored.read();
        for (std::size_t i = 0; i < 13; ++i) check(std::abs(actual[i] - source[i]) < 2e-3f, "round trip mismatch");
    }

    const auto providers = sf::query_providers(sf::queue{});
    check(!providers.empty() && providers.front().available, "b200 provider unavailable");
    {
        auto automatic = sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward);
        check(automatic.selected_provider() == sf::provider::b200, "automatic selection did not pick b200");
    }
    {  // sycl_tests.cpp:410-435: two plans on two streams
        device_buffer<std::complex<float>> ia(8), ib(8), oa(8), ob(8);
        std::vector<std::complex<float>> sa(8), sb(8);
        sa[0] = {1.0f, 0.0f};
        sb[1] = {1.0f, 0.0f};
        ia.write(sa);
        ib.write(sb);
        cudaStream_t s2;
        check(cudaStreamCreate(&s2) == cudaSuccess, "stream");
        auto first = sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward);
        auto second = sf::plan_dft_1d<float>(sf::queue{-1, reinterpret_cast<CUstream_st*>(s2)}, 8, sf::direction::forward);
        auto d1 = first.execute(ia.get(), oa.get());
        auto d2 = second.execute(ib.get(), ob.get());
        d1.wait_and_throw();
        d2.wait_and_throw();
        const auto a = oa.read();
        const auto b = ob.read();
        check(std::abs(a[0].real() - 1.0f) < 1e-5f && std::abs(b[0].real() - 1.0f) < 1e-5f, "concurrent plans failed");
        cudaStreamDestroy(s2);
    }
    {  // sycl_tests.cpp:437-449: memory the plan's device cannot see -> invalid_pointer
        std::vector<std::complex<float>> host(8);
        device_buffer<std::complex<float>> output(8);
        expect_error(sf::error_code::invalid_pointer, [&] {
            auto fft = sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward);
            fft.execute(host.data(), output.get());
        });
    }
    {  // sycl_tests.cpp:483-506: two producers on another stream, the FFT waits on both events
        device_buffer<std::complex<float>> input(8), output(8);
        cudaStream_t producer;
        check(cudaStreamCreate(&producer) == cudaSuccess, "stream");
        std::vector<std::complex<float>> impulse(4);
        impulse[0] = {1.0f, 0.0f};
        cudaMemcpyAsync(input.get(), impulse.data(), 4 * sizeof(std::complex<float>), cudaMemcpyHostToDevice, producer);
        auto first_half = sf::event::record(reinterpret_cast<CUstream_st*>(producer));
        cudaMemsetAsync(input.get() + 4, 0, 4 * sizeof(std::complex<float>), producer);
        auto second_half = sf::event::record(reinterpret_cast<CUstream_st*>(producer));
        auto fft = sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward);
        fft.execute(input.get(), output.get(), std::vector<sf::event>{first_half, second_half}).wait_and_throw();
        const auto actual = output.read();
        for (std::size_t i = 0; i < 8; ++i)
            check(std::abs(actual[i].real() - 1.0f) < 1e-5f && std::abs(actual[i].imag()) < 1e-5f,
                  "event-span dependency ordering failed");
        cudaStreamDestroy(producer);
    }
    {
        // B200 extension: split-precision tensor-core plans through the same plan API
        const std::size_t n = 256, batch = 16, count = n * batch;
        std::vector<std::complex<float>> source(count);
        for (std::size_t i = 0; i < count; ++i)
            source[i] = {static_cast<float>((i * 11 + 2) % 17) / 8.f, static_cast<float>((i * 3 + 1) % 13) / 7.f};
        const auto expected = reference_many(source, {n}, batch, sf::direction::forward);
        device_buffer<std::complex<float>> input(count), output(count);
        input.write(source);
        auto opts = make_plan_options(sf::placement::out_of_place, sf::normalization::none, sf::provider::b200);
        opts.split_precision = true;
        auto fft = sf::plan_many_dft<float>(sf::queue{}, {n}, batch, sf::direction::forward, opts);
        fft.execute(input.get(), output.get()).wait_and_throw();
        const auto actual = output.read();
        double num = 0, den = 0;
        for (std::size_t i = 0; i < count; ++i) {
            num += std::norm(std::complex<double>(actual[i]) - std::complex<double>(expected[i]));
            den += std::norm(std::complex<double>(expected[i]));
        }
        check(std::sqrt(num / den) < 2e-5, "split-precision plan mismatch");
    }
    {
        // B200 extension: real transforms (r2c against the direct DFT of the real lines, then
        // c2r with backward normalization back to the input)
        const std::size_t n = 64, batch = 3, h = n / 2 + 1;
        std::vector<float> real(n * batch);
        std::vector<std::complex<float>> as_complex(n * batch);
        for (std::size_t i = 0; i < n * batch; ++i) {
            real[i] = static_cast<float>((i * 7 + 3) % 11) / 5.f - 1.f;
            as_complex[i] = {real[i], 0.f};
        }
        const auto full = reference_many(as_complex, {n}, batch, sf::direction::forward);
        device_buffer<float> x(n * batch), back(n * batch);
        device_buffer<std::complex<float>> spec(h * batch);
        x.write(real);
        auto opts = make_plan_options(sf::placement::out_of_place, sf::normalization::backward);
        auto r2c = sf::plan_dft_r2c_1d<float>(sf::queue{}, n, batch, opts);
        auto c2r = sf::plan_dft_c2r_1d<float>(sf::queue{}, n, batch, opts);
        check(r2c.kind() == sf::real_kind::r2c && c2r.length() == n && c2r.batch_count() == batch, "real plan shape");
        auto done = r2c.execute(x.get(), spec.get());
        c2r.execute(spec.get(), back.get(), {done}).wait_and_throw();
        const auto s = spec.read();
        const auto y = back.read();
        double num = 0, den = 0, rnum = 0, rden = 0;
        for (std::size_t b = 0; b < batch; ++b)
            for (std::size_t k = 0; k < h; ++k) {
                num += std::norm(std::complex<double>(s[b * h + k]) - std::complex<double>(full[b * n + k]));
                den += std::norm(std::complex<double>(full[b * n + k]));
            }
        for (std::size_t i = 0; i < n * batch; ++i) {
            rnum += (double(y[i]) - real[i]) * (double(y[i]) - real[i]);
            rden += double(real[i]) * real[i];
        }
        check(std::sqrt(num / den) < 1e-5, "r2c plan mismatch");
        check(std::sqrt(rnum / rden) < 1e-5, "c2r round trip mismatch");
        expect_error(sf::error_code::invalid_argument, [&] { c2r.execute(x.get(), spec.get()); });
        // 2D: shape {6, 16}, 2 transforms; spectrum {6, 9} against the direct 2D DFT
        const std::size_t a = 6, m = 16, hm = m / 2 + 1, nb = 2;
        std::vector<double> real2(a * m * nb);
        std::vector<std::complex<double>> cplx2(a * m * nb);
        for (std::size_t i = 0; i < real2.size(); ++i) {
            real2[i] = static_cast<double>((i * 5 + 2) % 13) / 6.0 - 1.0;
            cplx2[i] = {real2[i], 0.0};
        }
        const auto full2 = reference_many(cplx2, {a, m}, nb, sf::direction::forward);
        device_buffer<double> x2(real2.size());
        device_buffer<std::complex<double>> s2(a * hm * nb);
        x2.write(real2);
        auto r2c2 = sf::plan_dft_r2c<double>(sf::queue{}, {a, m}, nb);
        check(r2c2.shape() == std::vector<std::size_t>{a, m} && r2c2.length() == m, "2D real plan shape");
        r2c2.execute(x2.get(), s2.get()).wait_and_throw();
        const auto got2 = s2.read();
        double n2 = 0, d2 = 0;
        for (std::size_t b = 0; b < nb; ++b)
            for (std::size_t i = 0; i < a; ++i)
                for (std::size_t k = 0; k < hm; ++k) {
                    const auto e = full2[(b * a + i) * m + k];
                    n2 += std::norm(got2[(b * a + i) * hm + k] - e);
                    d2 += std::norm(e);
                }
        check(std::sqrt(n2 / d2) < 1e-12, "2D r2c plan mismatch");
        expect_error(sf::error_code::invalid_argument, [] { (void)sf::plan_dft_r2c_1d<double>(sf::queue{}, 7); });
    }
    {
        // B200 extension: strided layouts -- 16-point transforms down the 6 columns of a 16 x 6
        // matrix written as contiguous rows, and 32-point transforms down 5 interleaved
        // columns in place
        const std::size_t n = 16, cols = 6;
        std::vector<std::complex<float>> matrix(n * cols), gathered(n * cols);
        for (std::size_t i = 0; i < n * cols; ++i)
            matrix[i] = {static_cast<float>((i * 5 + 1) % 9) / 4.f, static_cast<float>((i * 3 + 2) % 7) / 3.f};
        for (std::size_t c = 0; c < cols; ++c)
            for (std::size_t k = 0; k < n; ++k) gathered[c * n + k] = matrix[k * cols + c];
        const auto expected = reference_many(gathered, {n}, cols, sf::direction::forward);
        device_buffer<std::complex<float>> in(n * cols), out(n * cols);
        in.write(matrix);
        sf::data_layout lay{{static_cast<std::ptrdiff_t>(cols)}, 1, {1}, static_cast<std::ptrdiff_t>(n)};
        auto fft = sf::plan_many_dft<float>(sf::queue{}, {n}, cols, sf::direction::forward, make_plan_options(), lay);
        fft.execute(in.get(), out.get()).wait_and_throw();
        const auto got = out.read();
        double num = 0, den = 0;
        for (std::size_t i = 0; i < n * cols; ++i) {
            num += std::norm(std::complex<double>(got[i]) - std::complex<double>(expected[i]));
            den += std::norm(std::complex<double>(expected[i]));
        }
        check(std::sqrt(num / den) < 1e-5, "column layout mismatch");

        const std::size_t m = 32, b = 5;
        std::vector<std::complex<float>> inter(m * b), cols_in(m * b);
        for (std::size_t i = 0; i < m * b; ++i)
            inter[i] = {static_cast<float>((i * 13 + 4) % 17) / 8.f, static_cast<float>((i * 2 + 5) % 11) / 5.f};
        for (std::size_t c = 0; c < b; ++c)
            for (std::size_t k = 0; k < m; ++k) cols_in[c * m + k] = inter[k * b + c];
        const auto want = reference_many(cols_in, {m}, b, sf::direction::backward);
        device_buffer<std::complex<float>> io(m * b);
        io.write(inter);
        sf::data_layout il{{static_cast<std::ptrdiff_t>(b)}, 1, {static_cast<std::ptrdiff_t>(b)}, 1};
        auto ip = sf::plan_many_dft<float>(sf::queue{}, {m}, b, sf::direction::backward,
                                           make_plan_options(sf::placement::in_place), il);
        ip.execute(io.get()).wait_and_throw();
        const auto r = io.read();
        num = den = 0;
        for (std::size_t c = 0; c < b; ++c)
            for (std::size_t k = 0; k < m; ++k) {
                num += std::norm(std::complex<double>(r[k * b + c]) - std::complex<double>(want[c * m + k]));
                den += std::norm(std::complex<double>(want[c * m + k]));
            }
        check(std::sqrt(num / den) < 1e-5, "interleaved in-place layout mismatch");
        expect_error(sf::error_code::invalid_argument, [&] {
            sf::data_layout overlap{{1}, 1, {1}, 4};  // 8-point output rows 4 apart overlap
            (void)sf::plan_many_dft<float>(sf::queue{}, {8}, 3, sf::direction::forward, make_plan_options(), overlap);
        });
    }
    // sycl_tests.cpp:508-538
    expect_error(sf::error_code::provider_unavailable, [&] {
        (void)sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward,
                                     make_plan_options(sf::placement::out_of_place, sf::normalization::none,
                                                       sf::provider::cufft));
    });
    expect_error(sf::error_code::invalid_argument,
                 [&] { (void)sf::plan_dft_1d<float>(sf::queue{}, 8, static_cast<sf::direction>(0)); });
    expect_error(sf::error_code::invalid_pointer, [&] {
        auto fft = sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward);
        fft.execute(nullptr, nullptr);
    });
    expect_error(sf::error_code::invalid_argument, [&] {
        auto fft = sf::plan_dft_1d<float>(sf::queue{}, 8, sf::direction::forward,
                                          make_plan_options(sf::placement::in_place));
        device_buffer<std::complex<float>> a(8), b(8);
        fft.execute(a.get(), b.get());
    });
    expect_error(sf::error_code::invalid_state, [&] {
        auto original = sf::plan_dft_1d<float>(sf::queue{}, 4, sf::direction::forward);
        auto moved = std::move(original);
        (void)moved;
        original.execute(nullptr, nullptr);  // NOLINT(bugprone-use-after-move)
    });
    // host_tests.cpp:167-195: planning errors
    expect_error(sf::error_code::invalid_argument, [] { (void)sf::plan_dft_1d<float>(sf::queue{}, 0, sf::direction::forward); });
    expect_error(sf::error_code::invalid_argument, [] {
        (void)sf::plan_many_dft<float>(sf::queue{}, {static_cast<std::size_t>(-1), 2}, 1, sf::direction::forward);
    });
    expect_error(sf::error_code::invalid_argument,
                 [] { (void)sf::plan_many_dft<float>(sf::queue{}, {2, 2, 2, 2}, 1, sf::direction::forward); });
    {
        // Page-locked host buffers (host USM, which the reference's execute accepts,
        // sycl.cpp:72-85) stream through the device in chunks: same values as the device path.
        const std::size_t n = 4096, batch = 2100, count = n * batch;  // more than one 32 MiB chunk
        std::complex<float>*hin = nullptr, *hout = nullptr;
        check(cudaHostAlloc(reinterpret_cast<void**>(&hin), count * sizeof(std::complex<float>), 0) == cudaSuccess,
              "cudaHostAlloc");
        check(cudaHostAlloc(reinterpret_cast<void**>(&hout), count * sizeof(std::complex<float>), 0) == cudaSuccess,
              "cudaHostAlloc");
        std::vector<std::complex<float>> source(count);
        for (std::size_t i = 0; i < count; ++i)
            source[i] = {static_cast<float>((i * 5 + 1) % 9) / 4.f, static_cast<float>((i * 3 + 2) % 7) / 5.f};
        std::copy(source.begin(), source.end(), hin);
        device_buffer<std::complex<float>> din(count), dout(count);
        din.write(source);
        auto fft = sf::plan_many_dft<float>(sf::queue{}, {n}, batch, sf::direction::forward,
                                            make_plan_options(sf::placement::out_of_place, sf::normalization::forward));
        fft.execute(din.get(), dout.get()).wait_and_throw();
        fft.execute(hin, hout).wait_and_throw();
        const auto expected = dout.read();
        auto close = [&](const std::complex<float>* got) {
            for (std::size_t i = 0; i < count; ++i)
                if (std::abs(got[i] - expected[i]) > 1e-6f * (1.f + std::abs(expected[i]))) return false;
            return true;
        };
        check(close(hout), "host-buffer execute differs");
        auto inplace = sf::plan_many_dft<float>(sf::queue{}, {n}, batch, sf::direction::forward,
                                                make_plan_options(sf::placement::in_place, sf::normalization::forward));
        inplace.execute(hin).wait_and_throw();
        check(close(hin), "in-place host-buffer execute differs");
        cudaFreeHost(hin);
        cudaFreeHost(hout);
    }
    {
        // A bounded device wait that gives up surfaces as execution_failed on wait_and_throw
        // (the reference's code for a failed provider execution, sycl.cpp:671-676). The
        // 13440-point plan runs the copy-pipelined kernel; SYCLFFT_B200_WAIT_POLLS=0 makes its
        // copy waits give up at once (the copies still land before the blocks exit).
        const std::size_t n = 13440, batch = 16, count = n * batch;
        device_buffer<std::complex<float>> input(count), output(count);
        std::vector<std::complex<float>> source(count, {1.f, 0.f});
        input.write(source);
        setenv("SYCLFFT_B200_WAIT_POLLS", "0", 1);
        auto impatient = sf::plan_many_dft<float>(sf::queue{}, {n}, batch, sf::direction::forward);
        unsetenv("SYCLFFT_B200_WAIT_POLLS");
        auto failed = impatient.execute(input.get(), output.get());
        expect_error(sf::error_code::execution_failed, [&] { failed.wait_and_throw(); });
        failed.wait_and_throw();  // reported once
        auto healthy = sf::plan_many_dft<float>(sf::queue{}, {n}, batch, sf::direction::forward);
        healthy.execute(input.get(), output.get()).wait_and_throw();
        const auto actual = output.read();
        for (std::size_t b = 0; b < batch; ++b)
            check(std::abs(actual[b * n].real() - float(n)) < 1e-2f && std::abs(actual[b * n + 1]) < 1e-2f,
                  "transform after a reported timeout is wrong");
    }
    std::cout << "front-end tests passed\n";
    return 0;
} catch (const std::exception& ex) {
    std::cerr << "front-end tests failed: " << ex.what() << '\n';
    return 1;
}
