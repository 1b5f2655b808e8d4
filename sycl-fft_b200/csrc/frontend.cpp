// C++ front end of the syclfft B200 provider (include/syclfft_b200.hpp).
//
// Mirrors src/sycl/sycl.cpp's plan<Scalar>::impl for the device-provider path
// (sycl.cpp:424-491 construction and provider selection, 593-613 destruction, 615-686
// execute) and src/core/provider_loader.cpp (112-232: element-count validation,
// normalization scale, search paths, dlopen/dlsym, ABI check). Differences: there is no
// portable in-process provider to fall back to, so a missing or rejected B200 module is
// an error; and the normalization is passed to the module (fused into its last kernel)
// instead of a separate scaling pass.
#include "../../include/syclfft_b200.hpp"

#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <filesystem>
#include <limits>
#include <mutex>
#include <optional>
#include <sstream>

#include "../../include/syclfft_b200_provider.h"

namespace syclfft_b200 {

namespace detail {

std::size_t checked_element_count(const std::vector<std::size_t>& lengths, std::size_t batch_count) {
    if (lengths.empty() || lengths.size() > 3)
        throw exception(error_code::invalid_argument, "FFT rank must be between 1 and 3");
    if (batch_count == 0) throw exception(error_code::invalid_argument, "FFT batch count must be non-zero");
    std::size_t count = batch_count;
    for (const auto length : lengths) {
        if (length == 0) throw exception(error_code::invalid_argument, "FFT dimensions must be non-zero");
        if (count > std::numeric_limits<std::size_t>::max() / length)
            throw exception(error_code::invalid_argument, "FFT element count overflows size_t");
        count *= length;
    }
    return count;
}

double normalization_scale(normalization mode, direction dir, std::size_t transform_size) {
    switch (mode) {
        case normalization::none: return 1.0;
        case normalization::forward: return dir == direction::forward ? 1.0 / static_cast<double>(transform_size) : 1.0;
        case normalization::backward: return dir == direction::backward ? 1.0 / static_cast<double>(transform_size) : 1.0;
        case normalization::orthogonal: return 1.0 / std::sqrt(static_cast<double>(transform_size));
    }
    return 1.0;
}

const char* provider_name(provider value) noexcept {
    switch (value) {
        case provider::automatic: return "automatic";
        case provider::portable_sycl: return "portable_sycl";
        case provider::fftw: return "fftw";
        case provider::cufft: return "cufft";
        case provider::rocfft: return "rocfft";
        case provider::onemkl: return "onemkl";
        case provider::b200: return "b200";
    }
    return "unknown";
}

namespace {

std::filesystem::path library_directory() {
    Dl_info info{};
    if (dladdr(reinterpret_cast<void*>(&library_directory), &info) == 0 || !info.dli_fname) return {};
    return std::filesystem::path(info.dli_fname).parent_path();
}

void trace(const std::string& message) {
    // SYCLFFT_TRACE as in include/syclfft/detail/trace.hpp:8-18
    const char* enabled = std::getenv("SYCLFFT_TRACE");
    if (!enabled || enabled[0] == '\0' || enabled[0] == '0') return;
    std::fprintf(stderr, "[syclfft] %s\n", message.c_str());
}

}  // namespace

std::vector<std::string> provider_search_paths() {
    std::vector<std::string> result;
    if (const char* value = std::getenv("SYCLFFT_PLUGIN_PATH")) {
        std::stringstream stream(value);
        std::string item;
        while (std::getline(stream, item, ':'))
            if (!item.empty()) result.push_back(item);
    }
    const auto dir = library_directory();
    if (!dir.empty()) result.push_back((dir / "syclfft" / "providers").string());
    return result;
}

using syclfft_b200_create_ex_fn = void* (*)(const syclfft_b200_plan_config_v1*, uint32_t, char*, size_t);
using syclfft_b200_create_real_fn = void* (*)(const syclfft_b200_plan_config_v1*, int32_t, uint32_t, char*, size_t);
using syclfft_b200_create_strided_fn = void* (*)(const syclfft_b200_plan_config_v1*, const syclfft_b200_layout_v1*,
                                                 uint32_t, char*, size_t);
using syclfft_b200_take_status_fn = int (*)(void*);
using syclfft_b200_execute_host_fn = int (*)(const syclfft_b200_host_stage_v1*, uint32_t, const void*, void*, uint64_t,
                                             void*, char*, size_t);

struct loaded_provider {
    const syclfft_b200_provider_v1* api{};
    std::shared_ptr<void> module;
    syclfft_b200_create_ex_fn create_ex{};            // optional extensions: split precision,
    syclfft_b200_create_real_fn create_real{};        // real transforms,
    syclfft_b200_create_strided_fn create_strided{};  // strided layouts,
    syclfft_b200_take_status_fn take_status{};        // device-wait failures,
    syclfft_b200_execute_host_fn execute_host{};      // page-locked host buffers
};

// Owner of a provider plan: destroys it (keeping the module loaded until then) when the last
// front-end object referring to it -- the plan or one of its events -- is gone.
std::shared_ptr<void> own_plan(const loaded_provider& m, void* handle) {
    auto api = m.api;
    auto module = m.module;
    return std::shared_ptr<void>(handle, [api, module](void* h) {
        if (h) api->destroy(h);
    });
}

// Where a pointer lives: 1 = device (or managed), 2 = page-locked host memory.
int memory_kind(const void* pointer) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, pointer) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return attr.type == cudaMemoryTypeHost ? 2 : 1;
}

// provider_loader.cpp:178-232: first module in the search path that exports the entry
// point wins; a wrong ABI version is a plugin_error.
loaded_provider load_b200_provider() {
    std::string errors;
    for (const auto& directory : provider_search_paths()) {
        const auto path = std::filesystem::path(directory) / "syclfft_provider_b200.so";
        void* raw = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!raw) {
            const char* message = dlerror();
            errors += path.string() + ": " + (message ? message : "load failed") + "; ";
            continue;
        }
        auto module = std::shared_ptr<void>(raw, [](void* h) {
            if (h) dlclose(h);
        });
        void* symbol = dlsym(raw, "syclfft_b200_get_provider_v1");
        if (!symbol) {
            errors += path.string() + ": entry point 'syclfft_b200_get_provider_v1' missing; ";
            continue;
        }
        trace("core: provider symbol resolved");
        const auto* api = reinterpret_cast<syclfft_b200_get_provider_v1_fn>(symbol)();
        if (!api || api->abi_version != SYCLFFT_B200_PROVIDER_ABI_VERSION)
            throw exception(error_code::plugin_error, "Provider 'syclfft_provider_b200' has an incompatible ABI");
        auto create_ex = reinterpret_cast<syclfft_b200_create_ex_fn>(dlsym(raw, "syclfft_b200_create_ex"));
        auto create_real = reinterpret_cast<syclfft_b200_create_real_fn>(dlsym(raw, "syclfft_b200_create_real"));
        auto create_strided =
            reinterpret_cast<syclfft_b200_create_strided_fn>(dlsym(raw, "syclfft_b200_create_strided"));
        auto take_status = reinterpret_cast<syclfft_b200_take_status_fn>(dlsym(raw, "syclfft_b200_plan_take_status"));
        auto execute_host = reinterpret_cast<syclfft_b200_execute_host_fn>(dlsym(raw, "syclfft_b200_execute_host"));
        return {api, std::move(module), create_ex, create_real, create_strided, take_status, execute_host};
    }
    throw exception(error_code::provider_unavailable, "Unable to load provider 'syclfft_provider_b200': " + errors);
}

// sycl.cpp:72-85: non-null and an allocation the plan's device can access
void validate_device_pointer(const void* pointer, const char* name, int device) {
    if (!pointer) throw exception(error_code::invalid_pointer, std::string(name) + " must be non-null");
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, pointer);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw exception(error_code::invalid_pointer, std::string(name) + " is not a CUDA allocation");
    }
    if (attr.type == cudaMemoryTypeUnregistered)
        throw exception(error_code::invalid_pointer,
                        std::string(name) + " is not a device-accessible allocation in the plan context");
    if (attr.type == cudaMemoryTypeDevice && attr.device != device)
        throw exception(error_code::invalid_pointer, std::string(name) + " belongs to another device");
}

// data_layout rules: one stride per axis, strides >= 1, distances >= 1 for more than one
// transform, an output that never writes two elements to one address (sorted by stride, each
// stride exceeds the span of the smaller ones), equal layouts in place.
syclfft_b200_layout_v1 checked_layout(const data_layout& l, const std::vector<std::size_t>& lengths,
                                      std::size_t batch, bool in_place) {
    syclfft_b200_layout_v1 out{};
    for (int side = 0; side < 2; ++side) {
        const auto& strides = side ? l.out_strides : l.in_strides;
        const std::ptrdiff_t dist = side ? l.out_distance : l.in_distance;
        const std::string name = side ? "output" : "input";
        if (strides.size() != lengths.size())
            throw exception(error_code::invalid_argument, name + " layout needs one stride per axis");
        for (std::size_t k = 0; k < strides.size(); ++k) {
            if (strides[k] < 1) throw exception(error_code::invalid_argument, name + " strides must be >= 1");
            (side ? out.out_strides : out.in_strides)[k] = strides[k];
        }
        if (batch > 1 && dist < 1) throw exception(error_code::invalid_argument, name + " distance must be >= 1");
        (side ? out.out_distance : out.in_distance) = dist;
    }
    std::vector<std::pair<std::ptrdiff_t, std::size_t>> dims;
    for (std::size_t k = 0; k < lengths.size(); ++k)
        if (lengths[k] > 1) dims.push_back({l.out_strides[k], lengths[k]});
    if (batch > 1) dims.push_back({l.out_distance, batch});
    std::sort(dims.begin(), dims.end());
    long double reach = 0;
    for (const auto& d : dims) {
        if (static_cast<long double>(d.first) <= reach)
            throw exception(error_code::invalid_argument, "output layout overlaps itself");
        reach += static_cast<long double>(d.first) * static_cast<long double>(d.second - 1);
    }
    if (in_place) {
        bool same = batch <= 1 || l.in_distance == l.out_distance;
        for (std::size_t k = 0; k < lengths.size(); ++k)
            if (lengths[k] > 1 && l.in_strides[k] != l.out_strides[k]) same = false;
        if (!same) throw exception(error_code::invalid_argument, "an in-place plan needs equal input and output layouts");
    }
    return out;
}

}  // namespace detail

// ---------------------------------------------------------------- event
void event::wait_and_throw() const {
    if (!ev_) return;
    const cudaError_t e = cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(ev_.get()));
    if (e != cudaSuccess) throw exception(error_code::execution_failed, cudaGetErrorString(e));
    if (take_status_ && plan_) {
        const int code = take_status_(plan_);
        if (code > 0)
            throw exception(error_code::execution_failed, "a bounded wait in a B200 kernel gave up (status " +
                                                              std::to_string(code) +
                                                              "); the output of this execution is incomplete");
    }
}

event event::record(CUstream_st* stream, std::shared_ptr<void> owner, void* plan, int (*take_status)(void*)) {
    event out = record(stream);
    out.owner_ = std::move(owner);
    out.plan_ = plan;
    out.take_status_ = take_status;
    return out;
}

event event::record(CUstream_st* stream) {
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) throw exception(error_code::execution_failed, cudaGetErrorString(e));
    e = cudaEventRecord(ev, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaEventDestroy(ev);
        throw exception(error_code::execution_failed, cudaGetErrorString(e));
    }
    event out;
    out.ev_ = std::shared_ptr<CUevent_st>(reinterpret_cast<CUevent_st*>(ev),
                                          [](CUevent_st* p) { cudaEventDestroy(reinterpret_cast<cudaEvent_t>(p)); });
    return out;
}

// ---------------------------------------------------------------- plan
template <class Scalar>
class plan<Scalar>::impl {
public:
    impl(queue q, std::vector<std::size_t> lengths, std::size_t batch, syclfft_b200::direction dir,
         plan_options opts, const data_layout* layout = nullptr)
        : queue_(q),
          lengths_(std::move(lengths)),
          batch_count_(batch),
          element_count_(detail::checked_element_count(lengths_, batch_count_)),
          direction_(dir),
          options_(opts) {
        if (direction_ != syclfft_b200::direction::forward && direction_ != syclfft_b200::direction::backward)
            throw exception(error_code::invalid_argument, "Invalid FFT direction");
        // argument errors come before provider selection and device work, as the element count's
        std::optional<syclfft_b200_layout_v1> lay;
        if (layout)
            lay = detail::checked_layout(*layout, lengths_, batch_count_, options_.placement == placement::in_place);
        if (options_.preferred_provider != provider::automatic && options_.preferred_provider != provider::b200) {
            throw exception(error_code::provider_unavailable,
                            std::string(detail::provider_name(options_.preferred_provider)) +
                                " provider is not part of this build");
        }
        module_ = detail::load_b200_provider();
        if (queue_.device < 0) {
            const cudaError_t e = cudaGetDevice(&queue_.device);
            if (e != cudaSuccess) throw exception(error_code::provider_unavailable, cudaGetErrorString(e));
        }
        std::array<char, 1024> error{};
        if (!module_.api->supports(queue_.device, error.data(), error.size())) {
            throw exception(error_code::provider_unavailable,
                            error[0] ? error.data() : "B200 provider rejected the device");
        }
        syclfft_b200_plan_config_v1 config{};
        config.abi_version = SYCLFFT_B200_PROVIDER_ABI_VERSION;
        config.scalar = std::is_same_v<Scalar, double> ? SYCLFFT_B200_SCALAR_DOUBLE : SYCLFFT_B200_SCALAR_FLOAT;
        config.direction = static_cast<int32_t>(direction_);
        config.rank = static_cast<uint32_t>(lengths_.size());
        for (std::size_t i = 0; i < lengths_.size(); ++i) config.lengths[i] = lengths_[i];
        config.batch_count = batch_count_;
        config.in_place = options_.placement == placement::in_place ? 1 : 0;
        config.normalization = static_cast<uint32_t>(options_.normalization);
        config.measure = options_.planning == planning_mode::measure ? 1 : 0;
        config.device = queue_.device;
        strided_ = layout != nullptr;
        if (lay) {
            if (!module_.create_strided)
                throw exception(error_code::provider_unavailable, "B200 provider module lacks syclfft_b200_create_strided");
            uint32_t flags = SYCLFFT_B200_CREATE_SYNC;
            if (options_.split_precision && std::is_same_v<Scalar, float>) flags |= SYCLFFT_B200_CREATE_SPLIT_BF16;
            handle_ = module_.create_strided(&config, &*lay, flags, error.data(), error.size());
        } else if (options_.split_precision && std::is_same_v<Scalar, float>) {
            if (!module_.create_ex)
                throw exception(error_code::provider_unavailable, "B200 provider module lacks syclfft_b200_create_ex");
            handle_ = module_.create_ex(&config, SYCLFFT_B200_CREATE_SYNC | SYCLFFT_B200_CREATE_SPLIT_BF16,
                                        error.data(), error.size());
        } else {
            handle_ = module_.api->create(&config, error.data(), error.size());
        }
        if (!handle_) {
            throw exception(error_code::planning_failed, error[0] ? error.data() : "B200 plan creation failed");
        }
        owner_ = detail::own_plan(module_, handle_);
    }

    ~impl() {
        try {
            if (last_event_) last_event_->wait_and_throw();
        } catch (...) {
        }
    }

    void validate_pointer(const void* pointer, const char* name) const {
        detail::validate_device_pointer(pointer, name, queue_.device);
    }

    event execute(const complex_type* input, complex_type* output, const std::vector<event>& dependencies,
                  bool one_pointer) {
        validate_pointer(input, "input");
        validate_pointer(output, "output");
        if (options_.placement == placement::in_place && !one_pointer)
            throw exception(error_code::invalid_argument, "In-place plan must be executed with execute(inout)");
        if (options_.placement == placement::out_of_place && one_pointer)
            throw exception(error_code::invalid_argument, "Out-of-place plan requires input and output arguments");
        if (options_.placement == placement::out_of_place && static_cast<const void*>(input) == output)
            throw exception(error_code::invalid_argument, "Out-of-place plan requires distinct allocations");

        // sycl.cpp:637-641: one execution at a time per plan, ordered after the previous one.
        std::scoped_lock lock(mutex_);
        auto stream = reinterpret_cast<cudaStream_t>(queue_.stream);
        for (const auto& dep : dependencies) {
            if (dep.valid()) cudaStreamWaitEvent(stream, reinterpret_cast<cudaEvent_t>(dep.native()), 0);
        }
        if (last_event_ && last_event_->valid())
            cudaStreamWaitEvent(stream, reinterpret_cast<cudaEvent_t>(last_event_->native()), 0);
        std::array<char, 1024> error{};
        // page-locked host memory on both sides (host USM): streamed through the device in
        // overlapped chunks; otherwise the kernels address the buffers directly
        const bool host = !strided_ && detail::memory_kind(input) == 2 && detail::memory_kind(output) == 2;
        int rc = 0;
        if (host && module_.execute_host) {
            syclfft_b200_host_stage_v1 stage{handle_, 0, -1};
            rc = module_.execute_host(&stage, 1, input, output, 0, queue_.stream, error.data(), error.size());
        } else {
            rc = module_.api->execute(handle_, input, output, queue_.stream, error.data(), error.size());
        }
        if (rc != 0 || error[0])
            throw exception(error_code::execution_failed, error[0] ? error.data() : "B200 execution failed");
        event done = event::record(queue_.stream, owner_, handle_, module_.take_status);
        last_event_ = done;
        return done;
    }

    queue queue_;
    std::vector<std::size_t> lengths_;
    std::size_t batch_count_{};
    std::size_t element_count_{};
    syclfft_b200::direction direction_{syclfft_b200::direction::forward};
    plan_options options_{};
    detail::loaded_provider module_;
    void* handle_{};
    std::shared_ptr<void> owner_;  // destroys handle_ after the plan and its events are gone
    bool strided_ = false;
    std::optional<event> last_event_;
    std::mutex mutex_;
};

template <class Scalar>
plan<Scalar>::plan(queue q, std::vector<std::size_t> lengths, std::size_t batch_count, syclfft_b200::direction dir,
                   plan_options options)
    : impl_(std::make_unique<impl>(q, std::move(lengths), batch_count, dir, options)) {}

template <class Scalar>
plan<Scalar>::plan(queue q, std::vector<std::size_t> lengths, std::size_t batch_count, syclfft_b200::direction dir,
                   plan_options options, const data_layout& layout)
    : impl_(std::make_unique<impl>(q, std::move(lengths), batch_count, dir, options, &layout)) {}

template <class Scalar>
plan<Scalar>::plan(plan&&) noexcept = default;
template <class Scalar>
plan<Scalar>& plan<Scalar>::operator=(plan&&) noexcept = default;
template <class Scalar>
plan<Scalar>::~plan() = default;

#define SYCLFFT_B200_REQUIRE_IMPL()                                                          \
    if (!impl_) throw exception(error_code::invalid_state, "Cannot execute a moved-from plan")

template <class Scalar>
event plan<Scalar>::execute(complex_type* inout) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(inout, inout, {}, true);
}
template <class Scalar>
event plan<Scalar>::execute(complex_type* inout, const event& dependency) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(inout, inout, {dependency}, true);
}
template <class Scalar>
event plan<Scalar>::execute(complex_type* inout, const std::vector<event>& dependencies) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(inout, inout, dependencies, true);
}
template <class Scalar>
event plan<Scalar>::execute(const complex_type* input, complex_type* output) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(input, output, {}, false);
}
template <class Scalar>
event plan<Scalar>::execute(const complex_type* input, complex_type* output, const event& dependency) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(input, output, {dependency}, false);
}
template <class Scalar>
event plan<Scalar>::execute(const complex_type* input, complex_type* output, const std::vector<event>& dependencies) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(input, output, dependencies, false);
}

template <class Scalar>
std::vector<std::size_t> plan<Scalar>::shape() const {
    return impl_ ? impl_->lengths_ : std::vector<std::size_t>{};
}
template <class Scalar>
std::size_t plan<Scalar>::batch_count() const noexcept {
    return impl_ ? impl_->batch_count_ : 0;
}
template <class Scalar>
syclfft_b200::direction plan<Scalar>::direction() const noexcept {
    return impl_ ? impl_->direction_ : syclfft_b200::direction::forward;
}
template <class Scalar>
provider plan<Scalar>::selected_provider() const noexcept {
    return impl_ ? provider::b200 : provider::automatic;
}
template <class Scalar>
std::size_t plan<Scalar>::scratch_size_bytes() const noexcept {
    return impl_ ? static_cast<std::size_t>(impl_->module_.api->scratch_bytes(impl_->handle_)) : 0;
}

std::vector<provider_status> query_providers(const queue& q) {
    std::vector<provider_status> result;
    provider_status b200{provider::b200, "b200", true, false, {}};
    try {
        auto module = detail::load_b200_provider();
        int device = q.device;
        if (device < 0 && cudaGetDevice(&device) != cudaSuccess) throw std::runtime_error("no CUDA device");
        std::array<char, 1024> error{};
        b200.available = module.api->supports(device, error.data(), error.size()) != 0;
        if (!b200.available) b200.reason = error[0] ? error.data() : "device not supported";
    } catch (const std::exception& ex) {
        b200.reason = ex.what();
    }
    result.push_back(b200);
    result.push_back({provider::portable_sycl, "portable_sycl", false, false, "not part of this build"});
    result.push_back({provider::cufft, "cufft", false, false, "not part of this build"});
    result.push_back({provider::fftw, "fftw", false, false, "not part of this build"});
    result.push_back({provider::rocfft, "rocfft", false, false, "reserved for a future provider"});
    result.push_back({provider::onemkl, "onemkl", false, false, "reserved for a future provider"});
    return result;
}

template class plan<float>;
template class plan<double>;

// ---------------------------------------------------------------- real_plan
template <class Scalar>
class real_plan<Scalar>::impl {
public:
    impl(queue q, std::vector<std::size_t> lengths, std::size_t batch, real_kind kind, plan_options opts)
        : queue_(q), lengths_(std::move(lengths)), batch_count_(batch), kind_(kind), options_(opts) {
        (void)detail::checked_element_count(lengths_, batch_count_);
        n_ = lengths_.back();
        if (n_ % 2) throw exception(error_code::invalid_argument, "real transforms need an even last length");
        if (options_.placement != placement::out_of_place)
            throw exception(error_code::invalid_argument, "real transforms are out of place");
        if (kind_ != real_kind::r2c && kind_ != real_kind::c2r)
            throw exception(error_code::invalid_argument, "real transform kind must be r2c or c2r");
        if (options_.preferred_provider != provider::automatic && options_.preferred_provider != provider::b200) {
            throw exception(error_code::provider_unavailable,
                            std::string(detail::provider_name(options_.preferred_provider)) +
                                " provider is not part of this build");
        }
        module_ = detail::load_b200_provider();
        if (!module_.create_real)
            throw exception(error_code::provider_unavailable, "B200 provider module lacks syclfft_b200_create_real");
        if (queue_.device < 0) {
            const cudaError_t e = cudaGetDevice(&queue_.device);
            if (e != cudaSuccess) throw exception(error_code::provider_unavailable, cudaGetErrorString(e));
        }
        std::array<char, 1024> error{};
        if (!module_.api->supports(queue_.device, error.data(), error.size())) {
            throw exception(error_code::provider_unavailable,
                            error[0] ? error.data() : "B200 provider rejected the device");
        }
        syclfft_b200_plan_config_v1 config{};
        config.abi_version = SYCLFFT_B200_PROVIDER_ABI_VERSION;
        config.scalar = std::is_same_v<Scalar, double> ? SYCLFFT_B200_SCALAR_DOUBLE : SYCLFFT_B200_SCALAR_FLOAT;
        config.direction = kind_ == real_kind::r2c ? -1 : 1;
        config.rank = static_cast<uint32_t>(lengths_.size());
        for (std::size_t i = 0; i < lengths_.size(); ++i) config.lengths[i] = lengths_[i];
        config.batch_count = batch_count_;
        config.in_place = 0;
        config.normalization = static_cast<uint32_t>(options_.normalization);
        config.measure = options_.planning == planning_mode::measure ? 1 : 0;
        config.device = queue_.device;
        uint32_t flags = SYCLFFT_B200_CREATE_SYNC;
        if (options_.split_precision && std::is_same_v<Scalar, float>) flags |= SYCLFFT_B200_CREATE_SPLIT_BF16;
        handle_ = module_.create_real(&config, kind_ == real_kind::r2c ? SYCLFFT_B200_REAL_R2C : SYCLFFT_B200_REAL_C2R,
                                      flags, error.data(), error.size());
        if (!handle_)
            throw exception(error_code::planning_failed, error[0] ? error.data() : "B200 plan creation failed");
        owner_ = detail::own_plan(module_, handle_);
    }

    ~impl() {
        try {
            if (last_event_) last_event_->wait_and_throw();
        } catch (...) {
        }
    }

    event execute(const void* input, void* output, const std::vector<event>& dependencies, real_kind called) {
        if (called != kind_)
            throw exception(error_code::invalid_argument, kind_ == real_kind::r2c
                                                              ? "an r2c plan takes real input and complex output"
                                                              : "a c2r plan takes complex input and real output");
        detail::validate_device_pointer(input, "input", queue_.device);
        detail::validate_device_pointer(output, "output", queue_.device);
        if (input == output) throw exception(error_code::invalid_argument, "Out-of-place plan requires distinct allocations");
        std::scoped_lock lock(mutex_);
        auto stream = reinterpret_cast<cudaStream_t>(queue_.stream);
        for (const auto& dep : dependencies) {
            if (dep.valid()) cudaStreamWaitEvent(stream, reinterpret_cast<cudaEvent_t>(dep.native()), 0);
        }
        if (last_event_ && last_event_->valid())
            cudaStreamWaitEvent(stream, reinterpret_cast<cudaEvent_t>(last_event_->native()), 0);
        std::array<char, 1024> error{};
        const int rc = module_.api->execute(handle_, input, output, queue_.stream, error.data(), error.size());
        if (rc != 0 || error[0])
            throw exception(error_code::execution_failed, error[0] ? error.data() : "B200 execution failed");
        event done = event::record(queue_.stream, owner_, handle_, module_.take_status);
        last_event_ = done;
        return done;
    }

    queue queue_;
    std::vector<std::size_t> lengths_;
    std::size_t n_{};
    std::size_t batch_count_{};
    real_kind kind_{real_kind::r2c};
    plan_options options_{};
    detail::loaded_provider module_;
    void* handle_{};
    std::shared_ptr<void> owner_;  // destroys handle_ after the plan and its events are gone
    std::optional<event> last_event_;
    std::mutex mutex_;
};

template <class Scalar>
real_plan<Scalar>::real_plan(queue q, std::size_t n, std::size_t batch_count, real_kind kind, plan_options options)
    : impl_(std::make_unique<impl>(q, std::vector<std::size_t>{n}, batch_count, kind, options)) {}
template <class Scalar>
real_plan<Scalar>::real_plan(queue q, std::vector<std::size_t> lengths, std::size_t batch_count, real_kind kind,
                             plan_options options)
    : impl_(std::make_unique<impl>(q, std::move(lengths), batch_count, kind, options)) {}
template <class Scalar>
real_plan<Scalar>::real_plan(real_plan&&) noexcept = default;
template <class Scalar>
real_plan<Scalar>& real_plan<Scalar>::operator=(real_plan&&) noexcept = default;
template <class Scalar>
real_plan<Scalar>::~real_plan() = default;

template <class Scalar>
event real_plan<Scalar>::execute(const Scalar* input, complex_type* output, const std::vector<event>& dependencies) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(input, output, dependencies, real_kind::r2c);
}
template <class Scalar>
event real_plan<Scalar>::execute(const complex_type* input, Scalar* output, const std::vector<event>& dependencies) {
    SYCLFFT_B200_REQUIRE_IMPL();
    return impl_->execute(input, output, dependencies, real_kind::c2r);
}
template <class Scalar>
std::size_t real_plan<Scalar>::length() const noexcept {
    return impl_ ? impl_->n_ : 0;
}
template <class Scalar>
std::vector<std::size_t> real_plan<Scalar>::shape() const {
    return impl_ ? impl_->lengths_ : std::vector<std::size_t>{};
}
template <class Scalar>
std::size_t real_plan<Scalar>::batch_count() const noexcept {
    return impl_ ? impl_->batch_count_ : 0;
}
template <class Scalar>
real_kind real_plan<Scalar>::kind() const noexcept {
    return impl_ ? impl_->kind_ : real_kind::r2c;
}

template class real_plan<float>;
template class real_plan<double>;

}  // namespace syclfft_b200
