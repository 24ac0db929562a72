// b200.cuh -- how the C++ component layer reaches the library's C ABI
// (thermofem_b200.h): status codes become the exceptions the reference's
// components throw, and every component runs on a tf_ctx of its own.
//
// Ordering and synchrony: a tf_ctx has its own non-blocking stream (whole
// solves are captured into CUDA graphs there, which the legacy default
// stream does not allow).  The reference's components work on the default
// stream and return when their work is done; to keep exactly that contract
// each component call first makes its stream wait for the work already queued
// on the calling thread's legacy default stream, and returns after its own
// stream has drained.
#pragma once

#include <thermofem_b200.h>

#include <DataStructure/Memory.cuh>

#include <concepts>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>

namespace thermofem::b200 {

/// Throws the exception the reference raises for a failed C ABI status:
/// invalid_argument, logic_error, length_error, CudaError (with the CUDA
/// error code) or runtime_error.
inline void check(int status) {
    if (status == TF_OK) return;
    const char *last = tf_last_error();
    std::string message = last && *last ? last : tf_status_string(status);
    switch (status) {
        case TF_ERR_INVALID: throw std::invalid_argument(message);
        case TF_ERR_LOGIC: throw std::logic_error(message);
        case TF_ERR_LENGTH: throw std::length_error(message);
        case TF_ERR_CUDA:
        case TF_ERR_NOMEM: {
            int code = tf_last_cuda_error();
            if (!code) code = status == TF_ERR_NOMEM ? cudaErrorMemoryAllocation : cudaErrorUnknown;
            // the library's message is "<operation>: <CUDA message>"; CudaError adds the latter itself
            const std::string suffix = std::string(": ") + cudaGetErrorString(static_cast<cudaError_t>(code));
            if (message.size() > suffix.size() && message.compare(message.size() - suffix.size(), suffix.size(),
                                                                   suffix) == 0)
                message.resize(message.size() - suffix.size());
            throw CudaError(static_cast<cudaError_t>(code), message.c_str());
        }
        default: throw std::runtime_error(message);
    }
}

template <class T>
constexpr int valueType() {
    static_assert(std::same_as<T, float> || std::same_as<T, double>);
    return std::same_as<T, double> ? TF_F64 : TF_F32;
}
template <class I>
constexpr int indexType() {
    static_assert(sizeof(I) == 4 || sizeof(I) == 8);
    return sizeof(I) == 8 ? TF_I64 : TF_I32;
}

inline int currentDevice() {
    int device = 0;
    detail::cudaCall(cudaGetDevice(&device), "cudaGetDevice");
    return device;
}

/// A tf_ctx (stream, scratch arena) on one device, owned.
class Context {
  public:
    explicit Context(int device) : device_(device < 0 ? currentDevice() : device) {
        detail::DeviceSwitch on(device_);
        tf_ctx *h = nullptr;
        check(tf_ctx_create(device_, nullptr, &h));
        handle_.reset(h);
        cudaEvent_t e = nullptr;
        detail::cudaCall(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreateWithFlags");
        event_ = e;
    }
    ~Context() {
        if (event_) (void)cudaEventDestroy(event_);
    }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;

    [[nodiscard]] tf_ctx *get() const noexcept { return handle_.get(); }
    [[nodiscard]] int device() const noexcept { return device_; }
    [[nodiscard]] cudaStream_t stream() const noexcept { return static_cast<cudaStream_t>(tf_ctx_stream(get())); }

    /// The context stream waits for what the calling thread queued on the
    /// legacy default stream (where the reference's components run).
    void followDefaultStream() {
        detail::DeviceSwitch on(device_);
        detail::cudaCall(cudaEventRecord(event_, cudaStreamLegacy), "cudaEventRecord");
        detail::cudaCall(cudaStreamWaitEvent(stream(), event_, 0), "cudaStreamWaitEvent");
    }
    void synchronize() { check(tf_ctx_synchronize(get())); }

  private:
    struct Release {
        void operator()(tf_ctx *c) const noexcept { tf_ctx_destroy(c); }
    };
    int device_;
    std::unique_ptr<tf_ctx, Release> handle_;
    cudaEvent_t event_{nullptr};
};

/// One context per device and thread for the free functions of the
/// operation API (transfers, coarse factor, conversions).
inline Context &ambient(int device) {
    thread_local std::unordered_map<int, std::unique_ptr<Context>> contexts;
    auto &slot = contexts[device];
    if (!slot) slot = std::make_unique<Context>(device);
    return *slot;
}

/// Runs f on the context's device, ordered after the default stream, and
/// waits for the context's stream before returning.
template <class F>
decltype(auto) onContext(Context &ctx, F &&f) {
    detail::DeviceSwitch on(ctx.device());
    ctx.followDefaultStream();
    if constexpr (std::is_void_v<decltype(f())>) {
        f();
        ctx.synchronize();
    } else {
        auto result = f();
        ctx.synchronize();
        return result;
    }
}

}  // namespace thermofem::b200
