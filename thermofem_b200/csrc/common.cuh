// common.cuh -- shared host/device plumbing of the B200 sparse solve path:
// error model of the C ABI, device scope guard, RAII device buffers, the
// execution context and launch helpers.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>

#include "thermofem_b200.h"

namespace tfb {

// Internal failure carrying a C ABI status code.  Thrown inside the library
// and converted to a status at every extern "C" boundary.
struct Failure : std::exception {
    int code;
    std::string message;
    int cuda{0};  // the cudaError_t behind a TF_ERR_CUDA / TF_ERR_NOMEM, 0 otherwise
    Failure(int c, std::string m, int cu = 0) : code(c), message(std::move(m)), cuda(cu) {}
    const char *what() const noexcept override { return message.c_str(); }
};

[[noreturn]] inline void fail(int code, const std::string &msg) { throw Failure(code, msg); }
inline void require(bool ok, const char *msg, int code = TF_ERR_INVALID) {
    if (!ok) fail(code, msg);
}
inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        const std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
        throw Failure(e == cudaErrorMemoryAllocation ? TF_ERR_NOMEM : TF_ERR_CUDA, msg, static_cast<int>(e));
    }
}

// Records the message (and CUDA error code, 0 for none) of a failing call on
// this thread: tf_last_error / tf_last_cuda_error.
void set_last_error(const char *msg, int cuda = 0);

// Runs f and converts exceptions to a status (the ABI never throws).
template <class F>
int guard(F &&f) noexcept {
    try {
        f();
        return TF_OK;
    } catch (const Failure &e) {
        set_last_error(e.message.c_str(), e.cuda);
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return TF_ERR_NOMEM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return TF_ERR_RUNTIME;
    } catch (...) {
        set_last_error("unknown failure");
        return TF_ERR_RUNTIME;
    }
}

// Selects a device for the lifetime of the scope and restores the caller's.
class DeviceScope {
  public:
    explicit DeviceScope(int device) {
        cuda_check(cudaGetDevice(&previous_), "cudaGetDevice");
        if (device != previous_) cuda_check(cudaSetDevice(device), "cudaSetDevice");
    }
    ~DeviceScope() {
        int now = -1;
        if (cudaGetDevice(&now) == cudaSuccess && now != previous_) cudaSetDevice(previous_);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;

  private:
    int previous_{0};
};

// Owning device allocation (cudaMalloc / cudaFree).  Allocation happens in
// setup and workspace growth only; the solve loop never allocates.
template <class T>
class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { allocate(n); }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept { swap(o); }
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
        if (this != &o) {
            DeviceBuffer t(std::move(o));
            swap(t);
        }
        return *this;
    }
    void swap(DeviceBuffer &o) noexcept {
        std::swap(ptr_, o.ptr_);
        std::swap(size_, o.size_);
        std::swap(device_, o.device_);
    }
    void allocate(size_t n) {
        release();
        if (n) {
            cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
            cuda_check(cudaMalloc(&ptr_, n * sizeof(T)), "cudaMalloc");
        }
        size_ = n;
    }
    // Grows to at least n elements (contents not preserved).
    void reserve(size_t n) {
        if (n > size_) allocate(n);
    }
    void release() noexcept {
        if (ptr_) {
            int now = -1;
            cudaGetDevice(&now);
            if (now != device_) cudaSetDevice(device_);
            cudaFree(ptr_);
            if (now != device_) cudaSetDevice(now);
        }
        ptr_ = nullptr;
        size_ = 0;
    }
    T *data() const noexcept { return static_cast<T *>(ptr_); }
    size_t size() const noexcept { return size_; }
    bool empty() const noexcept { return size_ == 0; }

  private:
    void *ptr_{nullptr};
    size_t size_{0};
    int device_{-1};
};

}  // namespace tfb

// Execution context: one device, one stream, a scratch arena and a pinned
// host staging word for scalar readbacks.
struct tf_ctx {
    int device{0};
    cudaStream_t stream{nullptr};
    bool own_stream{false};
    int sm_count{148};
    int64_t launches{0};
    tfb::DeviceBuffer<unsigned char> scratch;  // grow-only, reused by primitives
    tfb::DeviceBuffer<unsigned char> scratch2;
    void *pinned{nullptr};                      // 256 bytes of pinned host memory
    int *fault{nullptr};                        // device word raised by a kernel whose bounded wait expired
    bool pdl{true};                             // launch_kernel adds programmatic dependent launch
    bool stable{false};                         // operators are read-only (solve / cycle enqueue)
    bool checked{false};                        // caller CSR validated before kernel-layer launches
    tf_ctx() = default;
    tf_ctx(const tf_ctx &) = delete;
    tf_ctx &operator=(const tf_ctx &) = delete;
    // Releases what tf_ctx_create acquired, also when it failed part way
    // (the caller makes the context's device current).
    ~tf_ctx() {
        if (stream) cudaStreamSynchronize(stream);
        scratch.release();
        scratch2.release();
        if (pinned) cudaFreeHost(pinned);
        if (fault) cudaFree(fault);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
    // Returns a scratch region of at least bytes (256-byte aligned start).
    void *arena(size_t bytes, int slot = 0) {
        auto &b = slot ? scratch2 : scratch;
        b.reserve(bytes + 256);
        return b.data();
    }
};

namespace tfb {

constexpr int kBlock = 256;

inline unsigned grid_for(int64_t n, int block = kBlock) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 0x7fffffff) g = 0x7fffffff;
    return static_cast<unsigned>(g);
}

// Checks the launch and counts it on the context.
inline void launched(tf_ctx *ctx, const char *name) {
    ++ctx->launches;
    cuda_check(cudaGetLastError(), name);
}

// Programmatic dependent launch.  A kernel started by launch_kernel may be
// scheduled while the kernel before it in the stream is still running:
// pdl_wait() returns once that kernel has completed and its writes are
// visible, so such a kernel calls it before any access to memory an earlier
// kernel writes or reads; pdl_trigger() lets the next kernel be scheduled
// (its CTAs then wait in their own pdl_wait).  Both are no-ops in a kernel
// launched without the attribute.
//
// The next kernel is scheduled once every CTA of this one has triggered or
// exited.  Kernels here do not trigger at entry: a next kernel scheduled
// while this one still runs takes SM slots, registers and shared memory
// (and with it L1) that this one needs.  Measured on B200 (PCG + AMG, FP32
// hierarchy), triggers at entry everywhere made the 256^3 solve 12 % slower
// than triggers after the work; entry triggers in the small kernels only
// gained 1 ms at 128^3 and lost 1.5 % at 256^3.  So a kernel enters with
// pdl_enter() (the wait alone) and triggers by exiting -- or, for the
// persistent row-tile SpMV kernels (tile.cuh), by pdl_trigger() after the
// main loop, so that the next kernel's launch and prologue overlap their
// tail (draining copies, a last-CTA scalar step).  The small-level region
// (coarse_cycle.cu), one CTA or cluster, triggers once it has loaded.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() { pdl_wait(); }

// Launches kernel<<<grid, block, smem, ctx->stream>>>(args...) with the
// programmatic-serialization attribute (when ctx->pdl) and counts it.  Every
// kernel launched here calls pdl_wait() (pdl_enter()) before touching memory
// that another kernel of the stream uses.
template <class... P, class... A>
void launch_kernel(tf_ctx *ctx, const char *name, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                   A &&...args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cfg.attrs = attr;
    cfg.numAttrs = ctx->pdl ? 1 : 0;
    cuda_check(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...), name);
    ++ctx->launches;
}

// Marks the context's operators read-only while a solve or cycle is
// enqueued: pipelined kernels may then stream the matrix before their
// predecessor has finished.
struct StableScope {
    tf_ctx *ctx;
    bool old;
    explicit StableScope(tf_ctx *c) : ctx(c), old(c->stable) { c->stable = true; }
    ~StableScope() { ctx->stable = old; }
};

// Synchronises the context stream and reads a device scalar.
template <class T>
T read_scalar(tf_ctx *ctx, const T *device_ptr) {
    static_assert(sizeof(T) <= 256, "scalar too large");
    cuda_check(cudaMemcpyAsync(ctx->pinned, device_ptr, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream),
               "scalar readback");
    cuda_check(cudaStreamSynchronize(ctx->stream), "scalar readback sync");
    T v;
    std::memcpy(&v, ctx->pinned, sizeof(T));
    return v;
}

inline void memset_async(tf_ctx *ctx, void *p, int value, size_t bytes) {
    if (bytes) cuda_check(cudaMemsetAsync(p, value, bytes, ctx->stream), "cudaMemsetAsync");
}

// Reads and clears the context's fault word; a raised word means a kernel
// gave up a bounded wait (its results are not valid).
inline void check_faults(tf_ctx *ctx) {
    if (!ctx->fault) return;
    if (read_scalar(ctx, ctx->fault)) {
        memset_async(ctx, ctx->fault, 0, sizeof(int));
        cudaStreamSynchronize(ctx->stream);
        fail(TF_ERR_TIMEOUT, "a pipelined kernel gave up a bounded wait; results are invalid");
    }
}

// Ends a capture left open on the context stream by a failed step of a
// capture INTO AN EXISTING GRAPH (cudaStreamBeginCaptureToGraph).  The graph
// that cudaStreamEndCapture hands back is then that existing graph, or a body
// graph owned by one of its nodes, so it is not destroyed here: the caller
// destroys its own graph once.  (A capture may also end this way when another
// thread synchronises the whole device while it is open, which invalidates
// it.)
inline void end_capture_into_graph(tf_ctx *ctx) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
        cudaGraph_t returned = nullptr;
        cudaStreamEndCapture(ctx->stream, &returned);
    }
    cudaGetLastError();
}

inline void copy_async(tf_ctx *ctx, void *dst, const void *src, size_t bytes) {
    if (bytes && dst != src) cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream), "cudaMemcpyAsync");
}

inline size_t type_size(int t) {
    switch (t) {
        case TF_F32: return 4;
        case TF_F64: return 8;
        case TF_I32: return 4;
        case TF_I64: return 8;
    }
    fail(TF_ERR_INVALID, "unknown element type");
}

inline void check_ctx(tf_ctx *ctx) { require(ctx != nullptr, "null context"); }

inline void check_csr(const tf_csr *a) {
    require(a != nullptr, "null CSR descriptor");
    require(a->rows >= 0 && a->cols >= 0 && a->nnz >= 0, "negative CSR dimension");
    require(a->index_type == TF_I32 || a->index_type == TF_I64, "CSR index type must be TF_I32 or TF_I64");
    require(a->value_type == TF_F32 || a->value_type == TF_F64, "CSR value type must be TF_F32 or TF_F64");
    require(a->offsets != nullptr || a->rows == 0, "null CSR offsets");
    require((a->indices != nullptr && a->values != nullptr) || a->nnz == 0, "null CSR entries");
    if (a->index_type == TF_I32) require(a->nnz <= INT32_MAX && a->rows < INT32_MAX, "CSR exceeds int32 indices", TF_ERR_LENGTH);
}

}  // namespace tfb

// Owned device CSR returned by setup stages.
struct tf_dcsr {
    int64_t rows{0}, cols{0}, nnz{0};
    int index_type{TF_I32}, value_type{TF_F64};
    tfb::DeviceBuffer<unsigned char> offsets, indices, values;
    tf_csr view() const {
        tf_csr v;
        v.rows = rows;
        v.cols = cols;
        v.nnz = nnz;
        v.index_type = index_type;
        v.value_type = value_type;
        v.offsets = offsets.data();
        v.indices = indices.data();
        v.values = values.data();
        return v;
    }
};

struct tf_transfer {
    int fine_rows{0}, coarse_rows{0};
    int32_t histogram[4]{0, 0, 0, 0};
    tfb::DeviceBuffer<int32_t> map, offsets, members;
};
