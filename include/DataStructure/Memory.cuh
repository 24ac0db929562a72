// Memory.cuh -- memory strategies, the CUDA error type and the byte storage
// of the thermofem_b200 C++ component layer.
//
// Drop-in for the reference header of the same path
// (include/DataStructure/Memory.cuh:1-179 of Mgepahmge/ThermoFEM): the same
// names, strategies, value semantics and exceptions, so code written against
// the reference compiles unchanged.  Header-only: the storage talks to the
// CUDA runtime directly (allocation, synchronous copies), as the reference's
// storage does; the compute path lives behind the library's C ABI.
//
// Semantics kept from the reference: a non-empty storage belongs to the
// device that was current when it was allocated; copies keep the source's
// strategy; moves leave the source empty; copyDataFrom keeps the target's
// address and strategy and needs equal sizes on one device; changeMemoryType
// keeps the contents and may move them; host copies are synchronous;
// destruction never throws.
#pragma once

#include <cuda_runtime_api.h>

#include <concepts>
#include <cstddef>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>

namespace thermofem {

/// Where a buffer lives: device memory, page-locked host memory, page-locked
/// host memory mapped into the device's address space, or managed memory.
enum class MemoryType { Global, Pinned, Mapped, Managed };

struct GlobalMemory {};   ///< cudaMalloc
struct PinnedMemory {};   ///< cudaMallocHost
struct MappedMemory {};   ///< cudaHostAlloc(cudaHostAllocMapped)
struct ManagedMemory {};  ///< cudaMallocManaged

template <class T>
concept MemoryPolicy = std::same_as<T, GlobalMemory> || std::same_as<T, PinnedMemory> ||
                       std::same_as<T, MappedMemory> || std::same_as<T, ManagedMemory>;

/// The strategy chosen at run time; its index is the MemoryType.
using MemoryStrategy = std::variant<GlobalMemory, PinnedMemory, MappedMemory, ManagedMemory>;

/// A failed CUDA runtime call: what() names the operation and the CUDA
/// message, code() is the cudaError_t.
class CudaError : public std::runtime_error {
  public:
    CudaError(cudaError_t code, const char *operation)
        : std::runtime_error(std::string(operation ? operation : "CUDA") + ": " + cudaGetErrorString(code)),
          code_(code) {}
    [[nodiscard]] cudaError_t code() const noexcept { return code_; }

  private:
    cudaError_t code_;
};

namespace detail {

inline void cudaCall(cudaError_t status, const char *operation) {
    if (status != cudaSuccess) throw CudaError(status, operation);
}

/// left * right, or std::length_error when it does not fit in size_t.
[[nodiscard]] inline std::size_t checkedProduct(std::size_t left, std::size_t right) {
    if (right && left > std::numeric_limits<std::size_t>::max() / right)
        throw std::length_error("Data structure size overflows size_t");
    return left * right;
}

/// Makes `device` current for the scope (no change for -1) and puts the
/// caller's device back at the end.
class DeviceSwitch {
  public:
    explicit DeviceSwitch(int device) {
        if (device < 0) return;
        cudaCall(cudaGetDevice(&saved_), "cudaGetDevice");
        if (saved_ != device) cudaCall(cudaSetDevice(device), "cudaSetDevice");
        else saved_ = -1;
    }
    ~DeviceSwitch() {
        if (saved_ >= 0) (void)cudaSetDevice(saved_);
    }
    DeviceSwitch(const DeviceSwitch &) = delete;
    DeviceSwitch &operator=(const DeviceSwitch &) = delete;

  private:
    int saved_{-1};
};

/// How each strategy allocates, frees and is reached from host and device.
struct StrategyOps {
    void *(*allocate)(std::size_t bytes);
    void (*release)(void *pointer) noexcept;
    bool hostAccessible;  // plain host loads and stores work
};

inline void *allocGlobal(std::size_t bytes) {
    void *p = nullptr;
    cudaCall(cudaMalloc(&p, bytes), "cudaMalloc");
    return p;
}
inline void *allocPinned(std::size_t bytes) {
    void *p = nullptr;
    cudaCall(cudaMallocHost(&p, bytes), "cudaMallocHost");
    return p;
}
inline void *allocMapped(std::size_t bytes) {
    int device = 0, canMap = 0;
    cudaCall(cudaGetDevice(&device), "cudaGetDevice");
    cudaCall(cudaDeviceGetAttribute(&canMap, cudaDevAttrCanMapHostMemory, device), "cudaDeviceGetAttribute");
    if (!canMap) throw std::runtime_error("CUDA device cannot map host memory");
    void *p = nullptr;
    cudaCall(cudaHostAlloc(&p, bytes, cudaHostAllocMapped), "cudaHostAlloc");
    return p;
}
inline void *allocManaged(std::size_t bytes) {
    void *p = nullptr;
    cudaCall(cudaMallocManaged(&p, bytes), "cudaMallocManaged");
    return p;
}
inline void freeDevice(void *p) noexcept { (void)cudaFree(p); }
inline void freeHost(void *p) noexcept { (void)cudaFreeHost(p); }

inline const StrategyOps &strategyOps(MemoryType type) {
    static const StrategyOps table[4] = {
        {allocGlobal, freeDevice, false},
        {allocPinned, freeHost, true},
        {allocMapped, freeHost, true},
        {allocManaged, freeDevice, true},
    };
    return table[static_cast<int>(type)];
}

/// Bytes owned under one strategy on one device.
class MemoryStorage {
  public:
    explicit MemoryStorage(MemoryStrategy strategy = GlobalMemory{}) noexcept : strategy_(strategy) {}
    MemoryStorage(std::size_t bytes, MemoryStrategy strategy) : strategy_(strategy) {
        if (!bytes) return;
        int device = 0;
        cudaCall(cudaGetDevice(&device), "cudaGetDevice");
        data_ = strategyOps(memoryType()).allocate(bytes);
        bytes_ = bytes;
        device_ = device;
    }
    MemoryStorage(const MemoryStorage &other) : strategy_(other.strategy_) {
        if (!other.bytes_) return;
        DeviceSwitch on(other.device_);
        MemoryStorage copy(other.bytes_, other.strategy_);
        copy.copyDataFrom(other);
        swap(copy);
    }
    MemoryStorage(MemoryStorage &&other) noexcept : strategy_(other.strategy_) { swap(other); }
    MemoryStorage &operator=(const MemoryStorage &other) {
        if (this != &other) {
            MemoryStorage copy(other);
            swap(copy);
        }
        return *this;
    }
    MemoryStorage &operator=(MemoryStorage &&other) noexcept {
        if (this != &other) {
            MemoryStorage taken(std::move(other));
            swap(taken);
        }
        return *this;
    }
    ~MemoryStorage() noexcept { release(); }

    void swap(MemoryStorage &other) noexcept {
        std::swap(data_, other.data_);
        std::swap(bytes_, other.bytes_);
        std::swap(device_, other.device_);
        std::swap(strategy_, other.strategy_);
    }

    void copyDataFrom(const MemoryStorage &other) {
        if (bytes_ != other.bytes_) throw std::invalid_argument("Buffer sizes must match");
        if (!bytes_ || this == &other) return;
        if (device_ != other.device_) throw std::invalid_argument("Cross-device copies are not supported");
        DeviceSwitch on(device_);
        if (hostReachable() && other.hostReachable()) std::memmove(data_, other.data_, bytes_);
        else cudaCall(cudaMemcpy(data_, other.data_, bytes_, cudaMemcpyDefault), "cudaMemcpy");
    }

    void changeMemoryType(MemoryStrategy strategy) {
        if (strategy.index() == strategy_.index()) return;
        if (!bytes_) {
            strategy_ = strategy;
            return;
        }
        DeviceSwitch on(device_);
        MemoryStorage moved(bytes_, strategy);
        moved.copyDataFrom(*this);
        swap(moved);
    }

    void copyFromHost(const void *source, std::size_t bytes) {
        if (bytes != bytes_ || (bytes && !source)) throw std::invalid_argument("Invalid host source or size");
        if (!bytes) return;
        DeviceSwitch on(device_);
        if (hostReachable()) std::memmove(data_, source, bytes);
        else cudaCall(cudaMemcpy(data_, source, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
    }

    void copyToHost(void *target, std::size_t bytes) const {
        if (bytes != bytes_ || (bytes && !target)) throw std::invalid_argument("Invalid host target or size");
        if (!bytes) return;
        DeviceSwitch on(device_);
        if (hostReachable()) std::memmove(target, data_, bytes);
        else cudaCall(cudaMemcpy(target, data_, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }

    [[nodiscard]] void *data() noexcept { return data_; }
    [[nodiscard]] const void *data() const noexcept { return data_; }

    /// Device address: the allocation itself, or for mapped memory its device
    /// alias; pinned memory has no guaranteed device view (std::logic_error).
    [[nodiscard]] void *deviceData() const {
        if (!bytes_) return nullptr;
        switch (memoryType()) {
            case MemoryType::Pinned:
                throw std::logic_error("Pinned memory has no guaranteed device view; use MappedMemory");
            case MemoryType::Mapped: {
                DeviceSwitch on(device_);
                void *alias = nullptr;
                cudaCall(cudaHostGetDevicePointer(&alias, data_, 0), "cudaHostGetDevicePointer");
                return alias;
            }
            default:
                return data_;
        }
    }
    /// Host address; device (global) memory has none (std::logic_error).
    [[nodiscard]] void *hostData() const {
        if (bytes_ && memoryType() == MemoryType::Global) throw std::logic_error("Global memory is not host accessible");
        return data_;
    }

    [[nodiscard]] std::size_t sizeBytes() const noexcept { return bytes_; }
    [[nodiscard]] int deviceId() const noexcept { return device_; }
    [[nodiscard]] MemoryType memoryType() const noexcept { return static_cast<MemoryType>(strategy_.index()); }
    [[nodiscard]] const MemoryStrategy &memoryStrategy() const noexcept { return strategy_; }

  private:
    bool hostReachable() const noexcept { return strategyOps(memoryType()).hostAccessible; }

    void release() noexcept {
        if (data_) {
            int current = -1;
            const bool known = cudaGetDevice(&current) == cudaSuccess;
            if (!known || current != device_) (void)cudaSetDevice(device_);
            strategyOps(memoryType()).release(data_);
            if (known && current != device_) (void)cudaSetDevice(current);
        }
        data_ = nullptr;
        bytes_ = 0;
        device_ = -1;
    }

    void *data_{nullptr};
    std::size_t bytes_{0};
    int device_{-1};
    MemoryStrategy strategy_;
};

}  // namespace detail
}  // namespace thermofem
