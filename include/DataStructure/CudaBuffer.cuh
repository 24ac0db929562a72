// CudaBuffer.cuh -- typed CUDA buffer with value semantics and a switchable
// memory strategy (drop-in for include/DataStructure/CudaBuffer.cuh of
// Mgepahmge/ThermoFEM, lines 1-150: same names and semantics).  Elements are
// uninitialised after allocation; the synchronous copies require the caller
// to have finished any asynchronous access first; changing the strategy may
// move the data (old pointers become invalid).
#pragma once

#include <DataStructure/Memory.cuh>

#include <span>
#include <type_traits>

namespace thermofem {

/// Elements that can be moved as bytes and need no constructor or destructor.
template <class T>
concept BufferElement = std::is_trivially_copyable_v<T> && std::is_trivially_default_constructible_v<T> &&
                        std::is_trivially_destructible_v<T> && !std::is_const_v<T> && !std::is_volatile_v<T> &&
                        !std::is_pointer_v<T> && (alignof(T) <= alignof(std::max_align_t));

template <BufferElement T>
class CudaBuffer {
  public:
    explicit CudaBuffer(MemoryStrategy strategy = GlobalMemory{}) noexcept : bytes_(strategy) {}
    explicit CudaBuffer(std::size_t count, MemoryStrategy strategy = GlobalMemory{})
        : bytes_(detail::checkedProduct(count, sizeof(T)), strategy) {}
    explicit CudaBuffer(std::span<const T> values, MemoryStrategy strategy = GlobalMemory{})
        : CudaBuffer(values.size(), strategy) {
        copyFromHost(values);
    }

    void copyDataFrom(const CudaBuffer &other) { bytes_.copyDataFrom(other.bytes_); }
    void changeMemoryType(MemoryStrategy strategy) { bytes_.changeMemoryType(strategy); }
    void copyFromHost(std::span<const T> values) {
        bytes_.copyFromHost(values.data(), detail::checkedProduct(values.size(), sizeof(T)));
    }
    void copyToHost(std::span<T> values) const {
        bytes_.copyToHost(values.data(), detail::checkedProduct(values.size(), sizeof(T)));
    }
    void swap(CudaBuffer &other) noexcept { bytes_.swap(other.bytes_); }

    [[nodiscard]] std::size_t size() const noexcept { return bytes_.sizeBytes() / sizeof(T); }
    [[nodiscard]] bool empty() const noexcept { return size() == 0; }
    [[nodiscard]] std::size_t sizeBytes() const noexcept { return bytes_.sizeBytes(); }
    [[nodiscard]] int deviceId() const noexcept { return bytes_.deviceId(); }
    [[nodiscard]] MemoryType memoryType() const noexcept { return bytes_.memoryType(); }
    [[nodiscard]] const MemoryStrategy &memoryStrategy() const noexcept { return bytes_.memoryStrategy(); }

    [[nodiscard]] T *data() noexcept { return static_cast<T *>(bytes_.data()); }
    [[nodiscard]] const T *data() const noexcept { return static_cast<const T *>(bytes_.data()); }
    [[nodiscard]] T *hostData() { return static_cast<T *>(bytes_.hostData()); }
    [[nodiscard]] const T *hostData() const { return static_cast<const T *>(bytes_.hostData()); }
    [[nodiscard]] T *deviceData() { return static_cast<T *>(bytes_.deviceData()); }
    [[nodiscard]] const T *deviceData() const { return static_cast<const T *>(bytes_.deviceData()); }

  private:
    detail::MemoryStorage bytes_;
};

}  // namespace thermofem
