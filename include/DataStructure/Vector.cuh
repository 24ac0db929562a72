// Vector.cuh -- one-dimensional vector over a CudaBuffer (drop-in for
// include/DataStructure/Vector.cuh of Mgepahmge/ThermoFEM, lines 22-106: the
// same constructors, copy/move semantics and accessors).  The vector owns
// one buffer; its length is the buffer's; no implicit conversion to the
// buffer (values() gives read access to it).
#pragma once

#include <DataStructure/CudaBuffer.cuh>

namespace thermofem {

template <BufferElement T>
class Vector {
  public:
    using ValueType = T;

    explicit Vector(MemoryStrategy strategy = GlobalMemory{}) noexcept : buffer_(strategy) {}
    explicit Vector(std::size_t count, MemoryStrategy strategy = GlobalMemory{}) : buffer_(count, strategy) {}
    explicit Vector(std::span<const T> values, MemoryStrategy strategy = GlobalMemory{}) : buffer_(values, strategy) {}

    void copyDataFrom(const Vector &other) { buffer_.copyDataFrom(other.buffer_); }
    void copyDataFrom(const CudaBuffer<T> &other) { buffer_.copyDataFrom(other); }
    void changeMemoryType(MemoryStrategy strategy) { buffer_.changeMemoryType(strategy); }
    void copyFromHost(std::span<const T> values) { buffer_.copyFromHost(values); }
    void copyToHost(std::span<T> values) const { buffer_.copyToHost(values); }
    void swap(Vector &other) noexcept { buffer_.swap(other.buffer_); }

    [[nodiscard]] std::size_t size() const noexcept { return buffer_.size(); }
    [[nodiscard]] bool empty() const noexcept { return buffer_.empty(); }
    [[nodiscard]] std::size_t sizeBytes() const noexcept { return buffer_.sizeBytes(); }
    [[nodiscard]] int deviceId() const noexcept { return buffer_.deviceId(); }
    [[nodiscard]] MemoryType memoryType() const noexcept { return buffer_.memoryType(); }
    [[nodiscard]] const MemoryStrategy &memoryStrategy() const noexcept { return buffer_.memoryStrategy(); }
    [[nodiscard]] const CudaBuffer<T> &values() const noexcept { return buffer_; }

    [[nodiscard]] T *data() noexcept { return buffer_.data(); }
    [[nodiscard]] const T *data() const noexcept { return buffer_.data(); }
    [[nodiscard]] T *hostData() { return buffer_.hostData(); }
    [[nodiscard]] const T *hostData() const { return buffer_.hostData(); }
    [[nodiscard]] T *deviceData() { return buffer_.deviceData(); }
    [[nodiscard]] const T *deviceData() const { return buffer_.deviceData(); }

  private:
    CudaBuffer<T> buffer_;
};

}  // namespace thermofem
