// CsrMatrix.cuh -- compressed-row sparse matrix over three CudaBuffers
// (drop-in for include/DataStructure/CsrMatrix.cuh of Mgepahmge/ThermoFEM,
// lines 36-217: the same constructors, checks, messages and accessors).
// Unsorted and duplicate column indices and explicit zeros are allowed; the
// structure is read-only, the values can be replaced; the three buffers
// always share one strategy; a default or moved-from matrix is 0 x 0 with no
// storage.  Host input is checked on the host before anything is allocated;
// buffers handed over by fromBuffers are checked on their GPU
// (tf_csr_validate) before the matrix takes them.
#pragma once

#include <DataStructure/CudaBuffer.cuh>
#include <thermofem/b200.cuh>

#include <concepts>
#include <cstdint>
#include <limits>
#include <utility>

namespace thermofem {

template <class T>
concept CsrIndex = std::signed_integral<T> && (sizeof(T) == 4 || sizeof(T) == 8);

namespace detail {

/// Checks offsets and column indices of a device CSR on its device
/// (replaces the reference's detail::validateDeviceCsr, src/DataStructure/
/// CsrMatrix.cu:12-58): std::invalid_argument when malformed.
inline void validateDeviceCsr(std::size_t rows, std::size_t columns, std::size_t count, const void *offsets,
                              const void *indices, bool wide, int device) {
    if (!rows) return;
    tf_csr view{static_cast<int64_t>(rows), static_cast<int64_t>(columns), static_cast<int64_t>(count),
                wide ? TF_I64 : TF_I32, TF_F64, offsets, indices, nullptr};
    auto &ctx = b200::ambient(device);
    b200::onContext(ctx, [&] {
        // the values are not read by the structural check
        view.values = count ? indices : nullptr;
        const int status = tf_csr_validate(ctx.get(), &view);
        if (status == TF_ERR_INVALID) throw std::invalid_argument("Invalid CSR device buffers");
        b200::check(status);
    });
}

}  // namespace detail

template <BufferElement T, CsrIndex Index = std::int32_t>
class CsrMatrix {
  public:
    using ValueType = T;

    CsrMatrix() = default;

    /// Takes three global buffers of one device (results of GPU algorithms)
    /// after checking them there; on failure the inputs are not moved from.
    static CsrMatrix fromBuffers(std::size_t rows, std::size_t columns, CudaBuffer<Index> &&offsets,
                                 CudaBuffer<Index> &&indices, CudaBuffer<T> &&values) {
        if (!std::in_range<Index>(rows) || !std::in_range<Index>(columns) || !std::in_range<Index>(values.size()) ||
            rows == std::numeric_limits<std::size_t>::max())
            throw std::length_error("CSR dimensions exceed index range");
        const bool global = offsets.memoryType() == MemoryType::Global &&
                            indices.memoryType() == MemoryType::Global && values.memoryType() == MemoryType::Global;
        const bool oneDevice = (indices.empty() || indices.deviceId() == offsets.deviceId()) &&
                               (values.empty() || values.deviceId() == offsets.deviceId());
        if (offsets.size() != rows + 1 || indices.size() != values.size() || !global || !oneDevice)
            throw std::invalid_argument("Invalid CSR device buffers");
        detail::validateDeviceCsr(rows, columns, values.size(), offsets.deviceData(), indices.deviceData(),
                                  sizeof(Index) == 8, offsets.deviceId());
        CsrMatrix m;
        m.rows_ = rows;
        m.columns_ = columns;
        m.offsets_ = std::move(offsets);
        m.indices_ = std::move(indices);
        m.values_ = std::move(values);
        return m;
    }

    CsrMatrix(std::size_t rows, std::size_t columns, std::span<const Index> rowOffsets,
              std::span<const Index> columnIndices, std::span<const T> values, MemoryStrategy strategy = GlobalMemory{})
        : rows_(rows), columns_(columns) {
        checkHost(rows, columns, rowOffsets, columnIndices, values.size());
        offsets_ = CudaBuffer<Index>(rowOffsets, strategy);
        indices_ = CudaBuffer<Index>(columnIndices, strategy);
        values_ = CudaBuffer<T>(values, strategy);
    }

    CsrMatrix(const CsrMatrix &) = default;
    CsrMatrix(CsrMatrix &&other) noexcept { swap(other); }
    CsrMatrix &operator=(const CsrMatrix &other) {
        if (this != &other) {
            CsrMatrix copy(other);
            swap(copy);
        }
        return *this;
    }
    CsrMatrix &operator=(CsrMatrix &&other) noexcept {
        if (this != &other) {
            CsrMatrix taken(std::move(other));
            swap(taken);
        }
        return *this;
    }

    void swap(CsrMatrix &other) noexcept {
        std::swap(rows_, other.rows_);
        std::swap(columns_, other.columns_);
        offsets_.swap(other.offsets_);
        indices_.swap(other.indices_);
        values_.swap(other.values_);
    }

    /// Moves all three buffers to another strategy; on failure nothing changes.
    void changeMemoryType(MemoryStrategy strategy) {
        if (values_.memoryStrategy().index() == strategy.index()) return;
        CsrMatrix moved(*this);
        moved.offsets_.changeMemoryType(strategy);
        moved.indices_.changeMemoryType(strategy);
        moved.values_.changeMemoryType(strategy);
        swap(moved);
    }

    void copyValuesFromHost(std::span<const T> values) { values_.copyFromHost(values); }

    [[nodiscard]] std::size_t rowCount() const noexcept { return rows_; }
    [[nodiscard]] std::size_t columnCount() const noexcept { return columns_; }
    [[nodiscard]] std::size_t nonZeroCount() const noexcept { return values_.size(); }
    [[nodiscard]] MemoryType memoryType() const noexcept { return values_.memoryType(); }
    [[nodiscard]] const CudaBuffer<Index> &rowOffsets() const noexcept { return offsets_; }
    [[nodiscard]] const CudaBuffer<Index> &columnIndices() const noexcept { return indices_; }
    [[nodiscard]] const CudaBuffer<T> &values() const noexcept { return values_; }
    [[nodiscard]] T *deviceValues() { return values_.deviceData(); }
    [[nodiscard]] const T *deviceValues() const { return values_.deviceData(); }

  private:
    static void checkHost(std::size_t rows, std::size_t columns, std::span<const Index> offsets,
                          std::span<const Index> indices, std::size_t count) {
        if (!std::in_range<Index>(rows) || !std::in_range<Index>(columns) || !std::in_range<Index>(count) ||
            rows == std::numeric_limits<std::size_t>::max())
            throw std::length_error("CSR dimensions exceed the index range");
        if (offsets.size() != rows + 1 || indices.size() != count || offsets.front() != 0 ||
            offsets.back() != static_cast<Index>(count))
            throw std::invalid_argument("Invalid CSR array sizes or endpoints");
        Index last = 0;
        for (Index o : offsets) {
            if (o < last || o > static_cast<Index>(count))
                throw std::invalid_argument("CSR row offsets must be nondecreasing and bounded");
            last = o;
        }
        for (Index c : indices)
            if (c < 0 || static_cast<std::size_t>(c) >= columns)
                throw std::invalid_argument("CSR column index is out of range");
    }

    std::size_t rows_{0}, columns_{0};
    CudaBuffer<Index> offsets_;
    CudaBuffer<Index> indices_;
    CudaBuffer<T> values_;
};

namespace b200 {

/// The C ABI's view of a matrix whose buffers the device can read.
template <class T, class I>
tf_csr describe(const CsrMatrix<T, I> &a) {
    const bool any = a.rowCount() > 0;
    return tf_csr{static_cast<int64_t>(a.rowCount()), static_cast<int64_t>(a.columnCount()),
                  static_cast<int64_t>(a.nonZeroCount()), indexType<I>(), valueType<T>(),
                  any ? a.rowOffsets().deviceData() : nullptr,
                  a.nonZeroCount() ? a.columnIndices().deviceData() : nullptr,
                  a.nonZeroCount() ? a.values().deviceData() : nullptr};
}

}  // namespace b200
}  // namespace thermofem
