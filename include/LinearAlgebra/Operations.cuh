// Operations.cuh -- the shared helpers of the linear-algebra layer that the
// solve path uses (drop-in for commonDevice, librarySize, hostCopy,
// deviceCopy and canonical of include/LinearAlgebra/Operations.cuh of
// Mgepahmge/ThermoFEM, lines 10-130).  The reference's general dense and
// sparse operations in that header (products, sums, transposes) are not part
// of the solve path and are not provided.
#pragma once

#include <DataStructure/Vector.cuh>
#include <LinearAlgebra/Backend.cuh>

#include <algorithm>
#include <initializer_list>
#include <limits>
#include <utility>

namespace thermofem::linalg::detail {

/// The one device the operands share (-1 entries are empty operands and
/// ignored); std::invalid_argument when two operands sit on different devices.
inline int commonDevice(std::initializer_list<int> devices) {
    int common = -1;
    for (int d : devices) {
        if (d < 0) continue;
        if (common >= 0 && d != common) throw std::invalid_argument("Operands belong to different CUDA devices");
        common = d;
    }
    return common;
}

inline int librarySize(std::size_t count) {
    if (!std::in_range<int>(count)) throw std::length_error("Operation exceeds 32-bit library interface range");
    return static_cast<int>(count);
}

template <BufferElement T>
std::vector<T> hostCopy(const CudaBuffer<T> &buffer) {
    std::vector<T> out(buffer.size());
    buffer.copyToHost(out);
    return out;
}
template <BufferElement T>
std::vector<T> hostCopy(const Vector<T> &vector) {
    return hostCopy(vector.values());
}

template <BufferElement T>
CudaBuffer<T> deviceCopy(const CudaBuffer<T> &buffer) {
    CudaBuffer<T> out(buffer.size());
    out.copyDataFrom(buffer);
    return out;
}
template <BufferElement T>
CudaBuffer<T> deviceCopy(const Vector<T> &vector) {
    return deviceCopy(vector.values());
}

/// Row-sorted copy with duplicate columns summed in their input order
/// (explicit zeros kept), index type Out, global memory.  Computed on the
/// host: callers use it only for inputs whose device check found unsorted
/// or repeated columns.
template <CsrIndex Out, Scalar T, CsrIndex I>
CsrMatrix<T, Out> canonical(const CsrMatrix<T, I> &m) {
    if (!std::in_range<Out>(m.rowCount()) || !std::in_range<Out>(m.columnCount()) ||
        !std::in_range<Out>(m.nonZeroCount()))
        throw std::length_error("Sparse operation exceeds its structural index range");
    const auto off = hostCopy(m.rowOffsets());
    const auto col = hostCopy(m.columnIndices());
    const auto val = hostCopy(m.values());
    std::vector<Out> rp(m.rowCount() + 1, 0), ci;
    std::vector<T> cv;
    ci.reserve(col.size());
    cv.reserve(val.size());
    std::vector<std::size_t> order;
    for (std::size_t r = 0; r < m.rowCount(); ++r) {
        order.clear();
        for (auto j = off[r]; j < off[r + 1]; ++j) order.push_back(static_cast<std::size_t>(j));
        std::stable_sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return col[a] < col[b]; });
        const std::size_t rowStart = ci.size();
        for (std::size_t j : order) {
            if (ci.size() > rowStart && ci.back() == static_cast<Out>(col[j])) cv.back() += val[j];
            else {
                ci.push_back(static_cast<Out>(col[j]));
                cv.push_back(val[j]);
            }
        }
        rp[r + 1] = static_cast<Out>(ci.size());
    }
    return CsrMatrix<T, Out>(m.rowCount(), m.columnCount(), rp, ci, cv);
}

}  // namespace thermofem::linalg::detail
