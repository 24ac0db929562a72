// Diagonal.cuh -- the inverse diagonal of a square CSR matrix (drop-in for
// linalg::inverseDiagonal, include/LinearAlgebra/Diagonal.cuh:13-36 of
// Mgepahmge/ThermoFEM).  Duplicate diagonal entries are summed; a missing,
// zero or nonfinite diagonal, or a nonfinite reciprocal, is
// std::invalid_argument.  The reference copies the matrix to the host for
// this; here it is one kernel on the matrix's device (tf_inverse_diagonal).
#pragma once

#include <LinearAlgebra/Operations.cuh>

namespace thermofem::linalg {

template <Scalar T, CsrIndex I>
Vector<T> inverseDiagonal(const CsrMatrix<T, I> &matrix) {
    if (!matrix.rowCount() || matrix.rowCount() != matrix.columnCount())
        throw std::invalid_argument("Inverse diagonal requires a nonempty square matrix");
    const int device = matrix.rowOffsets().deviceId();
    detail::OperationScope scope(device);
    const CsrMatrix<T, I> *source = &matrix;
    CsrMatrix<T, I> global;
    if (matrix.memoryType() != MemoryType::Global) {
        global = matrix;
        global.changeMemoryType(GlobalMemory{});
        source = &global;
    }
    Vector<T> inverse(matrix.rowCount());
    const tf_csr view = b200::describe(*source);
    auto &ctx = b200::ambient(device);
    b200::onContext(ctx, [&] {
        const int status = tf_inverse_diagonal(ctx.get(), &view, inverse.data());
        if (status == TF_ERR_INVALID) throw std::invalid_argument("Missing or invalid diagonal");
        b200::check(status);
    });
    return inverse;
}

}  // namespace thermofem::linalg
