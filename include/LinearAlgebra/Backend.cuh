// Backend.cuh -- the precision concept and the device scope of the
// linear-algebra layer (drop-in for the in-scope part of
// include/LinearAlgebra/Backend.cuh of Mgepahmge/ThermoFEM, lines 8-32).
// The reference's cuBLAS/cuSPARSE wrappers behind it (blas*, sparse*) belong
// to its general dense/sparse operations, which this library does not carry:
// the solve path runs on the library's own kernels.
#pragma once

#include <DataStructure/CsrMatrix.cuh>

#include <concepts>
#include <vector>

namespace thermofem::linalg {

template <class T>
concept Scalar = std::same_as<T, float> || std::same_as<T, double>;

namespace detail {

/// Makes an operation's device current and restores the caller's device
/// afterwards; -1 leaves the current device as it is.
class OperationScope {
  public:
    explicit OperationScope(int device) : on_(device) {}
    OperationScope(const OperationScope &) = delete;
    OperationScope &operator=(const OperationScope &) = delete;

  private:
    thermofem::detail::DeviceSwitch on_;
};

}  // namespace detail
}  // namespace thermofem::linalg
