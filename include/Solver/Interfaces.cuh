// Interfaces.cuh -- the three component roles (smoother, preconditioner,
// solver) and the solve report (drop-in for include/Solver/Interfaces.cuh:
// 10-112 of Mgepahmge/ThermoFEM: the same classes, virtual methods, report
// fields and contract checks).
//
//   Smoother::apply       improves x from its current value;
//   Preconditioner::apply overwrites x with M^-1 rhs (x's old value unused);
//   Solver::apply         solves A x = rhs from the initial guess in x and
//                         returns a SolveResult; contract violations throw,
//                         numeric outcomes are SolveStatus values.
#pragma once

#include <LinearAlgebra/IterationContext.cuh>

namespace thermofem {

enum class SolveStatus { Converged, MaxIterations, Breakdown, NonFinite };

template <linalg::Scalar T>
struct SolveResult {
    SolveStatus status_{SolveStatus::MaxIterations};
    int iterations_{};
    T residualNorm_{};      ///< ||rhs - A x||_2 of the returned x (true residual)
    T relativeResidual_{};  ///< residualNorm_ / ||rhs||_2, or residualNorm_ when rhs = 0
};

template <linalg::Scalar T, CsrIndex I = int>
class Smoother {
  public:
    virtual ~Smoother() = default;
    virtual void setup(const CsrMatrix<T, I> &matrix) = 0;
    virtual void apply(const Vector<T> &rhs, Vector<T> &x) = 0;
};

template <linalg::Scalar T, CsrIndex I = int>
class Preconditioner {
  public:
    virtual ~Preconditioner() = default;
    virtual void setup(const CsrMatrix<T, I> &matrix) = 0;
    virtual void apply(const Vector<T> &rhs, Vector<T> &x) = 0;
};

template <linalg::Scalar T, CsrIndex I = int>
class Solver {
  public:
    virtual ~Solver() = default;
    virtual void setup(const CsrMatrix<T, I> &matrix) = 0;
    virtual SolveResult<T> apply(const Vector<T> &rhs, Vector<T> &x) = 0;
};

namespace iteration {

template <linalg::Scalar T, CsrIndex I>
void validateMatrix(const CsrMatrix<T, I> &matrix) {
    if (!matrix.rowCount() || matrix.rowCount() != matrix.columnCount())
        throw std::invalid_argument("Solver requires a nonempty square matrix");
}

template <linalg::Scalar T>
void validateVectors(std::size_t n, int device, const Vector<T> &rhs, const Vector<T> &x) {
    if (rhs.size() != n || x.size() != n) throw std::invalid_argument("Solver vector shape mismatch");
    linalg::detail::commonDevice({device, rhs.deviceId(), x.deviceId()});
}

}  // namespace iteration

namespace b200 {

/// A vector's elements where kernels can reach them: the vector itself when
/// it is device-reachable (global, managed, mapped through its device alias),
/// else (pinned host memory) a device copy that is written back on
/// writeBack().
template <class T>
class DeviceSide {
  public:
    DeviceSide(const Vector<T> &v, bool load) : source_(&v) {
        if (v.memoryType() == MemoryType::Pinned && !v.empty()) {
            staged_ = std::make_unique<Vector<T>>(v.size());
            if (load) staged_->copyDataFrom(v);
            ptr_ = staged_->data();
        } else {
            ptr_ = v.empty() ? nullptr : const_cast<T *>(v.deviceData());
        }
    }
    T *get() const noexcept { return ptr_; }
    void writeBack(Vector<T> &target) {
        if (staged_) target.copyDataFrom(*staged_);
    }

  private:
    const Vector<T> *source_;
    std::unique_ptr<Vector<T>> staged_;
    T *ptr_{nullptr};
};

}  // namespace b200
}  // namespace thermofem
