// BiCgStab.cuh -- right-preconditioned BiCGStab (drop-in for
// include/Solver/BiCgStab.cuh:11-251 of Mgepahmge/ThermoFEM: BiCgStabOptions
// with the same fields, defaults and checks; the solver owns its
// preconditioner, an Amg with default options when none is given; the same
// setup, apply and reporting contract as Cg).  The shadow residual is reset
// with every refresh; a half step whose ||s|| meets the tolerance refreshes
// the residual and restarts; statuses: Converged, MaxIterations, Breakdown
// (rho = 0, r~.v = 0, t.t = 0 or omega = 0), NonFinite.
#pragma once

#include <Preconditioner/Amg.cuh>
#include <thermofem/krylov.cuh>

namespace thermofem {

template <linalg::Scalar T>
struct BiCgStabOptions {
    int maxIterations_{1000};
    T relativeTolerance_{std::same_as<T, float> ? T(1e-5) : T(1e-8)};
    T absoluteTolerance_{0};
    int residualRefreshInterval_{50};
};

template <linalg::Scalar T, CsrIndex I = int>
class BiCgStab final : public Solver<T, I> {
  public:
    explicit BiCgStab(BiCgStabOptions<T> options = {}, std::unique_ptr<Preconditioner<T, I>> preconditioner = {})
        : preconditioner_(std::move(preconditioner)), engine_(TF_SOLVER_BICGSTAB, checked(options)) {
        if (!preconditioner_) preconditioner_ = std::make_unique<Amg<T, I>>();
    }
    void setup(const CsrMatrix<T, I> &matrix) override { engine_.setup(matrix, *preconditioner_); }
    SolveResult<T> apply(const Vector<T> &rhs, Vector<T> &x) override {
        return engine_.apply(rhs, x, *preconditioner_, "BiCGStab");
    }

  private:
    static typename b200::KrylovEngine<T, I>::Options checked(const BiCgStabOptions<T> &o) {
        if (o.maxIterations_ < 0 || o.residualRefreshInterval_ < 1 || !std::isfinite(o.relativeTolerance_) ||
            o.relativeTolerance_ < 0 || o.relativeTolerance_ >= 1 || !std::isfinite(o.absoluteTolerance_) ||
            o.absoluteTolerance_ < 0)
            throw std::invalid_argument("Invalid BiCGStab options");
        return {o.maxIterations_, o.relativeTolerance_, o.absoluteTolerance_, o.residualRefreshInterval_};
    }
    std::unique_ptr<Preconditioner<T, I>> preconditioner_;
    b200::KrylovEngine<T, I> engine_;
};

}  // namespace thermofem
