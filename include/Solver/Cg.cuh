// Cg.cuh -- preconditioned conjugate gradients (drop-in for
// include/Solver/Cg.cuh:10-193 of Mgepahmge/ThermoFEM: CgOptions with the
// same fields, defaults and checks; Cg owning its preconditioner, Identity
// by default; setup snapshots the matrix and invalidates the solver until it
// succeeds; apply solves from the initial guess in x, may alias rhs and x,
// keeps x's address and memory type, and reports the true residual).
// The recurrence refreshes the residual from b - A x and restarts the
// direction every residualRefreshInterval_ iterations and whenever the
// recursive residual meets the tolerance; statuses: Converged,
// MaxIterations, Breakdown (r.z <= 0 or p.Ap <= 0), NonFinite.
#pragma once

#include <Preconditioner/Identity.cuh>
#include <thermofem/krylov.cuh>

namespace thermofem {

template <linalg::Scalar T>
struct CgOptions {
    int maxIterations_{1000};
    T relativeTolerance_{std::same_as<T, float> ? T(1e-5) : T(1e-8)};
    T absoluteTolerance_{0};
    int residualRefreshInterval_{50};
};

template <linalg::Scalar T, CsrIndex I = int>
class Cg final : public Solver<T, I> {
  public:
    explicit Cg(CgOptions<T> options = {}, std::unique_ptr<Preconditioner<T, I>> preconditioner = {})
        : preconditioner_(std::move(preconditioner)), engine_(TF_SOLVER_CG, checked(options)) {
        if (!preconditioner_) preconditioner_ = std::make_unique<Identity<T, I>>();
    }
    void setup(const CsrMatrix<T, I> &matrix) override { engine_.setup(matrix, *preconditioner_); }
    SolveResult<T> apply(const Vector<T> &rhs, Vector<T> &x) override {
        return engine_.apply(rhs, x, *preconditioner_, "CG");
    }

  private:
    static typename b200::KrylovEngine<T, I>::Options checked(const CgOptions<T> &o) {
        if (o.maxIterations_ < 0 || o.residualRefreshInterval_ < 1 || !std::isfinite(o.relativeTolerance_) ||
            o.relativeTolerance_ < 0 || o.relativeTolerance_ >= 1 || !std::isfinite(o.absoluteTolerance_) ||
            o.absoluteTolerance_ < 0)
            throw std::invalid_argument("Invalid CG options");
        return {o.maxIterations_, o.relativeTolerance_, o.absoluteTolerance_, o.residualRefreshInterval_};
    }
    // declared before the engine: the engine (and the solver it may hold,
    // which owns a hierarchy the preconditioner reports) goes first
    std::unique_ptr<Preconditioner<T, I>> preconditioner_;
    b200::KrylovEngine<T, I> engine_;
};

}  // namespace thermofem
