// krylov.cuh -- the machinery behind thermofem::Cg and thermofem::BiCgStab.
//
// Fused path: with the library's own preconditioners (Identity, or Amg with
// its default Jacobi smoothers) the whole solve is the library's solver
// (tf_solver_create / _setup / _apply): the recurrence of the reference
// (Cg.cuh:123-189, BiCgStab.cuh:144-247) with its scalars on the device,
// fused vector kernels, and the whole iteration loop captured into one CUDA
// graph; the Amg object then reports the hierarchy that solver built.
//
// Host path: with any other preconditioner (a caller's class, or Amg with a
// smoother factory) the same recurrence runs from the host: the library's
// SpMV, residual, dot and fused update kernels on the solver's context, and
// Preconditioner::apply called where the recurrence needs M^-1.  Both paths
// end with the true residual of the returned x and report it, as the
// reference does.
#pragma once

#include <Preconditioner/Amg.cuh>
#include <Preconditioner/Identity.cuh>

#include <algorithm>
#include <cmath>

namespace thermofem::b200 {

template <linalg::Scalar T, CsrIndex I>
class KrylovEngine {
  public:
    struct Options {
        int maxIterations;
        T relativeTolerance, absoluteTolerance;
        int refresh;
    };

    KrylovEngine(int kind, Options o) : kind_(kind), o_(o) {}

    void reset() noexcept { state_.reset(); }

    void setup(const CsrMatrix<T, I> &matrix, Preconditioner<T, I> &pre) {
        state_.reset();
        auto *amg = dynamic_cast<Amg<T, I> *>(&pre);
        if (amg) amg->forget();
        iteration::validateMatrix(matrix);
        const int device = matrix.rowOffsets().deviceId();
        linalg::detail::OperationScope scope(device);
        auto next = std::make_unique<State>(device, matrix.rowCount());
        CsrMatrix<T, I> global;
        const CsrMatrix<T, I> *m = &matrix;
        if (matrix.memoryType() != MemoryType::Global) {
            global = matrix;
            global.changeMemoryType(GlobalMemory{});
            m = &global;
        }
        auto *identity = dynamic_cast<Identity<T, I> *>(&pre);
        const bool fused = identity || (amg && amg->runsInLibrary());
        if (fused) {
            tf_solver_options so;
            tf_solver_options_default(valueType<T>(), &so);
            so.max_iterations = o_.maxIterations;
            so.relative_tolerance = static_cast<double>(o_.relativeTolerance);
            so.absolute_tolerance = static_cast<double>(o_.absoluteTolerance);
            so.residual_refresh_interval = o_.refresh;
            tf_amg_options ao;
            if (amg) ao = amg->libraryOptions();
            const tf_csr view = describe(*m);
            onContext(next->ctx, [&] {
                tf_solver *h = nullptr;
                check(tf_solver_create(next->ctx.get(), kind_, valueType<T>(), indexType<I>(), &so,
                                       amg ? TF_PRECOND_AMG : TF_PRECOND_IDENTITY, amg ? &ao : nullptr, &h));
                next->solver.reset(h);
                const int status = tf_solver_setup(h, &view);
                if (status == TF_ERR_INVALID) throw std::invalid_argument(tf_last_error());
                check(status);
            });
            if (identity) identity->setup(*m);
            if (amg) amg->adopt(tf_solver_amg(next->solver.get()), device);
        } else {
            next->host = std::make_unique<HostLoop>(*m);
            pre.setup(next->host->context.matrix());
        }
        state_ = std::move(next);
    }

    SolveResult<T> apply(const Vector<T> &rhs, Vector<T> &x, Preconditioner<T, I> &pre, const char *name) {
        if (!state_) throw std::logic_error(std::string(name) + " requires setup");
        State &s = *state_;
        iteration::validateVectors(s.n, s.ctx.device(), rhs, x);
        linalg::detail::OperationScope scope(s.ctx.device());
        if (s.solver) {
            tf_solve_result r{};
            // the solve's own copies (cudaMemcpyDefault) move rhs and x whatever their memory type
            onContext(s.ctx, [&] { check(tf_solver_apply(s.solver.get(), rhs.data(), x.data(), 0, &r)); });
            return {static_cast<SolveStatus>(r.status), r.iterations, static_cast<T>(r.residual_norm),
                    static_cast<T>(r.relative_residual)};
        }
        HostLoop &h = *s.host;
        h.rhs.copyDataFrom(rhs);
        h.x.copyDataFrom(x);
        const SolveResult<T> result = kind_ == TF_SOLVER_CG ? h.cg(o_, pre) : h.bicgstab(o_, pre);
        x.copyDataFrom(h.x);
        return result;
    }

  private:
    struct ReleaseSolver {
        void operator()(tf_solver *s) const noexcept { tf_solver_destroy(s); }
    };

    // The host-driven recurrences, on global work vectors.
    struct HostLoop {
        linalg::IterationContext<T, I> context;
        Vector<T> rhs, x, r, z, p, q, shadow, s, t, sh;
        CudaBuffer<double> norm2;
        explicit HostLoop(const CsrMatrix<T, I> &a)
            : context(a), rhs(a.rowCount()), x(a.rowCount()), r(a.rowCount()), z(a.rowCount()), p(a.rowCount()),
              q(a.rowCount()), shadow(a.rowCount()), s(a.rowCount()), t(a.rowCount()), sh(a.rowCount()), norm2(1) {}

        int64_t n() const { return static_cast<int64_t>(x.size()); }
        // the library's fused steps write a squared norm to the device; read it
        T readNorm() {
            double v = 0;
            norm2.copyToHost(std::span<double>(&v, 1));
            return static_cast<T>(std::sqrt(v));
        }

        // residual of the returned x; NonFinite, Converged or the status given
        SolveResult<T> finish(SolveStatus status, int iterations, T normB, T tol) {
            context.residual(rhs, x, r);
            const T res = context.norm(r);
            if (!std::isfinite(res) || !std::isfinite(normB)) status = SolveStatus::NonFinite;
            else if (res <= tol) status = SolveStatus::Converged;
            else if (status == SolveStatus::Converged) status = SolveStatus::MaxIterations;
            return {status, iterations, res, normB > 0 ? res / normB : res};
        }

        SolveResult<T> cg(const Options &o, Preconditioner<T, I> &pre) {
            const T normB = context.norm(rhs);
            const T tol = std::max(o.absoluteTolerance, o.relativeTolerance * normB);
            context.residual(rhs, x, r);
            T res = context.norm(r);
            if (!std::isfinite(normB) || !std::isfinite(res)) return finish(SolveStatus::NonFinite, 0, normB, tol);
            if (res <= tol) return finish(SolveStatus::Converged, 0, normB, tol);
            T rhoOld = 0;
            bool restart = true;
            for (int it = 1; it <= o.maxIterations; ++it) {
                pre.apply(r, z);
                const T rho = context.dot(r, z);
                if (!std::isfinite(rho)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (rho <= 0) return finish(SolveStatus::Breakdown, it, normB, tol);
                const T beta = restart ? T(0) : rho / rhoOld;
                if (!restart && !std::isfinite(beta)) return finish(SolveStatus::NonFinite, it, normB, tol);
                direction(TF_SOLVER_CG, beta, T(0), restart);
                restart = false;
                context.multiply(p, q);
                const T curvature = context.dot(p, q);
                if (!std::isfinite(curvature)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (curvature <= 0) return finish(SolveStatus::Breakdown, it, normB, tol);
                const T alpha = rho / curvature;
                if (!std::isfinite(alpha)) return finish(SolveStatus::NonFinite, it, normB, tol);
                res = step([&](tf_ctx *c) {
                    return tf_krylov_cg_update(c, valueType<T>(), n(), alpha, p.data(), q.data(), x.data(), r.data(),
                                               norm2.data());
                });
                if (!std::isfinite(res)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (res <= tol || it % o.refresh == 0) {
                    context.residual(rhs, x, r);
                    res = context.norm(r);
                    if (!std::isfinite(res) || res <= tol) return finish(SolveStatus::MaxIterations, it, normB, tol);
                    restart = true;
                }
                rhoOld = rho;
            }
            return finish(SolveStatus::MaxIterations, o.maxIterations, normB, tol);
        }

        SolveResult<T> bicgstab(const Options &o, Preconditioner<T, I> &pre) {
            const T normB = context.norm(rhs);
            const T tol = std::max(o.absoluteTolerance, o.relativeTolerance * normB);
            context.residual(rhs, x, r);
            T res = context.norm(r);
            if (!std::isfinite(normB) || !std::isfinite(res)) return finish(SolveStatus::NonFinite, 0, normB, tol);
            if (res <= tol) return finish(SolveStatus::Converged, 0, normB, tol);
            shadow.copyDataFrom(r);
            T rhoOld = 1, alpha = 1, omega = 1;
            bool restart = true;
            for (int it = 1; it <= o.maxIterations; ++it) {
                const T rho = context.dot(shadow, r);
                if (!std::isfinite(rho)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (rho == 0) return finish(SolveStatus::Breakdown, it, normB, tol);
                const T beta = restart ? T(0) : (rho / rhoOld) * (alpha / omega);
                if (!restart && !std::isfinite(beta)) return finish(SolveStatus::NonFinite, it, normB, tol);
                direction(TF_SOLVER_BICGSTAB, beta, omega, restart);
                restart = false;
                pre.apply(p, z);  // z = M^-1 p
                context.multiply(z, q);  // q = v = A z
                const T den = context.dot(shadow, q);
                if (!std::isfinite(den)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (den == 0) return finish(SolveStatus::Breakdown, it, normB, tol);
                alpha = rho / den;
                if (!std::isfinite(alpha)) return finish(SolveStatus::NonFinite, it, normB, tol);
                const T normS = step([&](tf_ctx *c) {
                    return tf_krylov_bicgstab_s(c, valueType<T>(), n(), alpha, r.data(), q.data(), z.data(), x.data(),
                                                s.data(), norm2.data());
                });
                if (!std::isfinite(normS)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (normS <= tol) {
                    // converged at the half step: refresh and decide on the true residual
                    context.residual(rhs, x, r);
                    res = context.norm(r);
                    if (res <= tol || !std::isfinite(res)) return finish(SolveStatus::MaxIterations, it, normB, tol);
                    shadow.copyDataFrom(r);
                    restart = true;
                    continue;
                }
                pre.apply(s, sh);  // sh = M^-1 s
                context.multiply(sh, t);
                const T tt = context.dot(t, t), ts = context.dot(t, s);
                if (!std::isfinite(tt) || !std::isfinite(ts)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (tt == 0) return finish(SolveStatus::Breakdown, it, normB, tol);
                omega = ts / tt;
                if (!std::isfinite(omega)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (omega == 0) return finish(SolveStatus::Breakdown, it, normB, tol);
                res = step([&](tf_ctx *c) {
                    return tf_krylov_bicgstab_update(c, valueType<T>(), n(), omega, sh.data(), s.data(), t.data(),
                                                     x.data(), r.data(), norm2.data());
                });
                if (!std::isfinite(res)) return finish(SolveStatus::NonFinite, it, normB, tol);
                if (res <= tol || it % o.refresh == 0) {
                    context.residual(rhs, x, r);
                    res = context.norm(r);
                    if (res <= tol || !std::isfinite(res)) return finish(SolveStatus::MaxIterations, it, normB, tol);
                    shadow.copyDataFrom(r);
                    restart = true;
                }
                rhoOld = rho;
            }
            return finish(SolveStatus::MaxIterations, o.maxIterations, normB, tol);
        }

        // p = z + beta p (CG) or p = r + beta (p - omega q) (BiCGStab); p = z / r on a restart
        void direction(int kind, T beta, T omega, bool restart) {
            stepVoid([&](tf_ctx *c) {
                return kind == TF_SOLVER_CG
                           ? tf_krylov_cg_direction(c, valueType<T>(), n(), beta, restart ? 1 : 0, z.data(), p.data())
                           : tf_krylov_bicgstab_direction(c, valueType<T>(), n(), beta, omega, restart ? 1 : 0,
                                                          r.data(), q.data(), p.data());
            });
        }
        template <class F>
        T step(F &&call) {
            stepVoid(std::forward<F>(call));
            return readNorm();
        }
        template <class F>
        void stepVoid(F &&call) {
            auto &c = ambient(x.deviceId());
            onContext(c, [&] { check(call(c.get())); });
        }
    };

    struct State {
        Context ctx;
        std::size_t n;
        std::unique_ptr<tf_solver, ReleaseSolver> solver;  // fused path
        std::unique_ptr<HostLoop> host;                    // host path
        State(int device, std::size_t rows) : ctx(device), n(rows) {}
    };

    int kind_;
    Options o_;
    std::unique_ptr<State> state_;
};

}  // namespace thermofem::b200
