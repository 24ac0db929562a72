// ref_gpu_shim.cu -- test infrastructure, never linked by the product.
//
// A C entry point over the reference's own GPU solve path (its Cg / BiCgStab
// with its aggregation Amg, cuSPARSE/cuBLAS/CUB underneath), compiled by
// oracle/Makefile from the reference sources where they lie into
// oracle/_ref/libref_gpu.so.  The tests call it to compare this library's
// solves with the reference's on the same inputs, and report its time.
//
// Reference API used: CsrMatrix(rows, cols, offsets, columns, values)
// (include/DataStructure/CsrMatrix.cuh:81-87), Vector(span)
// (include/DataStructure/Vector.cuh:34), copyToHost (Vector.cuh:65),
// AmgOptions (include/Preconditioner/Amg.cuh:14-25), Amg(options)
// (Amg.cuh:64), Identity (include/Preconditioner/Identity.cuh:17-36),
// Cg(options, preconditioner) (include/Solver/Cg.cuh:44),
// BiCgStab(options, preconditioner) (include/Solver/BiCgStab.cuh:50),
// setup / apply and SolveResult (include/Solver/Interfaces.cuh).
#include <Preconditioner/Amg.cuh>
#include <Preconditioner/Identity.cuh>
#include <Solver/BiCgStab.cuh>
#include <Solver/Cg.cuh>

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <exception>
#include <memory>
#include <span>
#include <vector>

namespace {

using namespace thermofem;

// T: the reference components' value type (double or float; float inputs
// are the double ones rounded, float results are widened back).
template <class T, class S, class O>
int run(const int32_t *rp, const int32_t *ci, const double *val64, int64_t n, const double *b64, double *x64,
        int precond, int cycle, double jacobi_weight, int coarse_rows, int repeats, int *iterations, int *status,
        double *rel_residual, double *setup_seconds, double *solve_seconds) {
    const int64_t nnz = rp[n];
    const std::vector<T> val(val64, val64 + nnz), b(b64, b64 + n);
    std::vector<T> x(x64, x64 + n);
    CsrMatrix<T> a(static_cast<std::size_t>(n), static_cast<std::size_t>(n),
                   std::span<const int>(rp, static_cast<std::size_t>(n + 1)),
                   std::span<const int>(ci, static_cast<std::size_t>(nnz)),
                   std::span<const T>(val.data(), static_cast<std::size_t>(nnz)));
    AmgOptions<T> ao;
    ao.jacobiWeight_ = static_cast<T>(jacobi_weight);
    ao.coarseRows_ = coarse_rows;
    ao.cycle_ = cycle == 1 ? multigrid::Cycle::W : (cycle == 2 ? multigrid::Cycle::F : multigrid::Cycle::V);
    O so;
    // precond 0: Identity, passed explicitly (BiCgStab builds an Amg when given none)
    S solver(so, precond ? std::unique_ptr<Preconditioner<T>>(std::make_unique<Amg<T>>(ao))
                         : std::unique_ptr<Preconditioner<T>>(std::make_unique<Identity<T>>()));
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    solver.setup(a);
    cudaDeviceSynchronize();
    *setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    Vector<T> rhs(std::span<const T>(b.data(), static_cast<std::size_t>(n)));
    double best = 0;
    for (int r = 0; r < (repeats < 1 ? 1 : repeats); ++r) {
        Vector<T> xv(std::span<const T>(x.data(), static_cast<std::size_t>(n)));
        cudaDeviceSynchronize();
        t0 = std::chrono::steady_clock::now();
        const auto res = solver.apply(rhs, xv);
        cudaDeviceSynchronize();
        const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (r == 0 || t < best) best = t;
        if (r + 1 == (repeats < 1 ? 1 : repeats)) {
            std::vector<T> out(static_cast<std::size_t>(n));
            xv.copyToHost(std::span<T>(out.data(), out.size()));
            for (int64_t i = 0; i < n; ++i) x64[i] = static_cast<double>(out[static_cast<std::size_t>(i)]);
            *iterations = res.iterations_;
            *status = static_cast<int>(res.status_);
            *rel_residual = static_cast<double>(res.relativeResidual_);
        }
    }
    *solve_seconds = best;
    return 0;
}

}  // namespace

// Solves A x = b with the reference's solver (FP64, or FP32 with single;
// kind 0 PCG, 1 BiCGStab;
// precond 1 its aggregation AMG, cycle 0 V, 1 W, 2 F; precond 0 identity)
// from the initial guess in x, `repeats`
// times from that guess; x receives the last solution.  Times are host wall
// clock around device-synchronised calls (setup once, the fastest solve).
// Returns 0, or -1 after printing the exception the reference raised.
extern "C" int ref_gpu_solve(int kind, const int32_t *rp, const int32_t *ci, const double *val, int64_t n,
                             const double *b, double *x, int precond, int cycle, double jacobi_weight, int coarse_rows,
                             int repeats, int single, int *iterations, int *status, double *rel_residual,
                             double *setup_seconds, double *solve_seconds) {
    try {
#define TF_REF_RUN(T, S, O)                                                                                      \
    return run<T, S, O>(rp, ci, val, n, b, x, precond, cycle, jacobi_weight, coarse_rows, repeats, iterations, \
                        status, rel_residual, setup_seconds, solve_seconds)
        if (single) {
            if (kind == 1) TF_REF_RUN(float, BiCgStab<float>, BiCgStabOptions<float>);
            TF_REF_RUN(float, Cg<float>, CgOptions<float>);
        }
        if (kind == 1) TF_REF_RUN(double, BiCgStab<double>, BiCgStabOptions<double>);
        TF_REF_RUN(double, Cg<double>, CgOptions<double>);
#undef TF_REF_RUN
    } catch (const std::exception &e) {
        std::fprintf(stderr, "reference solve failed: %s\n", e.what());
        return -1;
    }
}

// Builds the reference's Amg<double> (include/Preconditioner/Amg.cuh:81-143)
// on the matrix and reports its diagnostics: the level count, per level the
// rows, nonzeros and aggregate-size histogram (levelStatistics,
// Amg.cuh:163-172), the stop reason and the coarse solver.  Up to `capacity`
// levels are written; stop_reason / coarse_solver receive NUL-terminated text
// (64 bytes each).  Returns the level count, or -1 after printing the
// exception the reference raised.
extern "C" int ref_gpu_amg_levels(const int32_t *rp, const int32_t *ci, const double *val, int64_t n,
                                  double jacobi_weight, int coarse_rows, int capacity, int64_t *rows, int64_t *nnz,
                                  int64_t *histogram, char *stop_reason, char *coarse_solver) {
    try {
        const int64_t count = rp[n];
        CsrMatrix<double> a(static_cast<std::size_t>(n), static_cast<std::size_t>(n),
                            std::span<const int>(rp, static_cast<std::size_t>(n + 1)),
                            std::span<const int>(ci, static_cast<std::size_t>(count)),
                            std::span<const double>(val, static_cast<std::size_t>(count)));
        AmgOptions<double> ao;
        ao.jacobiWeight_ = jacobi_weight;
        ao.coarseRows_ = coarse_rows;
        Amg<double> amg(ao);
        amg.setup(a);
        const auto &stats = amg.levelStatistics();
        for (std::size_t d = 0; d < stats.size() && static_cast<int>(d) < capacity; ++d) {
            rows[d] = static_cast<int64_t>(stats[d].rows_);
            nnz[d] = static_cast<int64_t>(stats[d].nonzeros_);
            for (int k = 0; k < 4; ++k) histogram[4 * d + k] = stats[d].aggregateSizes_[k];
        }
        std::snprintf(stop_reason, 64, "%s", amg.stopReason().c_str());
        std::snprintf(coarse_solver, 64, "%s", amg.coarseSolver().c_str());
        return static_cast<int>(amg.levelCount());
    } catch (const std::exception &e) {
        std::fprintf(stderr, "reference AMG setup failed: %s\n", e.what());
        return -1;
    }
}

namespace {

// A Preconditioner that forwards to an Amg owned elsewhere and sets it up
// once, so that the reference's Cg and BiCgStab (each of which owns its
// preconditioner) solve with one hierarchy, built once.
struct SharedAmg final : Preconditioner<double> {
    Amg<double> *amg;
    bool *ready;
    SharedAmg(Amg<double> *a, bool *r) : amg(a), ready(r) {}
    void setup(const CsrMatrix<double> &m) override {
        if (!*ready) {
            amg->setup(m);
            *ready = true;
        }
    }
    void apply(const Vector<double> &rhs, Vector<double> &x) override { amg->apply(rhs, x); }
};

}  // namespace

// The reference's FP64 PCG and BiCGStab (V-cycle AMG, the given Jacobi
// weight and coarse limit, rtol 1e-8) on one matrix and right-hand side,
// from a zero guess, with one AMG setup shared by both.  Per solver k
// (0 PCG, 1 BiCGStab): iterations[k], status[k], rel_residual[k], the
// fastest of `repeats` solves solve_seconds[k], and the solution in
// x_pcg / x_bicgstab.  setup_seconds: the AMG setup plus each solver's
// own setup.  Host wall clock around device-synchronised calls.  Returns 0,
// or -1 after printing the exception the reference raised.
extern "C" int ref_gpu_solve_pair(const int32_t *rp, const int32_t *ci, const double *val, int64_t n,
                                  const double *b, double jacobi_weight, int coarse_rows, int repeats,
                                  double *setup_seconds, int *iterations, int *status, double *rel_residual,
                                  double *solve_seconds, double *x_pcg, double *x_bicgstab) {
    try {
        const int64_t count = rp[n];
        CsrMatrix<double> a(static_cast<std::size_t>(n), static_cast<std::size_t>(n),
                            std::span<const int>(rp, static_cast<std::size_t>(n + 1)),
                            std::span<const int>(ci, static_cast<std::size_t>(count)),
                            std::span<const double>(val, static_cast<std::size_t>(count)));
        AmgOptions<double> ao;
        ao.jacobiWeight_ = jacobi_weight;
        ao.coarseRows_ = coarse_rows;
        Amg<double> amg(ao);
        bool ready = false;
        Cg<double> cg(CgOptions<double>{}, std::make_unique<SharedAmg>(&amg, &ready));
        BiCgStab<double> bicg(BiCgStabOptions<double>{}, std::make_unique<SharedAmg>(&amg, &ready));
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        cg.setup(a);
        bicg.setup(a);
        cudaDeviceSynchronize();
        *setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const Vector<double> rhs(std::span<const double>(b, static_cast<std::size_t>(n)));
        const std::vector<double> zeros(static_cast<std::size_t>(n), 0.0);
        Solver<double> *solvers[2] = {&cg, &bicg};
        double *outs[2] = {x_pcg, x_bicgstab};
        for (int k = 0; k < 2; ++k) {
            double best = 0;
            for (int r = 0; r < (repeats < 1 ? 1 : repeats); ++r) {
                Vector<double> x(std::span<const double>(zeros.data(), zeros.size()));
                cudaDeviceSynchronize();
                t0 = std::chrono::steady_clock::now();
                const auto res = solvers[k]->apply(rhs, x);
                cudaDeviceSynchronize();
                const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                if (r == 0 || t < best) best = t;
                iterations[k] = res.iterations_;
                status[k] = static_cast<int>(res.status_);
                rel_residual[k] = res.relativeResidual_;
                if (outs[k]) x.copyToHost(std::span<double>(outs[k], static_cast<std::size_t>(n)));
            }
            solve_seconds[k] = best;
        }
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "reference solve failed: %s\n", e.what());
        return -1;
    }
}
