// Amg.cuh -- the aggregation AMG preconditioner (drop-in for
// include/Preconditioner/Amg.cuh:13-278 of Mgepahmge/ThermoFEM: AmgOptions
// with the same fields, defaults and checks, AmgLevelStatistics, the
// SmootherFactory injection, transactional setup, the diagnostics).
//
// Two ways to run, one hierarchy.  Setup always builds the hierarchy with
// the library (tf_amg_setup: device canonicalisation, strength graphs,
// handshake matching, Galerkin products, dense coarse LU up to 64 rows, all
// bit-identical to the reference's setup).  Then:
//   - default smoothers (Jacobi with preSweeps_/postSweeps_ and
//     jacobiWeight_): apply is the library's cycle, recorded once into a
//     CUDA graph with fused smoothing, residual, transfer and coarse-solve
//     kernels (tf_amg_apply);
//   - a SmootherFactory: the smoothers are the caller's components, one per
//     pre- and post-smoothing stage of every level above the coarsest (a
//     stage with zero sweeps is skipped), set up on that level's operator;
//     apply then walks multigrid::executeCycle on the host over the same
//     hierarchy and the library's transfer, residual and coarse kernels.
// The coarse solve is the pivoted LU when the last level has <= 64 rows and
// is not singular, else coarseSweeps_ Jacobi sweeps (never from the
// factory).  apply starts from zero, may alias rhs and x, and keeps x's
// address and memory type.
//
// Extensions (no reference counterpart): singleHierarchy_ stores the
// hierarchy and runs the cycle in FP32 under a double preconditioner (the
// mixed-precision mode); smallLevelRows_ sets the size below which levels
// run as one shared-memory launch.
#pragma once

#include <Multigrid/Cycle.cuh>
#include <Multigrid/GpuAggregation.cuh>
#include <Smoother/Jacobi.cuh>

#include <array>
#include <functional>
#include <string>
#include <vector>

namespace thermofem {

template <linalg::Scalar T>
struct AmgOptions {
    int maxLevels_{20};         ///< 1..20
    int coarseRows_{64};        ///< stop coarsening at this many rows, 1..64
    int matchingRounds_{8};     ///< handshake rounds per matching stage, 1..8
    int preSweeps_{1}, postSweeps_{1};
    int coarseSweeps_{8};       ///< Jacobi sweeps when the coarse LU is not used
    T jacobiWeight_{T(0.75)};
    T strengthThreshold_{T(0.25)};
    bool absorbSingletons_{true};
    bool compactSortKeys_{false};
    multigrid::Cycle cycle_{multigrid::Cycle::V};
    bool singleHierarchy_{false};  ///< extension: FP32 hierarchy and cycle for T = double
    int smallLevelRows_{1200};     ///< extension: shared-memory region for levels up to this size
};

struct AmgLevelStatistics {
    std::size_t rows_{}, nonzeros_{};
    std::array<int, 4> aggregateSizes_{};
};

namespace b200 {
template <linalg::Scalar T, CsrIndex I>
class KrylovEngine;
}

template <linalg::Scalar T, CsrIndex I = int>
class Amg final : public Preconditioner<T, I> {
  public:
    using SmootherFactory = std::function<std::unique_ptr<Smoother<T, I>>()>;

    explicit Amg(AmgOptions<T> options = {}, SmootherFactory factory = {})
        : options_(options), factory_(std::move(factory)) {
        const auto &o = options;
        const bool cycleKnown =
            o.cycle_ == multigrid::Cycle::V || o.cycle_ == multigrid::Cycle::W || o.cycle_ == multigrid::Cycle::F;
        if (o.maxLevels_ < 1 || o.maxLevels_ > 20 || o.coarseRows_ < 1 || o.coarseRows_ > 64 ||
            o.matchingRounds_ < 1 || o.matchingRounds_ > 8 || o.preSweeps_ < 0 || o.postSweeps_ < 0 ||
            o.coarseSweeps_ < 1 || !std::isfinite(o.strengthThreshold_) || o.strengthThreshold_ < 0 ||
            o.strengthThreshold_ > 1 || !std::isfinite(o.jacobiWeight_) || o.jacobiWeight_ <= 0 ||
            o.jacobiWeight_ >= 2 || !cycleKnown || o.smallLevelRows_ < 0)
            throw std::invalid_argument("Invalid AMG options");
    }

    void setup(const CsrMatrix<T, I> &matrix) override {
        iteration::validateMatrix(matrix);
        const int device = matrix.rowOffsets().deviceId();
        linalg::detail::OperationScope scope(device);
        auto next = std::make_unique<State>(device);
        CsrMatrix<T, I> global;
        const CsrMatrix<T, I> *m = &matrix;
        if (matrix.memoryType() != MemoryType::Global) {
            global = matrix;
            global.changeMemoryType(GlobalMemory{});
            m = &global;
        }
        const tf_csr view = b200::describe(*m);
        tf_amg_options o = libraryOptions();
        b200::onContext(next->ctx, [&] {
            tf_amg *h = nullptr;
            b200::check(tf_amg_create(next->ctx.get(), b200::valueType<T>(), b200::indexType<I>(), &o, &h));
            next->owned.reset(h);
            b200::check(tf_amg_setup(h, &view));
        });
        next->hierarchy = next->owned.get();
        next->readDiagnostics();
        if (factory_) buildLevels(*next);
        state_ = std::move(next);
    }

    void apply(const Vector<T> &rhs, Vector<T> &x) override {
        if (!state_) throw std::logic_error("AMG requires setup");
        State &s = *state_;
        iteration::validateVectors(s.rows(), s.ctx.device(), rhs, x);
        linalg::detail::OperationScope scope(s.ctx.device());
        if (s.levels.empty()) {
            b200::DeviceSide<T> in(rhs, true), out(x, false);
            b200::onContext(s.ctx, [&] { b200::check(tf_amg_apply(s.hierarchy, in.get(), out.get())); });
            out.writeBack(x);
            s.readVisits();
            return;
        }
        s.levels.front().rhs.copyDataFrom(rhs);
        std::fill(s.visits.begin(), s.visits.end(), 0);
        HostCycle walk{s, options_};
        multigrid::executeCycle(options_.cycle_, 0, walk, true);
        s.ctx.synchronize();
        x.copyDataFrom(s.levels.front().x);
    }

    std::size_t levelCount() const noexcept { return state_ ? state_->statistics.size() : 0; }
    const std::vector<AmgLevelStatistics> &levelStatistics() const { return state().statistics; }
    const std::string &stopReason() const { return state().stopReason; }
    const std::string &coarseSolver() const { return state().coarseSolver; }
    const std::vector<std::size_t> &lastCycleVisits() const { return state().visits; }

  private:
    // the solvers' engine builds this hierarchy inside a fused solve and hands it over
    friend class b200::KrylovEngine<T, I>;

    struct ReleaseAmg {
        void operator()(tf_amg *a) const noexcept { tf_amg_destroy(a); }
    };

    // One level of the host-driven cycle (factory smoothers only).
    struct Level {
        CsrMatrix<T, I> matrix;
        tf_csr view{};
        Vector<T> rhs, x, residual;
        std::unique_ptr<Smoother<T, I>> pre, post;
        const int32_t *map{nullptr}, *offsets{nullptr}, *members{nullptr};
        int coarseRows{0};
    };

    struct State {
        b200::Context ctx;
        std::unique_ptr<tf_amg, ReleaseAmg> owned;
        tf_amg *hierarchy{nullptr};  // owned, or the hierarchy of the solver that holds this preconditioner
        std::vector<AmgLevelStatistics> statistics;
        std::vector<std::size_t> visits;
        std::string stopReason, coarseSolver;
        std::vector<Level> levels;  // factory path
        int luRows{0};
        const double *lu{nullptr};
        const int32_t *pivots{nullptr};
        std::unique_ptr<Jacobi<T, I>> fallback;

        explicit State(int device) : ctx(device) {}
        std::size_t rows() const { return statistics.empty() ? 0 : statistics.front().rows_; }

        void readDiagnostics() {
            const int n = tf_amg_level_count(hierarchy);
            statistics.assign(static_cast<std::size_t>(n), {});
            for (int d = 0; d < n; ++d) {
                int64_t rows = 0, nnz = 0;
                int32_t hist[4] = {};
                b200::check(tf_amg_level_stats(hierarchy, d, &rows, &nnz, hist));
                auto &st = statistics[static_cast<std::size_t>(d)];
                st.rows_ = static_cast<std::size_t>(rows);
                st.nonzeros_ = static_cast<std::size_t>(nnz);
                for (int k = 0; k < 4; ++k) st.aggregateSizes_[static_cast<std::size_t>(k)] = hist[k];
            }
            stopReason = tf_amg_stop_reason(hierarchy);
            coarseSolver = tf_amg_coarse_solver(hierarchy);
            visits.assign(static_cast<std::size_t>(n), 0);
        }
        void readVisits() {
            std::vector<int64_t> v(visits.size());
            if (!v.empty()) b200::check(tf_amg_last_visits(hierarchy, v.data(), static_cast<int>(v.size())));
            for (std::size_t d = 0; d < v.size(); ++d) visits[d] = static_cast<std::size_t>(v[d]);
        }
    };

    // The cycle's steps for executeCycle, on the level vectors of the factory
    // path.  Library kernels go to the context stream; a user smoother orders
    // itself after the legacy default stream, so the context stream is
    // drained before each smoother call.
    struct HostCycle {
        State &s;
        const AmgOptions<T> &o;
        tf_ctx *c() const { return s.ctx.get(); }
        Level &at(std::size_t d) { return s.levels[d]; }
        bool isCoarsest(std::size_t d) const { return d + 1 == s.levels.size(); }
        void begin(std::size_t d) { ++s.visits[d]; }
        void clear(std::size_t d) {
            auto &x = at(d).x;
            thermofem::detail::cudaCall(cudaMemsetAsync(x.data(), 0, x.sizeBytes(), s.ctx.stream()), "cudaMemsetAsync");
        }
        void coarseSolve(std::size_t d) {
            Level &l = at(d);
            if (s.luRows) {
                b200::check(tf_coarse_lu_solve(c(), s.luRows, s.lu, s.pivots, b200::valueType<T>(), l.rhs.data(),
                                               l.x.data()));
            } else {
                s.ctx.synchronize();
                s.fallback->apply(l.rhs, l.x);
            }
        }
        void smooth(Smoother<T, I> *sm, std::size_t d) {
            if (!sm) return;
            s.ctx.synchronize();
            sm->apply(at(d).rhs, at(d).x);
        }
        void preSmooth(std::size_t d) { smooth(at(d).pre.get(), d); }
        void postSmooth(std::size_t d) { smooth(at(d).post.get(), d); }
        void restrictVector(std::size_t d, const Vector<T> &fine) {
            Level &l = at(d);
            b200::check(tf_restrict(c(), b200::valueType<T>(), l.coarseRows, l.offsets, l.members, fine.data(),
                                    at(d + 1).rhs.data()));
        }
        void restrictRhs(std::size_t d) { restrictVector(d, at(d).rhs); }
        void restrictResidual(std::size_t d) {
            Level &l = at(d);
            b200::check(tf_residual(c(), &l.view, l.rhs.data(), l.x.data(), l.residual.data()));
            restrictVector(d, l.residual);
        }
        void prolong(std::size_t d) {
            Level &l = at(d);
            b200::check(tf_prolong(c(), b200::valueType<T>(), static_cast<int64_t>(l.x.size()), l.map,
                                   at(d + 1).x.data(), l.x.data()));
        }
    };

    tf_amg_options libraryOptions() const {
        tf_amg_options o;
        tf_amg_options_default(&o);
        o.max_levels = options_.maxLevels_;
        o.coarse_rows = options_.coarseRows_;
        o.matching_rounds = options_.matchingRounds_;
        o.pre_sweeps = options_.preSweeps_;
        o.post_sweeps = options_.postSweeps_;
        o.coarse_sweeps = options_.coarseSweeps_;
        o.jacobi_weight = static_cast<double>(options_.jacobiWeight_);
        o.strength_threshold = static_cast<double>(options_.strengthThreshold_);
        o.absorb_singletons = options_.absorbSingletons_ ? 1 : 0;
        o.compact_sort_keys = options_.compactSortKeys_ ? 1 : 0;
        o.cycle = options_.cycle_ == multigrid::Cycle::W ? TF_CYCLE_W
                  : options_.cycle_ == multigrid::Cycle::F ? TF_CYCLE_F
                                                            : TF_CYCLE_V;
        o.hierarchy_type = (options_.singleHierarchy_ && !factory_) ? TF_F32 : -1;
        o.coarse_lu_rows = 64;
        o.small_level_rows = options_.smallLevelRows_;
        o.damping_model = nullptr;
        return o;
    }

    // The factory path: typed copies of the level operators, the caller's
    // smoothers on them, the level vectors, the transfers and the coarse solve.
    void buildLevels(State &s) {
        const std::size_t L = s.statistics.size();
        s.levels.resize(L);
        for (std::size_t d = 0; d < L; ++d) {
            Level &l = s.levels[d];
            tf_csr v{};
            b200::check(tf_amg_level_matrix(s.hierarchy, static_cast<int>(d), &v));
            l.matrix = typedCopy(v, s.ctx);
            l.view = b200::describe(l.matrix);
            const std::size_t n = l.matrix.rowCount();
            l.rhs = Vector<T>(n);
            l.x = Vector<T>(n);
            l.residual = Vector<T>(n);
            if (d + 1 < L) {
                b200::check(tf_amg_level_transfer(s.hierarchy, static_cast<int>(d), &l.map, &l.offsets, &l.members,
                                                  &l.coarseRows));
                if (options_.preSweeps_) l.pre = makeSmoother(l.matrix);
                if (options_.postSweeps_) l.post = makeSmoother(l.matrix);
            }
        }
        const double *lu = nullptr;
        const int32_t *piv = nullptr;
        b200::check(tf_amg_coarse_factor(s.hierarchy, &s.luRows, &lu, &piv));
        s.lu = lu;
        s.pivots = piv;
        if (!s.luRows) {
            s.fallback = std::make_unique<Jacobi<T, I>>(options_.coarseSweeps_, options_.jacobiWeight_);
            s.fallback->setup(s.levels.back().matrix);
        }
    }

    std::unique_ptr<Smoother<T, I>> makeSmoother(const CsrMatrix<T, I> &a) {
        auto sm = factory_();
        if (!sm) throw std::invalid_argument("AMG smoother factory returned null");
        sm->setup(a);
        return sm;
    }

    // A level operator (the hierarchy's storage: T values, int32 indices) as
    // a CsrMatrix<T, I> of its own buffers.
    static CsrMatrix<T, I> typedCopy(const tf_csr &v, b200::Context &ctx) {
        const std::size_t n = static_cast<std::size_t>(v.rows), nnz = static_cast<std::size_t>(v.nnz);
        CudaBuffer<I> rp(n + 1), ci(nnz);
        CudaBuffer<T> val(nnz);
        b200::onContext(ctx, [&] {
            auto indices = [&](CudaBuffer<I> &dst, const void *src, std::size_t count) {
                if (!count) return;
                if constexpr (sizeof(I) == 4)
                    thermofem::detail::cudaCall(cudaMemcpyAsync(dst.data(), src, count * 4, cudaMemcpyDeviceToDevice,
                                                                ctx.stream()),
                                                "cudaMemcpyAsync");
                else
                    b200::check(tf_convert(ctx.get(), static_cast<int64_t>(count), TF_I32, src, TF_I64, dst.data()));
            };
            indices(rp, v.offsets, n + 1);
            indices(ci, v.indices, nnz);
            if (nnz)
                b200::check(tf_convert(ctx.get(), static_cast<int64_t>(nnz), v.value_type, v.values,
                                       b200::valueType<T>(), val.data()));
        });
        return CsrMatrix<T, I>::fromBuffers(n, n, std::move(rp), std::move(ci), std::move(val));
    }

    // A fused solver built this preconditioner's hierarchy inside its own
    // solve (tf_solver with the AMG preconditioner): the diagnostics and
    // apply use that hierarchy, owned by the solver.
    void adopt(tf_amg *solverHierarchy, int device) {
        auto next = std::make_unique<State>(device);
        next->hierarchy = solverHierarchy;
        next->readDiagnostics();
        state_ = std::move(next);
    }
    void forget() noexcept { state_.reset(); }
    bool runsInLibrary() const noexcept { return !factory_; }
    const AmgOptions<T> &options() const noexcept { return options_; }

    const State &state() const {
        if (!state_) throw std::logic_error("AMG requires setup");
        return *state_;
    }

    AmgOptions<T> options_;
    SmootherFactory factory_;
    std::unique_ptr<State> state_;
};

}  // namespace thermofem
