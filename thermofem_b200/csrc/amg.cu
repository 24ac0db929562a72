// amg.cu -- aggregation AMG hierarchy and its V/W/F cycle.
//
// Setup follows Amg::setup (include/Preconditioner/Amg.cuh:81-143) stage by
// stage on the device: canonical native FP64/int32 operator, per-level
// validation, strength graph, two-stage matching with absorption, Galerkin
// coarse operator, and the stop rules (coarse size, level limit, empty
// strength graph, no contraction).  The last level is factored by the
// pivoted dense LU when small enough, otherwise fixed-sweep Jacobi is the
// coarse solver, exactly as the reference chooses.
//
// The cycle follows executeCycle (include/Multigrid/Cycle.cuh:35-63) with
// the reference's clear/visit semantics, but every level step is a fused
// kernel: a pre-smooth from a zero guess is x = w Dinv b (no SpMV), the
// residual is one pass, and the first post-smooth sweep reads x + P e on the
// fly instead of running a separate prolongation.  The whole cycle is
// captured once into a CUDA graph and replayed on every apply.
#include <algorithm>
#include <cstring>
#include <istream>
#include <ostream>
#include <vector>

#include "coarse_cycle.cuh"
#include "engine.cuh"
#include "mlp.cuh"

namespace tfb {

AmgConfig::AmgConfig(const tf_amg_options &opt) : o(opt) {
    const auto &p = opt;
    if (p.max_levels < 1 || p.max_levels > 20 || p.coarse_rows < 1 || p.coarse_rows > 256 || p.matching_rounds < 1 ||
        p.matching_rounds > 8 || p.pre_sweeps < 0 || p.post_sweeps < 0 || p.coarse_sweeps < 1 ||
        !std::isfinite(p.strength_threshold) || p.strength_threshold < 0 || p.strength_threshold > 1 ||
        !std::isfinite(p.jacobi_weight) || p.jacobi_weight <= 0 || p.jacobi_weight >= 2 ||
        (p.cycle != TF_CYCLE_V && p.cycle != TF_CYCLE_W && p.cycle != TF_CYCLE_F) ||
        (p.hierarchy_type != -1 && p.hierarchy_type != TF_F32 && p.hierarchy_type != TF_F64 &&
         p.hierarchy_type != TF_F32_VALUES) ||
        p.coarse_lu_rows < 1 || p.coarse_lu_rows > 256 || p.small_level_rows < 0)
        fail(TF_ERR_INVALID, "Invalid AMG options");
    model = damping_model_of(p.damping_model);
}

std::unique_ptr<tf_dcsr> to_native(tf_ctx *ctx, const tf_csr &a) {
    check_csr(&a);
    require(a.rows > 0 && a.rows == a.cols && a.rows < INT32_MAX, "Solver requires a nonempty square matrix");
    if (a.nnz > INT32_MAX / 2) fail(TF_ERR_LENGTH, "AMG native index capacity exceeded");
    auto m = std::make_unique<tf_dcsr>();
    m->rows = m->cols = a.rows;
    m->nnz = a.nnz;
    m->offsets.allocate(static_cast<size_t>(a.rows + 1) * 4);
    m->indices.allocate(static_cast<size_t>(a.nnz) * 4);
    m->values.allocate(static_cast<size_t>(a.nnz) * 8);
    auto *rp = reinterpret_cast<int32_t *>(m->offsets.data());
    auto *ci = reinterpret_cast<int32_t *>(m->indices.data());
    auto *v = reinterpret_cast<double *>(m->values.data());
    if (a.index_type == TF_I32) {
        convert(ctx, a.rows + 1, static_cast<const int32_t *>(a.offsets), rp);
        convert(ctx, a.nnz, static_cast<const int32_t *>(a.indices), ci);
    } else {
        convert(ctx, a.rows + 1, static_cast<const int64_t *>(a.offsets), rp);
        convert(ctx, a.nnz, static_cast<const int64_t *>(a.indices), ci);
    }
    if (a.value_type == TF_F64) convert(ctx, a.nnz, static_cast<const double *>(a.values), v);
    else convert(ctx, a.nnz, static_cast<const float *>(a.values), v);
    const int flags = csr_canonical_flags(ctx, csr_of(*m));
    if (flags & 2) fail(TF_ERR_INVALID, "AMG invalid CSR or nonfinite coefficient");
    if (flags == 0) return m;
    return canonicalize(ctx, csr_of(*m));
}

const std::vector<std::string> &setup_phase_names() {
    static const std::vector<std::string> names = {
        "level copies and diagonals",  // validation, storage copies, inverse diagonal, learned damping
        "column and sliced copies",
        "SpMV shape tuning",
        "strength graphs",
        "aggregation",
        "Galerkin products",
        "coarse LU",
        "small-level region",
        "layout selection"};
    return names;
}

namespace {

enum SetupPhase { kPhLevel, kPhColumns, kPhTuning, kPhStrength, kPhAggregate, kPhGalerkin, kPhCoarse, kPhSmall,
                  kPhLayouts, kPhEnd };

// Events recorded on the context stream where a setup phase starts; the
// span to the next event is charged to the phase.
class PhaseMarks {
  public:
    ~PhaseMarks() {
        for (auto &m : marks_) cudaEventDestroy(m.second);
    }
    void mark(tf_ctx *ctx, int phase) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess || cudaEventRecord(e, ctx->stream) != cudaSuccess) {
            if (e) cudaEventDestroy(e);
            cudaGetLastError();
            return;
        }
        marks_.emplace_back(phase, e);
    }
    // after the stream has drained
    std::vector<double> totals() const {
        std::vector<double> ms(kPhEnd, 0.0);
        for (size_t i = 0; i + 1 < marks_.size(); ++i) {
            float t = 0;
            if (marks_[i].first < kPhEnd && cudaEventElapsedTime(&t, marks_[i].second, marks_[i + 1].second) == cudaSuccess)
                ms[marks_[i].first] += t;
        }
        cudaGetLastError();
        return ms;
    }

  private:
    std::vector<std::pair<int, cudaEvent_t>> marks_;
};

// Checkpoint streams: sized arrays, device arrays staged through host
// memory on the context stream; a short or failed stream is an error.
struct Writer {
    tf_ctx *ctx;
    std::ostream &out;
    void bytes(const void *p, size_t n) {
        out.write(static_cast<const char *>(p), static_cast<std::streamsize>(n));
        if (!out) fail(TF_ERR_RUNTIME, "AMG checkpoint: write failed");
    }
    template <class P>
    void pod(const P &v) {
        bytes(&v, sizeof v);
    }
    void str(const std::string &v) {
        pod(static_cast<int32_t>(v.size()));
        bytes(v.data(), v.size());
    }
    void device(const void *d, int64_t n) {
        std::vector<char> h(static_cast<size_t>(n));
        if (n) {
            cuda_check(cudaMemcpyAsync(h.data(), d, static_cast<size_t>(n), cudaMemcpyDeviceToHost, ctx->stream),
                       "AMG checkpoint");
            cuda_check(cudaStreamSynchronize(ctx->stream), "AMG checkpoint");
        }
        pod(n);
        bytes(h.data(), h.size());
    }
};
struct Reader {
    tf_ctx *ctx;
    std::istream &in;
    void bytes(void *p, size_t n) {
        in.read(static_cast<char *>(p), static_cast<std::streamsize>(n));
        if (!in || static_cast<size_t>(in.gcount()) != n) fail(TF_ERR_INVALID, "AMG checkpoint: file truncated or unreadable");
    }
    template <class P>
    P pod() {
        P v{};
        bytes(&v, sizeof v);
        return v;
    }
    std::string str() {
        const int32_t n = pod<int32_t>();
        if (n < 0 || n > 256) fail(TF_ERR_INVALID, "AMG checkpoint: bad string");
        std::string v(static_cast<size_t>(n), '\0');
        bytes(v.data(), v.size());
        return v;
    }
    void device(void *d, int64_t n) {
        if (pod<int64_t>() != n) fail(TF_ERR_INVALID, "AMG checkpoint: array size does not match its level");
        std::vector<char> h(static_cast<size_t>(n));
        bytes(h.data(), h.size());
        if (n) {
            cuda_check(cudaMemcpyAsync(d, h.data(), static_cast<size_t>(n), cudaMemcpyHostToDevice, ctx->stream),
                       "AMG checkpoint");
            cuda_check(cudaStreamSynchronize(ctx->stream), "AMG checkpoint");
        }
    }
};

template <class S, class V = S>
struct Level {
    int64_t n{0}, nnz{0};
    DeviceBuffer<int32_t> rp, ci;
    DeviceBuffer<V> val;  // values, stored in V (FP32 under an FP64 cycle, or S)
    DeviceBuffer<S> val_s;  // V != S: the values widened to S, for the small-level region only
    DeviceBuffer<S> dinv, rhs, x0, x1, r;
    DeviceBuffer<int32_t> map, off, mem;
    DeviceBuffer<int16_t> cd;  // columns as row offsets, when they fit
    SlicedCopy<V> sl;          // sliced copy for the SpMV family, when built
    bool sliced_on{true};      // the cycle streams sl (chosen at setup, select_layouts)
    int coarse{0};
    int cur{0};
    S *x() const { return cur ? x1.data() : x0.data(); }
    S *other() const { return cur ? x0.data() : x1.data(); }
    Csr<S, int32_t, V> csr() const {
        Csr<S, int32_t, V> c;
        c.rows = c.cols = n;
        c.nnz = nnz;
        c.rp = rp.data();
        c.ci = ci.data();
        c.val = val.data();
        c.cd = cd.data();
        if (sliced_on) sl.attach(c);
        return c;
    }
    // Values and structure alone, in V (what the copy builders read).
    Csr<V, int32_t> values() const {
        Csr<V, int32_t> c;
        c.rows = c.cols = n;
        c.nnz = nnz;
        c.rp = rp.data();
        c.ci = ci.data();
        c.val = val.data();
        c.cd = cd.data();
        return c;
    }
};

// S: the cycle's vectors and arithmetic; V: how the level operators' values
// are stored (V = S, or FP32 values under an FP64 cycle).
template <class S, class V = S>
class HierarchyImpl final : public Hierarchy {
  public:
    HierarchyImpl(const AmgConfig &cfg) : cfg_(cfg), w_(static_cast<S>(cfg.model ? 1.0 : cfg.o.jacobi_weight)) {
        // THERMOFEM_B200_FUSE: 0 launches every transfer on its own, 1 fuses
        // restrictions everywhere and prolongations into fine levels of at
        // most kScatterRows rows, 2 fuses every prolongation.
        const char *f = std::getenv("THERMOFEM_B200_FUSE");
        fuse_ = f ? std::atoi(f) : 1;
    }
    ~HierarchyImpl() override {
        if (exec_) cudaGraphExecDestroy(exec_);
    }

    void build(tf_ctx *ctx, const tf_dcsr &fine) {
        const auto &o = cfg_.o;
        PhaseMarks marks;
        // The native operator of the current level; level 0 borrows `fine`.
        std::unique_ptr<tf_dcsr> owned;
        const tf_dcsr *native = &fine;
        DeviceBuffer<double> row_max;
        for (int depth = 0;; ++depth) {
            marks.mark(ctx, kPhLevel);
            const auto nc = csr_of(*native);
            row_max.allocate(static_cast<size_t>(nc.rows));
            if (!row_stats(ctx, nc, row_max.data()))
                fail(TF_ERR_INVALID, "Native AMG: missing/zero diagonal, non-finite value or reciprocal in hierarchy");
            levels_.emplace_back();
            Level<S, V> &l = levels_.back();
            l.n = nc.rows;
            l.nnz = nc.nnz;
            l.rp.allocate(static_cast<size_t>(l.n) + 1);
            l.ci.allocate(static_cast<size_t>(l.nnz));
            l.val.allocate(static_cast<size_t>(l.nnz));
            copy_async(ctx, l.rp.data(), nc.rp, (l.n + 1) * sizeof(int32_t));
            copy_async(ctx, l.ci.data(), nc.ci, l.nnz * sizeof(int32_t));
            convert(ctx, l.nnz, nc.val, l.val.data());
            for (auto *b : {&l.dinv, &l.rhs, &l.x0, &l.x1, &l.r}) b->allocate(static_cast<size_t>(l.n));
            // The diagonal must also invert in the iteration precision.
            inverse_diagonal(ctx, l.csr(), l.dinv.data());
            // learned damping: dinv_i scaled by omega_i, sweeps with weight 1
            if constexpr (std::is_same_v<S, V>) {
                if (cfg_.model) learned_damping(ctx, *cfg_.model, l.csr(), depth, l.dinv.data());
            }
            marks.mark(ctx, kPhColumns);
            column_copies(ctx, l);
            marks.mark(ctx, kPhTuning);
            tune_level(ctx, l);
            LevelStats st;
            st.rows = l.n;
            st.nnz = l.nnz;
            stats.push_back(st);
            if (l.n <= o.coarse_rows) {
                stop_reason = "coarse size";
                break;
            }
            if (depth + 1 == o.max_levels) {
                stop_reason = "level limit";
                break;
            }
            marks.mark(ctx, kPhStrength);
            auto graph = strength_graph(ctx, nc, row_max.data(), o.strength_threshold);
            if (graph->nnz == 0) {
                stop_reason = "empty strength graph";
                break;
            }
            marks.mark(ctx, kPhAggregate);
            auto t = aggregate(ctx, csr_of(*graph), o.matching_rounds, o.absorb_singletons != 0);
            if (t->coarse_rows >= t->fine_rows) {
                stop_reason = "no contraction";
                break;
            }
            marks.mark(ctx, kPhGalerkin);
            auto coarse = galerkin(ctx, nc, t->map.data(), t->coarse_rows);
            for (int k = 0; k < 4; ++k) stats.back().histogram[k] = t->histogram[k];
            l.map = std::move(t->map);
            l.off = std::move(t->offsets);
            l.mem = std::move(t->members);
            l.coarse = t->coarse_rows;
            owned = std::move(coarse);
            native = owned.get();
        }
        marks.mark(ctx, kPhCoarse);
        const auto last = csr_of(*native);
        bool singular = false;
        if (last.rows <= o.coarse_lu_rows) {
            const int n = static_cast<int>(last.rows);
            lu_.allocate(static_cast<size_t>(n) * n);
            piv_.allocate(static_cast<size_t>(n));
            factored_ = coarse_lu_factor(ctx, last, lu_.data(), piv_.data());
            singular = !factored_;
            if (factored_) {
                inv_.allocate(static_cast<size_t>(n) * n);
                coarse_inverse(ctx, n, lu_.data(), piv_.data(), inv_.data());
            }
        }
        coarse_solver = factored_ ? "pivoted GPU LU" : (singular ? "Jacobi (singular LU)" : "Jacobi (coarsening stopped)");
        finish_setup(ctx, marks);
    }

    // The 2-byte column stream and the banded or sliced copy of a level
    // (derived from its structure and values alone).
    void column_copies(tf_ctx *ctx, Level<S, V> &l) {
        if (delta_columns_enabled() && l.nnz > 0) {
            l.cd.allocate(static_cast<size_t>(l.nnz));
            if (!delta_columns(ctx, l.n, l.rp.data(), l.ci.data(), l.cd.data())) l.cd.release();
        }
        if (sliced_enabled() && !(banded_enabled() && build_banded(ctx, l.values(), l.sl)) && l.cd.data())
            build_sliced(ctx, l.values(), l.sl, true);
    }
    // Launch shape of this level's row-tile kernels (cached by shape).
    void tune_level(tf_ctx *ctx, Level<S, V> &l) {
        fill_zero(ctx, l.n, l.rhs.data());
        tune_spmv(ctx, l.csr(), static_cast<const S *>(l.rhs.data()), l.r.data());
    }
    void finish_setup(tf_ctx *ctx, PhaseMarks &marks) {
        visits.assign(levels_.size(), 0);
        marks.mark(ctx, kPhSmall);
        plan_small_levels(ctx);
        marks.mark(ctx, kPhLayouts);
        select_layouts(ctx);
        marks.mark(ctx, kPhEnd);
        cuda_check(cudaStreamSynchronize(ctx->stream), "AMG setup");
        setup_ms = marks.totals();
    }

    // ---- checkpoint: the results of the setup phases that coarsen (each
    // level's operator in its storage, its damped inverse diagonal, the
    // aggregates, the coarse factor, the statistics) -- everything else is
    // derived again on restore by the code that derives it in build, so a
    // restored hierarchy applies with the same bits.
    static constexpr char kMagic[8] = {'T', 'F', 'B', 'A', 'M', 'G', '0', '1'};

    void save(tf_ctx *ctx, std::ostream &out) const override {
        Writer w{ctx, out};
        w.bytes(kMagic, sizeof kMagic);
        w.pod(static_cast<int32_t>(sizeof(S)));
        w.pod(static_cast<int32_t>(sizeof(V)));
        w.pod(static_cast<double>(w_));
        w.pod(static_cast<int32_t>(levels_.size()));
        w.str(stop_reason);
        w.str(coarse_solver);
        for (size_t d = 0; d < levels_.size(); ++d) {
            const Level<S, V> &l = levels_[d];
            const bool last = d + 1 == levels_.size();
            w.pod(l.n);
            w.pod(l.nnz);
            w.pod(static_cast<int32_t>(last ? 0 : l.coarse));
            w.bytes(stats[d].histogram, sizeof stats[d].histogram);
            w.device(l.rp.data(), (l.n + 1) * sizeof(int32_t));
            w.device(l.ci.data(), l.nnz * sizeof(int32_t));
            w.device(l.val.data(), l.nnz * sizeof(V));
            w.device(l.dinv.data(), l.n * sizeof(S));
            if (!last) {
                w.device(l.map.data(), l.n * sizeof(int32_t));
                w.device(l.off.data(), (static_cast<int64_t>(l.coarse) + 1) * sizeof(int32_t));
                w.device(l.mem.data(), l.n * sizeof(int32_t));
            }
        }
        const int32_t nlu = factored_ ? static_cast<int32_t>(levels_.back().n) : 0;
        w.pod(nlu);
        if (nlu) {
            w.device(lu_.data(), static_cast<size_t>(nlu) * nlu * sizeof(double));
            w.device(piv_.data(), static_cast<size_t>(nlu) * sizeof(int32_t));
            w.device(inv_.data(), static_cast<size_t>(nlu) * nlu * sizeof(double));
        }
        out.flush();
        if (!out) fail(TF_ERR_RUNTIME, "AMG checkpoint: write failed");
    }

    void restore(tf_ctx *ctx, std::istream &in) {
        PhaseMarks marks;
        Reader r{ctx, in};
        char magic[sizeof kMagic];
        r.bytes(magic, sizeof magic);
        if (std::memcmp(magic, kMagic, sizeof kMagic) != 0) fail(TF_ERR_INVALID, "AMG checkpoint: not a hierarchy file");
        const auto sv = r.pod<int32_t>(), vv = r.pod<int32_t>();
        if (sv != static_cast<int32_t>(sizeof(S)) || vv != static_cast<int32_t>(sizeof(V)))
            fail(TF_ERR_INVALID, "AMG checkpoint: the hierarchy type differs from this component's");
        if (r.pod<double>() != static_cast<double>(w_))
            fail(TF_ERR_INVALID, "AMG checkpoint: built with another Jacobi weight or damping model");
        const int32_t nl = r.pod<int32_t>();
        if (nl < 1 || nl > cfg_.o.max_levels) fail(TF_ERR_INVALID, "AMG checkpoint: bad level count");
        stop_reason = r.str();
        coarse_solver = r.str();
        for (int32_t d = 0; d < nl; ++d) {
            marks.mark(ctx, kPhLevel);
            const bool last = d + 1 == nl;
            levels_.emplace_back();
            Level<S, V> &l = levels_.back();
            l.n = r.pod<int64_t>();
            l.nnz = r.pod<int64_t>();
            l.coarse = r.pod<int32_t>();
            if (l.n < 1 || l.n >= INT32_MAX || l.nnz < 0 || l.nnz >= INT32_MAX || (!last && (l.coarse < 1 || l.coarse >= l.n)))
                fail(TF_ERR_INVALID, "AMG checkpoint: bad level sizes");
            if (d > 0 && l.n != levels_[d - 1].coarse) fail(TF_ERR_INVALID, "AMG checkpoint: levels do not chain");
            LevelStats st;
            st.rows = l.n;
            st.nnz = l.nnz;
            r.bytes(st.histogram, sizeof st.histogram);
            stats.push_back(st);
            l.rp.allocate(static_cast<size_t>(l.n) + 1);
            l.ci.allocate(static_cast<size_t>(l.nnz));
            l.val.allocate(static_cast<size_t>(l.nnz));
            for (auto *b : {&l.dinv, &l.rhs, &l.x0, &l.x1, &l.r}) b->allocate(static_cast<size_t>(l.n));
            r.device(l.rp.data(), (l.n + 1) * sizeof(int32_t));
            r.device(l.ci.data(), l.nnz * sizeof(int32_t));
            r.device(l.val.data(), l.nnz * sizeof(V));
            r.device(l.dinv.data(), l.n * sizeof(S));
            if (!last) {
                l.map.allocate(static_cast<size_t>(l.n));
                l.off.allocate(static_cast<size_t>(l.coarse) + 1);
                l.mem.allocate(static_cast<size_t>(l.n));
                r.device(l.map.data(), l.n * sizeof(int32_t));
                r.device(l.off.data(), (static_cast<int64_t>(l.coarse) + 1) * sizeof(int32_t));
                r.device(l.mem.data(), l.n * sizeof(int32_t));
            }
            // the operator's structure is checked as a caller's would be
            // (every later kernel trusts it), then its copies are derived
            if (!csr_structure_ok(ctx, l.n, l.n, l.nnz, l.rp.data(), l.ci.data()))
                fail(TF_ERR_INVALID, "AMG checkpoint: level operator structure is invalid");
            if (!last && indices_out_of_range(ctx, l.n, l.map.data(), l.coarse))
                fail(TF_ERR_INVALID, "AMG checkpoint: aggregate map entry out of range");
            marks.mark(ctx, kPhColumns);
            column_copies(ctx, l);
            marks.mark(ctx, kPhTuning);
            tune_level(ctx, l);
        }
        marks.mark(ctx, kPhCoarse);
        const int32_t nlu = r.pod<int32_t>();
        if (nlu) {
            if (nlu != levels_.back().n) fail(TF_ERR_INVALID, "AMG checkpoint: coarse factor size");
            lu_.allocate(static_cast<size_t>(nlu) * nlu);
            piv_.allocate(static_cast<size_t>(nlu));
            inv_.allocate(static_cast<size_t>(nlu) * nlu);
            r.device(lu_.data(), static_cast<size_t>(nlu) * nlu * sizeof(double));
            r.device(piv_.data(), static_cast<size_t>(nlu) * sizeof(int32_t));
            r.device(inv_.data(), static_cast<size_t>(nlu) * nlu * sizeof(double));
        }
        factored_ = nlu > 0;
        finish_setup(ctx, marks);
    }

    // Which levels the cycle streams through their sliced copy, decided in
    // the cycle itself: a kernel timed alone (tile::autotune) meets its
    // operator either cold or warm in L2, while inside a cycle a mid-size
    // level is partly resident and its neighbours' epilogues and
    // programmatic launch overlap change the balance.  For every launched
    // level with a sliced copy, finest first, the captured cycle is timed
    // (CUDA events, 2 warm-up and 8 timed replays, each after the L2 cache
    // is flushed) with the copy streamed and without, and the faster is kept.  Either choice gives the same
    // bits.  Skipped when THERMOFEM_B200_SLICED_SHAPE forces a shape or
    // THERMOFEM_B200_SLICED_SELECT=0.
    void select_layouts(tf_ctx *ctx) {
        if (std::getenv("THERMOFEM_B200_SLICED_SHAPE")) return;
        if (const char *v = std::getenv("THERMOFEM_B200_SLICED_SELECT"); v && v[0] == '0') return;
        std::vector<size_t> cand;
        // (levels under 16,384 rows are launch-latency bound: their layout is left as built)
        for (size_t d = 0; d < levels_.size() && d < coop_from_; ++d)
            if (levels_[d].sl.sp.data() && levels_[d].n >= 16384) cand.push_back(d);
        if (cand.empty()) return;
        StableScope stable(ctx);
        fill_zero(ctx, levels_.front().n, levels_.front().rhs.data());
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        // a solve runs its outer loop (an operator stream larger than the L2
        // cache) between cycles: every timed replay starts after a write of
        // more than the L2 size
        void *flush = ctx->arena(tile::kTuneFlushBytes, 1);
        auto time_cycle = [&](float *ms) {
            capture(ctx);
            if (!exec_) return false;
            bool ok = true;
            for (int r = 0; r < 2 && ok; ++r) ok = cudaGraphLaunch(exec_, ctx->stream) == cudaSuccess;
            *ms = 0;
            for (int r = 0; r < 8 && ok; ++r) {
                float t = 0;
                ok = cudaMemsetAsync(flush, r, tile::kTuneFlushBytes, ctx->stream) == cudaSuccess &&
                     cudaEventRecord(e0, ctx->stream) == cudaSuccess &&
                     cudaGraphLaunch(exec_, ctx->stream) == cudaSuccess &&
                     cudaEventRecord(e1, ctx->stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
                     cudaEventElapsedTime(&t, e0, e1) == cudaSuccess;
                *ms += t;
            }
            cudaGraphExecDestroy(exec_);
            exec_ = nullptr;
            return ok;
        };
        bool ok = true;
        for (size_t d : cand) {
            float on = 0, off = 0;
            levels_[d].sliced_on = true;
            ok = time_cycle(&on);
            levels_[d].sliced_on = false;
            ok = ok && time_cycle(&off);
            levels_[d].sliced_on = ok && on <= off;
            if (tile::tune_log())
                std::fprintf(stderr, "select_layouts level %zu rows=%lld cycle %.2f us sliced, %.2f us csr\n", d,
                             static_cast<long long>(levels_[d].n), on * 1e3f / 8, off * 1e3f / 8);
            if (!ok) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // the cycle graph of the first apply is captured with the kept layouts
        cudaGetLastError();
        capture_failed_ = false;
        for (auto &l : levels_) l.cur = 0;
        std::fill(visits.begin(), visits.end(), 0);
        check_faults(ctx);
    }

    void apply(tf_ctx *ctx, const double *rhs, double *x) override { apply_t(ctx, rhs, x); }
    void apply(tf_ctx *ctx, const float *rhs, float *x) override { apply_t(ctx, rhs, x); }
    int storage_type() const override { return std::is_same_v<S, double> ? TF_F64 : TF_F32; }
    int64_t rows() const override { return levels_.front().n; }
    int level_count() const override { return static_cast<int>(levels_.size()); }
    tf_csr level_matrix(int d) const override {
        const auto &l = levels_.at(static_cast<size_t>(d));
        const int vt = std::is_same_v<V, double> ? TF_F64 : TF_F32;
        tf_csr c{l.n, l.n, l.nnz, TF_I32, vt, l.rp.data(), l.ci.data(), l.val.data()};
        return c;
    }
    void level_spmv(tf_ctx *ctx, int d, const void *x, void *y) const override {
        const auto &l = levels_.at(static_cast<size_t>(d));
        StableScope stable(ctx);
        spmv(ctx, l.csr(), static_cast<const S *>(x), static_cast<S *>(y));
    }
    int level_spmv_layout(tf_ctx *ctx, int d, int64_t *entries) const override {
        const auto &l = levels_.at(static_cast<size_t>(d));
        if (!streams_sliced(ctx, l.csr(), l.sl.entries, entries)) return l.cd.data() ? 0 : 4;
        return l.sl.perm.data() ? 2 : (l.sl.banded() ? 3 : 1);
    }
    void level_transfer(int d, const int32_t **map, const int32_t **off, const int32_t **mem,
                        int *coarse) const override {
        const auto &l = levels_.at(static_cast<size_t>(d));
        *map = l.map.data();
        *off = l.off.data();
        *mem = l.mem.data();
        *coarse = l.coarse;
    }
    void coarse_factor(int *rows, const double **lu, const int32_t **pivots) const override {
        *rows = factored_ ? static_cast<int>(levels_.back().n) : 0;
        *lu = factored_ ? lu_.data() : nullptr;
        *pivots = factored_ ? piv_.data() : nullptr;
    }
    int64_t kernels_per_cycle() const override { return per_cycle_; }

  private:
    template <class T>
    void apply_t(tf_ctx *ctx, const T *rhs, T *x) {
        StableScope stable(ctx);  // level operators are read-only from here on
        Level<S, V> &f = levels_.front();
        convert(ctx, f.n, rhs, f.rhs.data());
        run_cycle(ctx);
        convert(ctx, f.n, levels_.front().x(), x);
    }
    const void *apply_open(tf_ctx *ctx, const double *rhs) override { return open_t(ctx, rhs); }
    const void *apply_open(tf_ctx *ctx, const float *rhs) override { return open_t(ctx, rhs); }
    template <class T>
    const void *open_t(tf_ctx *ctx, const T *rhs) {
        StableScope stable(ctx);
        Level<S, V> &f = levels_.front();
        cudaStreamCaptureStatus capturing;
        cuda_check(cudaStreamIsCapturing(ctx->stream, &capturing), "capture status");
        if (capturing != cudaStreamCaptureStatusNone && fuse_ > 0) {
            // inside the caller's capture the cycle is recorded inline (as
            // run_cycle does), so its first kernel may read rhs itself: the
            // conversion is held for the finest level's first op
            pin_ = {rhs, std::is_same_v<T, double>};
            enqueue(ctx);
            return levels_.front().x();
        }
        convert(ctx, f.n, rhs, f.rhs.data());
        run_cycle(ctx);
        return levels_.front().x();
    }

    void run_cycle(tf_ctx *ctx) {
        cudaStreamCaptureStatus capturing;
        cuda_check(cudaStreamIsCapturing(ctx->stream, &capturing), "capture status");
        if (capturing != cudaStreamCaptureStatusNone) {  // inside a caller's capture: record inline
            enqueue(ctx);
            return;
        }
        if (!exec_ && !capture_failed_) capture(ctx);
        if (exec_) {
            cuda_check(cudaGraphLaunch(exec_, ctx->stream), "cycle graph launch");
            ctx->launches += per_cycle_;
            for (size_t d = 0; d < levels_.size(); ++d) levels_[d].cur = final_cur_[d];
            visits = captured_visits_;
        } else {
            enqueue(ctx);
        }
    }

    void capture(tf_ctx *ctx) {
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            capture_failed_ = true;
            return;
        }
        const int64_t before = ctx->launches;
        cudaGraph_t graph = nullptr;
        try {
            enqueue(ctx);
        } catch (const Failure &) {
            // a step the driver cannot capture: run uncaptured from now on
            cudaStreamEndCapture(ctx->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            ctx->launches = before;
            capture_failed_ = true;
            return;
        }
        per_cycle_ = ctx->launches - before;
        ctx->launches = before;
        cuda_check(cudaStreamEndCapture(ctx->stream, &graph), "cycle capture");
        cudaError_t e = cudaGraphInstantiate(&exec_, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            exec_ = nullptr;
            capture_failed_ = true;
            return;
        }
        final_cur_.resize(levels_.size());
        for (size_t d = 0; d < levels_.size(); ++d) final_cur_[d] = levels_[d].cur;
        captured_visits_ = visits;
    }

    void enqueue(tf_ctx *ctx) {
        for (auto &l : levels_) l.cur = 0;
        std::fill(visits.begin(), visits.end(), 0);
        entry_ = 0;
        rec_.clear();
        pr_ = {};
        pw_ = {};
        cycle(ctx, cfg_.o.cycle, 0, true);
        if (!dry_) flush(ctx);
    }

    // ---- level operations: launched, or recorded as a small-level program step ----
    void op_jacobi_zero(tf_ctx *ctx, Level<S, V> &l) {
        if (recording_) {
            if (rec_.size() > region_start_) {
                CoarseStep<S> &prev = rec_.back();
                if ((prev.op == kStepResidualRestrict || prev.op == kStepRestrict) && prev.coarse_rhs == l.rhs.data() &&
                    !prev.cx) {
                    // the restriction's pass also does this zero-guess sweep
                    prev.cdinv = l.dinv.data();
                    prev.cx = l.x();
                    prev.cw = w_;
                    return;
                }
            }
            CoarseStep<S> s;
            s.op = kStepJacobiZero;
            s.n = static_cast<int>(l.n);
            s.w = w_;
            s.dinv = l.dinv.data();
            s.rhs = l.rhs.data();
            s.xout = l.x();
            rec_.push_back(s);
        } else if (!dry_) {
            if (fusing() && pin_.src && &l == &levels_.front()) {
                const PendingInput in = pin_;
                pin_ = {};
                if (in.f64)
                    jacobi_zero_convert(ctx, l.n, l.dinv.data(), static_cast<const double *>(in.src), l.rhs.data(),
                                        l.x(), w_);
                else
                    jacobi_zero_convert(ctx, l.n, l.dinv.data(), static_cast<const float *>(in.src), l.rhs.data(),
                                        l.x(), w_);
                return;
            }
            if (fusing() && pr_.coarse == &l) {
                restrict_jacobi_zero(ctx, l.n, pr_.fine->off.data(), pr_.fine->mem.data(), pr_.src, l.rhs.data(),
                                     l.dinv.data(), l.x(), w_);
                pr_ = {};
                return;
            }
            flush(ctx);
            jacobi_zero(ctx, l.n, l.dinv.data(), l.rhs.data(), l.x(), w_, nullptr);
        }
    }

    void op_zero(tf_ctx *ctx, Level<S, V> &l) {
        if (recording_) {
            CoarseStep<S> s;
            s.op = kStepZero;
            s.n = static_cast<int>(l.n);
            s.xout = l.x();
            rec_.push_back(s);
        } else if (!dry_) {
            flush(ctx);
            fill_zero(ctx, l.n, l.x());
        }
    }

    void sweep(tf_ctx *ctx, Level<S, V> &l, const int32_t *map = nullptr, const S *e = nullptr) {
        if (recording_) {
            CoarseStep<S> s;
            s.op = kStepSweep;
            s.n = static_cast<int>(l.n);
            s.w = w_;
            s.rp = l.rp.data();
            s.ci = l.ci.data();
            if constexpr (std::is_same_v<S, V>) s.val = l.val.data();
            s.dinv = l.dinv.data();
            s.rhs = l.rhs.data();
            s.xin = l.x();
            s.xout = l.other();
            s.map = map;
            s.e = e;
            rec_.push_back(s);
        } else if (!dry_) {
            flush(ctx);
            if (fusing() && !map) pw_ = {kWriteSweep, &l, l.x(), l.other(), {}};  // may take a prolongation
            else jacobi_sweep(ctx, l.csr(), l.dinv.data(), l.rhs.data(), l.x(), l.other(), w_, nullptr, map, e);
        }
        l.cur ^= 1;
    }

    void op_residual_restrict(tf_ctx *ctx, Level<S, V> &l, Level<S, V> &c) {
        if (recording_) {
            CoarseStep<S> s;
            s.op = kStepResidualRestrict;
            s.n = static_cast<int>(l.n);
            s.nc = l.coarse;
            s.rp = l.rp.data();
            s.ci = l.ci.data();
            if constexpr (std::is_same_v<S, V>) s.val = l.val.data();
            s.rhs = l.rhs.data();
            s.xin = l.x();
            s.off = l.off.data();
            s.mem = l.mem.data();
            s.coarse_rhs = c.rhs.data();
            rec_.push_back(s);
        } else if (!dry_) {
            flush(ctx);
            residual(ctx, l.csr(), l.rhs.data(), l.x(), l.r.data());
            if (fusing()) pr_ = {&l, &c, l.r.data()};  // taken by the coarse level's first op
            else restrict_sum(ctx, l.coarse, l.off.data(), l.mem.data(), l.r.data(), c.rhs.data());
        }
    }

    void op_restrict_rhs(tf_ctx *ctx, Level<S, V> &l, Level<S, V> &c) {
        if (recording_) {
            CoarseStep<S> s;
            s.op = kStepRestrict;
            s.nc = l.coarse;
            s.rhs = l.rhs.data();
            s.off = l.off.data();
            s.mem = l.mem.data();
            s.coarse_rhs = c.rhs.data();
            rec_.push_back(s);
        } else if (!dry_) {
            flush(ctx);
            if (fusing()) pr_ = {&l, &c, l.rhs.data()};
            else restrict_sum(ctx, l.coarse, l.off.data(), l.mem.data(), l.rhs.data(), c.rhs.data());
        }
    }

    void op_prolong(tf_ctx *ctx, Level<S, V> &l, Level<S, V> &c) {
        if (recording_) {
            CoarseStep<S> s;
            s.op = kStepProlong;
            s.n = static_cast<int>(l.n);
            s.xin = l.x();
            s.xout = l.x();
            s.map = l.map.data();
            s.e = c.x();
            rec_.push_back(s);
        } else if (!dry_) {
            if (prolong_fusable(l, c)) {
                launch_write(ctx, &l);
                return;
            }
            flush(ctx);
            prolong_add(ctx, l.n, l.map.data(), c.x(), l.x());
        }
    }

    void op_dense(tf_ctx *ctx, Level<S, V> &l) {
        if (recording_) {
            CoarseStep<S> s;
            s.op = kStepDense;
            s.n = static_cast<int>(l.n);
            s.inv = inv_.data();
            s.rhs = l.rhs.data();
            s.xout = l.x();
            rec_.push_back(s);
        } else if (!dry_) {
            if (fusing()) {
                // restriction into it (if pending) now, prolongation of it later
                const PendingRestrict r = pr_.coarse == &l ? pr_ : PendingRestrict{};
                if (r.coarse) pr_ = {};
                flush(ctx);
                pw_ = {kWriteDense, &l, nullptr, l.x(), r};
                return;
            }
            coarse_dense_apply(ctx, static_cast<int>(l.n), inv_.data(), l.rhs.data(), l.x());
        }
    }

    // ---- transfer fusion (launch path) ----
    // A restriction is held until the coarse level's first op, which takes it
    // in (restrict_jacobi_zero, dense); a sweep or dense solve is held until
    // the next op, which is its prolongation when fusable (jacobi_scatter,
    // dense with scatter).  Anything held is launched before any other op, so
    // the kernel order and every value are those of the unfused cycle.
    struct PendingRestrict {
        Level<S, V> *fine{nullptr}, *coarse{nullptr};
        const S *src{nullptr};
    };
    static constexpr int kWriteNone = 0, kWriteSweep = 1, kWriteDense = 2, kWriteProgram = 3;
    struct PendingWrite {
        int kind{kWriteNone};
        Level<S, V> *l{nullptr};
        const S *xin{nullptr};
        S *xout{nullptr};
        PendingRestrict r;
        // kWriteProgram: small-level region entry, its entry transfer and the
        // root buffer that holds its result
        int entry{0}, root_cur{0};
        ProgramIO<S> io;
    };

    bool fusing() const { return fuse_ > 0 && !recording_ && !dry_; }

    bool prolong_fusable(const Level<S, V> &l, const Level<S, V> &c) const {
        return fusing() && pw_.kind != kWriteNone && pw_.l == &c && pw_.xout == c.x() &&
               (fuse_ >= 2 || l.n <= kScatterRows);
    }

    // Launches the held write; with `fine` set, fused with the prolongation
    // of its result into fine->x().
    void launch_write(tf_ctx *ctx, Level<S, V> *fine) {
        const PendingWrite w = pw_;
        pw_ = {};
        const int32_t *off = fine ? fine->off.data() : nullptr;
        const int32_t *mem = fine ? fine->mem.data() : nullptr;
        S *fx = fine ? fine->x() : nullptr;
        Level<S, V> &l = *w.l;
        if (w.kind == kWriteProgram) {
            ProgramIO<S> io = w.io;
            io.soff = off;
            io.smem = mem;
            io.sfine = fx;
            tail_.launch(ctx, w.entry, io, w.root_cur);
            return;
        }
        if (w.kind == kWriteSweep) {
            if (fine)
                jacobi_sweep_scatter(ctx, l.csr(), l.dinv.data(), l.rhs.data(), w.xin, w.xout, w_, off, mem, fx);
            else
                jacobi_sweep(ctx, l.csr(), l.dinv.data(), l.rhs.data(), w.xin, w.xout, w_, nullptr, nullptr,
                             static_cast<const S *>(nullptr));
        } else if (w.kind == kWriteDense) {
            if (!fine && !w.r.coarse) {
                coarse_dense_apply(ctx, static_cast<int>(l.n), inv_.data(), l.rhs.data(), w.xout);
                return;
            }
            const S *rf = w.r.coarse ? w.r.src : nullptr;
            const int32_t *roff = w.r.coarse ? w.r.fine->off.data() : nullptr;
            const int32_t *rmem = w.r.coarse ? w.r.fine->mem.data() : nullptr;
            coarse_dense_apply_fused(ctx, static_cast<int>(l.n), inv_.data(), l.rhs.data(), w.xout, rf, roff, rmem,
                                     off, mem, fx);
        }
    }

    void flush(tf_ctx *ctx) {
        if (pin_.src) {
            const PendingInput in = pin_;
            pin_ = {};
            Level<S, V> &f = levels_.front();
            if (in.f64) convert(ctx, f.n, static_cast<const double *>(in.src), f.rhs.data());
            else convert(ctx, f.n, static_cast<const float *>(in.src), f.rhs.data());
        }
        if (pw_.kind != kWriteNone) launch_write(ctx, nullptr);
        if (pr_.coarse) {
            const PendingRestrict r = pr_;
            pr_ = {};
            restrict_sum(ctx, r.fine->coarse, r.fine->off.data(), r.fine->mem.data(), r.src, r.coarse->rhs.data());
        }
    }

    // `sweeps` Jacobi sweeps; cleared: x is the zero vector on entry.
    void smooth(tf_ctx *ctx, Level<S, V> &l, int sweeps, bool cleared) {
        int done = 0;
        if (cleared) {
            if (sweeps > 0) {
                op_jacobi_zero(ctx, l);
                done = 1;
            } else {
                op_zero(ctx, l);
            }
        }
        for (; done < sweeps; ++done) sweep(ctx, l);
    }

    // Entering the first small level starts a recorded sub-cycle that runs as
    // one cluster launch (its program was recorded by the setup dry run; the
    // recursion here replays the same steps to keep ping-pong state and visit
    // counts).  A restriction into the level that is still held goes into the
    // launch; the launch itself is held like a sweep, so that the
    // prolongation of its result can go into it too.
    void cycle(tf_ctx *ctx, int kind, size_t d, bool zero) {
        if (recording_ || d != coop_from_) return cycle_body(ctx, kind, d, zero);
        Level<S, V> &l = levels_[d];
        ProgramIO<S> io;
        if (!dry_ && fusing() && pr_.coarse == &l) {
            io.rsrc = pr_.src;
            io.roff = pr_.fine->off.data();
            io.rmem = pr_.fine->mem.data();
            io.rrhs = l.rhs.data();
            io.rn = static_cast<int>(l.n);
            pr_ = {};
        }
        if (!dry_) flush(ctx);
        recording_ = true;
        const size_t start = rec_.size();
        region_start_ = start;
        cycle_body(ctx, kind, d, zero);
        recording_ = false;
        if (dry_) {
            entries_.emplace_back(start, rec_.size() - start);
            return;
        }
        const CoarseStep<S> last = rec_.back();
        rec_.resize(start);
        PendingWrite w;
        w.kind = kWriteProgram;
        w.l = &l;
        w.entry = static_cast<int>(entry_++);
        w.root_cur = l.cur;
        w.io = io;
        if (fusing() && (last.op == kStepSweep || last.op == kStepDense) && last.xout == l.x()) {
            w.xout = l.x();
            pw_ = w;
        } else {
            pw_ = w;
            launch_write(ctx, nullptr);
        }
    }

    void cycle_body(tf_ctx *ctx, int kind, size_t d, bool zero) {
        Level<S, V> &l = levels_[d];
        ++visits[d];
        const bool cleared = zero || kind == TF_CYCLE_F;
        if (d + 1 == levels_.size()) {
            if (factored_) op_dense(ctx, l);
            else smooth(ctx, l, cfg_.o.coarse_sweeps, cleared);
            return;
        }
        Level<S, V> &c = levels_[d + 1];
        if (kind == TF_CYCLE_F) {
            op_restrict_rhs(ctx, l, c);
            cycle(ctx, TF_CYCLE_F, d + 1, true);
            op_zero(ctx, l);
            op_prolong(ctx, l, c);
            cycle(ctx, TF_CYCLE_V, d, false);
            return;
        }
        smooth(ctx, l, cfg_.o.pre_sweeps, cleared);
        op_residual_restrict(ctx, l, c);
        cycle(ctx, kind, d + 1, true);
        if (kind == TF_CYCLE_W) cycle(ctx, kind, d + 1, false);
        const int post = cfg_.o.post_sweeps;
        if (prolong_fusable(l, c)) {
            // x += P e fused into the coarse level's last kernel
            op_prolong(ctx, l, c);
            smooth(ctx, l, post, false);
        } else if (post > 0 && l.n <= kFusedProlongRows) {
            // small level: x + P e read on the fly by the first sweep
            sweep(ctx, l, l.map.data(), c.x());
            smooth(ctx, l, post - 1, false);
        } else {
            // large level: a streaming x += P e pass keeps the sweep's x
            // gathers single-hop (x~_j = x_j + e[map_j] costs two dependent
            // loads per nonzero)
            op_prolong(ctx, l, c);
            smooth(ctx, l, post, false);
        }
    }

    // The small-level region: the first level (below the finest) with at
    // most small_level_rows rows, or the first one below it whose levels fit
    // in the cluster's shared memory.  Its sub-cycles are recorded by a dry
    // run of the cycle (nothing is launched) and translated into region
    // steps; without a fitting region every level is launched.
    void plan_small_levels(tf_ctx *ctx) {
        const size_t none = levels_.size();
        coop_from_ = none;
        if (cfg_.o.small_level_rows <= 0) return;
        {
        size_t root = none;
        for (size_t d = 1; d < levels_.size(); ++d)
            if (levels_[d].n <= cfg_.o.small_level_rows) {
                root = d;
                break;
            }
        for (; root < levels_.size(); ++root) {
            // record this root's sub-cycles first: their length sizes the plan
            coop_from_ = root;
            entries_.clear();
            dry_ = true;
            enqueue(ctx);
            dry_ = false;
            size_t max_steps = 1;
            for (const auto &e : entries_) max_steps = std::max(max_steps, e.second);
            std::vector<TailLevel<S>> tl;
            for (size_t d = root; d < levels_.size(); ++d) {
                const Level<S, V> &l = levels_[d];
                TailLevel<S> t;
                t.n = l.n;
                t.rp = l.rp.data();
                t.ci = l.ci.data();
                t.cd = l.cd.data();
                if constexpr (std::is_same_v<S, V>) {
                    t.val = l.val.data();
                } else {
                    // the region computes in S from its own copy of the values
                    // (widening FP32 to FP64 is exact: the same products as the
                    // launched kernels, which widen each value as they read it)
                    Level<S, V> &lw = levels_[d];
                    if (!lw.val_s.data()) {
                        lw.val_s.allocate(static_cast<size_t>(lw.nnz));
                        convert(ctx, lw.nnz, lw.val.data(), lw.val_s.data());
                    }
                    t.val = lw.val_s.data();
                }
                t.dinv = l.dinv.data();
                t.rhs = l.rhs.data();
                t.x0 = l.x0.data();
                t.x1 = l.x1.data();
                if (d + 1 < levels_.size()) {
                    t.map = l.map.data();
                    t.off = l.off.data();
                    t.mem = l.mem.data();
                }
                tl.push_back(t);
            }
            const int dense_n = factored_ ? static_cast<int>(levels_.back().n) : 0;
            TailParent parent;
            parent.n = levels_[root - 1].n;
            parent.off = levels_[root - 1].off.data();
            parent.mem = levels_[root - 1].mem.data();
            bool ok = tail_.plan(ctx, tl, parent, factored_ ? inv_.data() : nullptr, dense_n, w_,
                                 static_cast<int>(max_steps));
            for (const auto &[first, count] : entries_) ok = ok && tail_.add_entry(rec_, first, count);
            rec_.clear();
            entries_.clear();
            if (ok) {
                tail_.upload(ctx);
                return;
            }
            coop_from_ = none;
        }
        }
    }

    static constexpr int64_t kFusedProlongRows = 131072;
    static constexpr int64_t kScatterRows = 131072;

    AmgConfig cfg_;
    S w_;
    std::vector<Level<S, V>> levels_;
    DeviceBuffer<double> lu_, inv_;
    DeviceBuffer<int32_t> piv_;
    bool factored_{false};
    cudaGraphExec_t exec_{nullptr};
    bool capture_failed_{false};
    int64_t per_cycle_{0};
    std::vector<int> final_cur_;
    std::vector<int64_t> captured_visits_;
    // small-level sub-cycles (one cluster launch each)
    size_t coop_from_{~size_t(0)};
    bool recording_{false}, dry_{false};
    // transfer fusion
    int fuse_{1};
    PendingRestrict pr_;
    PendingWrite pw_;
    // The cycle input still to be converted into the finest level's rhs
    // (taken by that level's zero-guess sweep, else launched by flush).
    struct PendingInput {
        const void *src{nullptr};
        bool f64{false};
    } pin_;
    std::vector<CoarseStep<S>> rec_;
    std::vector<std::pair<size_t, size_t>> entries_;
    size_t entry_{0};
    TailRegion<S> tail_;
    size_t region_start_{0};
};

}  // namespace

std::unique_ptr<Hierarchy> restore_hierarchy(tf_ctx *ctx, const AmgConfig &cfg, int storage_type,
                                             std::istream &in) {
    if (storage_type == TF_F32_VALUES) {
        auto h = std::make_unique<HierarchyImpl<double, float>>(cfg);
        h->restore(ctx, in);
        return h;
    }
    if (storage_type == TF_F32) {
        auto h = std::make_unique<HierarchyImpl<float>>(cfg);
        h->restore(ctx, in);
        return h;
    }
    auto h = std::make_unique<HierarchyImpl<double>>(cfg);
    h->restore(ctx, in);
    return h;
}

std::unique_ptr<Hierarchy> build_hierarchy(tf_ctx *ctx, const AmgConfig &cfg, int storage_type,
                                           const tf_dcsr &native) {
    if (storage_type == TF_F32_VALUES) {
        require(cfg.model == nullptr, "learned damping needs a hierarchy whose values and vectors share a type");
        auto h = std::make_unique<HierarchyImpl<double, float>>(cfg);
        h->build(ctx, native);
        return h;
    }
    if (storage_type == TF_F32) {
        auto h = std::make_unique<HierarchyImpl<float>>(cfg);
        h->build(ctx, native);
        return h;
    }
    auto h = std::make_unique<HierarchyImpl<double>>(cfg);
    h->build(ctx, native);
    return h;
}

}  // namespace tfb
