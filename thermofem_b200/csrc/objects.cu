// objects.cu -- component objects of the C ABI: AMG preconditioner, Jacobi
// smoother and Krylov solvers (the setup/apply components of
// include/Preconditioner/Amg.cuh, include/Smoother/Jacobi.cuh and
// include/Solver/{Cg,BiCgStab}.cuh).  Setup is transactional for AMG and
// Jacobi (a failure keeps the previous state) and invalidating for solvers,
// as in the reference.
#include <fstream>
#include <string>

#include "engine.cuh"

using namespace tfb;

struct tf_amg {
    tf_ctx *ctx;
    int value_type, index_type;
    AmgConfig cfg;
    std::unique_ptr<Hierarchy> owned;
    Hierarchy *h{nullptr};  // owned.get(), or a solver's hierarchy for borrowed views
};

struct tf_jacobi {
    tf_ctx *ctx;
    int value_type, index_type;
    int sweeps;
    double weight;
    bool ready{false};
    int64_t n{0}, nnz{0};
    DeviceBuffer<int32_t> rp, ci;
    DeviceBuffer<unsigned char> val, dinv, rhs, x0, x1;
};

struct tf_solver {
    tf_ctx *ctx;
    int value_type, index_type;
    std::unique_ptr<Krylov> k;
    std::unique_ptr<tf_amg> view;        // borrowed view of the AMG preconditioner
};

struct tf_batch {
    tf_ctx *ctx{nullptr};
    std::vector<tf_solver *> solvers;
    std::vector<int64_t> generations;  // of the solvers when the graph was built
    cudaGraphExec_t exec{nullptr};
    bool graph_failed{false};
    void *pinned{nullptr};  // one state record per solver, read back after a launch
    size_t state_bytes{0};
    ~tf_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (pinned) cudaFreeHost(pinned);
    }
};

namespace {

void check_types(int value_type, int index_type) {
    require(value_type == TF_F32 || value_type == TF_F64, "value type must be TF_F32 or TF_F64");
    require(index_type == TF_I32 || index_type == TF_I64, "index type must be TF_I32 or TF_I64");
}

void check_matrix_types(const tf_csr *a, int value_type, int index_type) {
    check_csr(a);
    require(a->value_type == value_type && a->index_type == index_type, "matrix types differ from the component's");
}

}  // namespace

extern "C" {

void tf_amg_options_default(tf_amg_options *o) {
    if (!o) return;
    o->max_levels = 20;
    o->coarse_rows = 64;
    o->matching_rounds = 8;
    o->pre_sweeps = 1;
    o->post_sweeps = 1;
    o->coarse_sweeps = 8;
    o->jacobi_weight = 0.75;
    o->strength_threshold = 0.25;
    o->absorb_singletons = 1;
    o->compact_sort_keys = 0;
    o->cycle = TF_CYCLE_V;
    o->hierarchy_type = -1;
    o->coarse_lu_rows = 64;
    o->small_level_rows = 1200;
    o->damping_model = nullptr;
}

void tf_solver_options_default(int value_type, tf_solver_options *o) {
    if (!o) return;
    o->max_iterations = 1000;
    o->relative_tolerance = value_type == TF_F32 ? static_cast<double>(1e-5f) : 1e-8;
    o->absolute_tolerance = 0;
    o->residual_refresh_interval = 50;
}

int tf_amg_create(tf_ctx *ctx, int value_type, int index_type, const tf_amg_options *opt, tf_amg **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out && opt, "null argument");
        *out = nullptr;
        check_types(value_type, index_type);
        *out = new tf_amg{ctx, value_type, index_type, AmgConfig(*opt), nullptr, nullptr};
    });
}

int tf_amg_destroy(tf_amg *m) {
    return guard([&] {
        if (!m) return;
        DeviceScope scope(m->ctx->device);
        delete m;
    });
}

int tf_amg_setup(tf_amg *m, const tf_csr *a) {
    return guard([&] {
        require(m != nullptr, "null AMG");
        check_matrix_types(a, m->value_type, m->index_type);
        require(a->rows > 0 && a->rows == a->cols, "Solver requires a nonempty square matrix");
        DeviceScope scope(m->ctx->device);
        auto native = to_native(m->ctx, *a);
        const int storage = m->cfg.o.hierarchy_type == -1 ? m->value_type : m->cfg.o.hierarchy_type;
        auto h = build_hierarchy(m->ctx, m->cfg, storage, *native);
        m->owned = std::move(h);
        m->h = m->owned.get();
    });
}

int tf_amg_apply(tf_amg *m, const void *rhs, void *x) {
    return guard([&] {
        require(m != nullptr, "null AMG");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        require(rhs && x, "null vector");
        DeviceScope scope(m->ctx->device);
        if (m->value_type == TF_F64)
            m->h->apply(m->ctx, static_cast<const double *>(rhs), static_cast<double *>(x));
        else
            m->h->apply(m->ctx, static_cast<const float *>(rhs), static_cast<float *>(x));
        cuda_check(cudaStreamSynchronize(m->ctx->stream), "AMG apply");
        check_faults(m->ctx);
    });
}

int tf_amg_level_count(const tf_amg *m) { return m && m->h ? m->h->level_count() : 0; }

int tf_amg_level_stats(const tf_amg *m, int level, int64_t *rows, int64_t *nnz, int32_t histogram[4]) {
    return guard([&] {
        require(m != nullptr, "null AMG");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        require(level >= 0 && level < m->h->level_count(), "level out of range");
        const auto &s = m->h->stats[static_cast<size_t>(level)];
        if (rows) *rows = s.rows;
        if (nnz) *nnz = s.nnz;
        if (histogram)
            for (int k = 0; k < 4; ++k) histogram[k] = s.histogram[k];
    });
}

const char *tf_amg_stop_reason(const tf_amg *m) { return m && m->h ? m->h->stop_reason.c_str() : ""; }
const char *tf_amg_coarse_solver(const tf_amg *m) { return m && m->h ? m->h->coarse_solver.c_str() : ""; }

int tf_amg_last_visits(const tf_amg *m, int64_t *visits, int capacity) {
    return guard([&] {
        require(m != nullptr && visits != nullptr, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        const auto &v = m->h->visits;
        for (int d = 0; d < capacity && d < static_cast<int>(v.size()); ++d) visits[d] = v[static_cast<size_t>(d)];
    });
}

int tf_amg_setup_phases(const tf_amg *m, double *ms, int capacity) {
    return guard([&] {
        require(m != nullptr && ms != nullptr, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        const auto &t = m->h->setup_ms;
        for (int k = 0; k < capacity && k < static_cast<int>(t.size()); ++k) ms[k] = t[static_cast<size_t>(k)];
    });
}

int tf_amg_setup_phase_count(void) { return static_cast<int>(setup_phase_names().size()); }

const char *tf_amg_setup_phase_name(int phase) {
    const auto &n = setup_phase_names();
    return phase >= 0 && phase < static_cast<int>(n.size()) ? n[static_cast<size_t>(phase)].c_str() : "";
}

int tf_amg_level_matrix(const tf_amg *m, int level, tf_csr *out) {
    return guard([&] {
        require(m != nullptr && out != nullptr, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        require(level >= 0 && level < m->h->level_count(), "level out of range");
        *out = m->h->level_matrix(level);
    });
}

int tf_amg_level_spmv(const tf_amg *m, int level, const void *x, void *y) {
    return guard([&] {
        require(m != nullptr && x != nullptr && y != nullptr && x != y, "null or aliased argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        require(level >= 0 && level < m->h->level_count(), "level out of range");
        DeviceScope scope(m->ctx->device);
        m->h->level_spmv(m->ctx, level, x, y);
    });
}

int tf_amg_level_spmv_layout(const tf_amg *m, int level, int *sliced, int64_t *entries) {
    return guard([&] {
        require(m != nullptr && sliced != nullptr && entries != nullptr, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        require(level >= 0 && level < m->h->level_count(), "level out of range");
        *sliced = m->h->level_spmv_layout(m->ctx, level, entries);
    });
}

int tf_amg_level_transfer(const tf_amg *m, int level, const int32_t **map, const int32_t **offsets,
                          const int32_t **members, int *coarse_rows) {
    return guard([&] {
        require(m != nullptr && map && offsets && members && coarse_rows, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        require(level >= 0 && level + 1 < m->h->level_count(), "level has no transfer");
        m->h->level_transfer(level, map, offsets, members, coarse_rows);
    });
}

int tf_amg_coarse_factor(const tf_amg *m, int *rows, const double **lu, const int32_t **pivots) {
    return guard([&] {
        require(m != nullptr && rows && lu && pivots, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        m->h->coarse_factor(rows, lu, pivots);
    });
}

int tf_amg_save(const tf_amg *m, const char *path) {
    return guard([&] {
        require(m != nullptr && path != nullptr, "null argument");
        if (!m->h) fail(TF_ERR_LOGIC, "AMG requires setup");
        DeviceScope scope(m->ctx->device);
        std::ofstream out(path, std::ios::binary | std::ios::trunc);
        if (!out) fail(TF_ERR_RUNTIME, std::string("AMG checkpoint: cannot open ") + path);
        m->h->save(m->ctx, out);
    });
}

int tf_amg_load(tf_amg *m, const char *path) {
    return guard([&] {
        require(m != nullptr && path != nullptr, "null argument");
        DeviceScope scope(m->ctx->device);
        std::ifstream in(path, std::ios::binary);
        if (!in) fail(TF_ERR_INVALID, std::string("AMG checkpoint: cannot open ") + path);
        const int storage = m->cfg.o.hierarchy_type == -1 ? m->value_type : m->cfg.o.hierarchy_type;
        // transactional, as setup: the previous hierarchy stays on failure
        auto h = restore_hierarchy(m->ctx, m->cfg, storage, in);
        m->owned = std::move(h);
        m->h = m->owned.get();
    });
}

int tf_jacobi_create(tf_ctx *ctx, int value_type, int index_type, int sweeps, double weight, tf_jacobi **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out != nullptr, "null output");
        *out = nullptr;
        check_types(value_type, index_type);
        const double w = value_type == TF_F32 ? static_cast<double>(static_cast<float>(weight)) : weight;
        if (sweeps < 1 || !std::isfinite(w) || w <= 0 || w >= 2) fail(TF_ERR_INVALID, "Invalid Jacobi parameters");
        auto *j = new tf_jacobi();
        j->ctx = ctx;
        j->value_type = value_type;
        j->index_type = index_type;
        j->sweeps = sweeps;
        j->weight = w;
        *out = j;
    });
}

int tf_jacobi_destroy(tf_jacobi *j) {
    return guard([&] {
        if (!j) return;
        DeviceScope scope(j->ctx->device);
        delete j;
    });
}

int tf_jacobi_setup(tf_jacobi *j, const tf_csr *a) {
    return guard([&] {
        require(j != nullptr, "null Jacobi");
        check_matrix_types(a, j->value_type, j->index_type);
        require(a->rows > 0 && a->rows == a->cols, "Solver requires a nonempty square matrix");
        DeviceScope scope(j->ctx->device);
        tf_ctx *ctx = j->ctx;
        std::unique_ptr<tf_dcsr> native;
        try {
            native = to_native(ctx, *a);
        } catch (const Failure &f) {
            if (f.code == TF_ERR_INVALID) fail(TF_ERR_INVALID, "Matrix contains nonfinite entries");
            throw;
        }
        const size_t vs = type_size(j->value_type);
        const int64_t n = native->rows, nnz = native->nnz;
        DeviceBuffer<int32_t> rp(static_cast<size_t>(n) + 1), ci(static_cast<size_t>(nnz));
        DeviceBuffer<unsigned char> val(static_cast<size_t>(nnz) * vs), dinv(static_cast<size_t>(n) * vs);
        const auto nc = csr_of(*native);
        copy_async(ctx, rp.data(), nc.rp, (n + 1) * 4);
        copy_async(ctx, ci.data(), nc.ci, nnz * 4);
        if (j->value_type == TF_F64) {
            convert(ctx, nnz, nc.val, reinterpret_cast<double *>(val.data()));
            Csr<double, int32_t> c{n, n, nnz, rp.data(), ci.data(), reinterpret_cast<const double *>(val.data())};
            inverse_diagonal(ctx, c, reinterpret_cast<double *>(dinv.data()));
        } else {
            convert(ctx, nnz, nc.val, reinterpret_cast<float *>(val.data()));
            Csr<float, int32_t> c{n, n, nnz, rp.data(), ci.data(), reinterpret_cast<const float *>(val.data())};
            inverse_diagonal(ctx, c, reinterpret_cast<float *>(dinv.data()));
        }
        DeviceBuffer<unsigned char> rhs(static_cast<size_t>(n) * vs), x0(static_cast<size_t>(n) * vs),
            x1(static_cast<size_t>(n) * vs);
        cuda_check(cudaStreamSynchronize(ctx->stream), "Jacobi setup");
        j->n = n;
        j->nnz = nnz;
        j->rp = std::move(rp);
        j->ci = std::move(ci);
        j->val = std::move(val);
        j->dinv = std::move(dinv);
        j->rhs = std::move(rhs);
        j->x0 = std::move(x0);
        j->x1 = std::move(x1);
        j->ready = true;
    });
}

int tf_jacobi_apply(tf_jacobi *j, const void *rhs, void *x) {
    return guard([&] {
        require(j != nullptr, "null Jacobi");
        if (!j->ready) fail(TF_ERR_LOGIC, "Jacobi requires setup");
        require(rhs && x, "null vector");
        DeviceScope scope(j->ctx->device);
        tf_ctx *ctx = j->ctx;
        const size_t bytes = static_cast<size_t>(j->n) * type_size(j->value_type);
        copy_async(ctx, j->rhs.data(), rhs, bytes);
        copy_async(ctx, j->x0.data(), x, bytes);
        auto run = [&](auto t) {
            using T = decltype(t);
            Csr<T, int32_t> c{j->n, j->n, j->nnz, j->rp.data(), j->ci.data(), reinterpret_cast<const T *>(j->val.data())};
            T *xa = reinterpret_cast<T *>(j->x0.data()), *xb = reinterpret_cast<T *>(j->x1.data());
            for (int s = 0; s < j->sweeps; ++s) {
                jacobi_sweep(ctx, c, reinterpret_cast<const T *>(j->dinv.data()), reinterpret_cast<const T *>(j->rhs.data()),
                             xa, xb, static_cast<T>(j->weight), nullptr, nullptr, static_cast<const T *>(nullptr));
                std::swap(xa, xb);
            }
            copy_async(ctx, x, xa, bytes);
        };
        if (j->value_type == TF_F64) run(double{});
        else run(float{});
        cuda_check(cudaStreamSynchronize(ctx->stream), "Jacobi apply");
        check_faults(ctx);
    });
}

int tf_solver_create(tf_ctx *ctx, int kind, int value_type, int index_type, const tf_solver_options *opt, int precond,
                     const tf_amg_options *amg_opt, tf_solver **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out && opt, "null argument");
        *out = nullptr;
        check_types(value_type, index_type);
        auto s = std::make_unique<tf_solver>();
        s->ctx = ctx;
        s->value_type = value_type;
        s->index_type = index_type;
        s->k = make_krylov(kind, value_type, index_type, *opt, precond, amg_opt);
        *out = s.release();
    });
}

int tf_solver_destroy(tf_solver *s) {
    return guard([&] {
        if (!s) return;
        DeviceScope scope(s->ctx->device);
        delete s;
    });
}

int tf_solver_setup(tf_solver *s, const tf_csr *a) {
    return guard([&] {
        require(s != nullptr, "null solver");
        check_matrix_types(a, s->value_type, s->index_type);
        DeviceScope scope(s->ctx->device);
        s->view.reset();
        s->k->setup(s->ctx, *a);
    });
}

int tf_solver_apply(tf_solver *s, const void *rhs, void *x, int host_buffers, tf_solve_result *result) {
    return guard([&] {
        require(s != nullptr && result != nullptr, "null argument");
        require(rhs && x, "null vector");
        DeviceScope scope(s->ctx->device);
        // Host buffers: the solve's own input and output copies (unified
        // addressing, cudaMemcpyDefault) move rhs and x between the host and
        // the solver's vectors directly; the solve ends with a stream sync.
        if (host_buffers && s->k->rows() == 0) fail(TF_ERR_LOGIC, "solver requires setup");
        *result = s->k->solve(s->ctx, rhs, x);
    });
}

tf_amg *tf_solver_amg(tf_solver *s) {
    if (!s || !s->k || !s->k->amg()) return nullptr;
    if (!s->view) {
        tf_amg_options o;
        tf_amg_options_default(&o);
        s->view.reset(new tf_amg{s->ctx, s->value_type, s->index_type, AmgConfig(o), nullptr, s->k->amg()});
    }
    s->view->h = s->k->amg();
    return s->view.get();
}

double tf_solver_last_apply_ms(const tf_solver *s) { return s && s->k ? s->k->last_ms : 0.0; }

int tf_solver_last_execution(const tf_solver *s) { return s && s->k ? s->k->last_execution : -1; }

int tf_solver_spmv(tf_solver *s, const void *x, void *y) {
    return guard([&] {
        require(s != nullptr && x != nullptr && y != nullptr && x != y, "null or aliased argument");
        DeviceScope scope(s->ctx->device);
        s->k->spmv(s->ctx, x, y);
    });
}

int tf_solver_spmv_layout(const tf_solver *s, int *sliced, int64_t *entries) {
    return guard([&] {
        require(s != nullptr && sliced != nullptr && entries != nullptr, "null argument");
        *sliced = s->k->spmv_layout(s->ctx, entries);
    });
}

int tf_solver_set_graph_mode(tf_solver *s, int mode) {
    return guard([&] {
        require(s != nullptr && (mode == 0 || mode == 1), "graph mode must be 0 or 1");
        s->k->graph_mode = mode;
    });
}

int tf_batch_create(tf_ctx *ctx, int count, tf_solver *const *solvers, tf_batch **out) {
    return guard([&] {
        require(out != nullptr, "null argument");
        *out = nullptr;
        check_ctx(ctx);
        require(count >= 1 && solvers != nullptr, "a batch needs at least one solver");
        auto b = std::make_unique<tf_batch>();
        b->ctx = ctx;
        for (int k = 0; k < count; ++k) {
            require(solvers[k] != nullptr && solvers[k]->ctx == ctx, "batched solvers must share the batch context");
            for (int j = 0; j < k; ++j) require(solvers[j] != solvers[k], "a solver appears twice in the batch");
            b->solvers.push_back(solvers[k]);
        }
        DeviceScope scope(ctx->device);
        b->state_bytes = (b->solvers.front()->k->state_bytes() + 15) & ~size_t(15);
        cuda_check(cudaMallocHost(&b->pinned, b->state_bytes * static_cast<size_t>(count)), "cudaMallocHost");
        *out = b.release();
    });
}

int tf_batch_destroy(tf_batch *b) {
    return guard([&] {
        if (!b) return;
        DeviceScope scope(b->ctx->device);
        delete b;
    });
}

int tf_batch_apply(tf_batch *b, const void *const *rhs, void *const *x, tf_solve_result *results) {
    return guard([&] {
        require(b != nullptr && rhs != nullptr && x != nullptr && results != nullptr, "null argument");
        tf_ctx *ctx = b->ctx;
        DeviceScope scope(ctx->device);
        const size_t count = b->solvers.size();
        bool stale = b->exec == nullptr;
        for (size_t k = 0; k < count; ++k) {
            require(rhs[k] != nullptr && x[k] != nullptr, "null vector");
            const int64_t g = b->solvers[k]->k->generation();
            if (g == 0) fail(TF_ERR_LOGIC, "batched solver requires setup");
            if (b->generations.size() != count || b->generations[k] != g) stale = true;
        }
        if (stale && !b->graph_failed) {
            // every solve as an independent branch of one graph
            if (b->exec) cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
            cudaGraph_t g = nullptr;
            try {
                cuda_check(cudaGraphCreate(&g, 0), "graph create");
                for (auto *s : b->solvers) s->k->batch_nodes(ctx, g);
                cuda_check(cudaGraphInstantiate(&b->exec, g, 0), "batch graph instantiate");
            } catch (const Failure &) {
                end_capture_into_graph(ctx);
                b->exec = nullptr;
                b->graph_failed = true;
            }
            if (g) cudaGraphDestroy(g);
            b->generations.clear();
            for (auto *s : b->solvers) b->generations.push_back(s->k->generation());
        }
        if (!b->exec) {
            // CUDA refused the batch graph: the same solves one by one
            for (size_t k = 0; k < count; ++k) results[k] = b->solvers[k]->k->solve(ctx, rhs[k], x[k]);
            return;
        }
        for (size_t k = 0; k < count; ++k) b->solvers[k]->k->batch_stage(ctx, rhs[k], x[k]);
        cuda_check(cudaGraphLaunch(b->exec, ctx->stream), "batch graph launch");
        unsigned char *host = static_cast<unsigned char *>(b->pinned);
        for (size_t k = 0; k < count; ++k) b->solvers[k]->k->batch_finish(ctx, x[k], host + k * b->state_bytes);
        cuda_check(cudaStreamSynchronize(ctx->stream), "batch");
        for (size_t k = 0; k < count; ++k) {
            results[k] = b->solvers[k]->k->batch_result(host + k * b->state_bytes);
            ctx->launches += b->solvers[k]->k->batch_launches(results[k].iterations);
        }
        check_faults(ctx);
    });
}

}  // extern "C"
