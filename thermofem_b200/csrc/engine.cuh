// engine.cuh -- the AMG hierarchy and the Krylov solvers behind the
// component API (include/Preconditioner/Amg.cuh, include/Solver/Cg.cuh,
// include/Solver/BiCgStab.cuh of the reference).
#pragma once
#include <istream>
#include <memory>
#include <ostream>
#include <string>
#include <vector>

#include "ops.cuh"

namespace tfb {

struct LevelStats {
    int64_t rows{0}, nnz{0};
    int32_t histogram[4]{0, 0, 0, 0};
};

// Validated copy of tf_amg_options.
struct DampingModel;

struct AmgConfig {
    tf_amg_options o;
    std::shared_ptr<const DampingModel> model;  // per-row damping (snapshot of o.damping_model)
    explicit AmgConfig(const tf_amg_options &opt);
};

// Canonical FP64/int32 copy of a square CSR (GpuAggregation::canonical after
// toNativeMatrix, src/Multigrid/GpuAggregation.cu:991-1007,1099-1136).
std::unique_ptr<tf_dcsr> to_native(tf_ctx *ctx, const tf_csr &a);

// A built hierarchy; the storage/arithmetic type of the cycle is fixed at
// construction (TF_F64 or TF_F32).
class Hierarchy {
  public:
    virtual ~Hierarchy() = default;
    // x = M^-1 rhs (zero initial guess); enqueued on the context stream.
    // rhs may alias x.  Vector type T is the caller's (float or double).
    virtual void apply(tf_ctx *ctx, const double *rhs, double *x) = 0;
    virtual void apply(tf_ctx *ctx, const float *rhs, float *x) = 0;
    // apply without its last step: x = M^-1 rhs is left in the finest
    // level's own storage (storage_type()) and returned, for a caller that
    // converts it inside its next kernel.
    virtual const void *apply_open(tf_ctx *ctx, const double *rhs) = 0;
    virtual const void *apply_open(tf_ctx *ctx, const float *rhs) = 0;
    virtual int storage_type() const = 0;
    virtual int64_t rows() const = 0;
    virtual int level_count() const = 0;
    virtual tf_csr level_matrix(int d) const = 0;
    // y = A_d x with level d's operator as the cycle streams it (its column
    // storage included); x, y of the level's storage type.
    virtual void level_spmv(tf_ctx *ctx, int d, const void *x, void *y) const = 0;
    // 1 (2: rows sorted within tiles) when level d's SpMV streams its sliced
    // copy (entries incl. padding), 0 for CSR.
    virtual int level_spmv_layout(tf_ctx *ctx, int d, int64_t *entries) const = 0;
    virtual void level_transfer(int d, const int32_t **map, const int32_t **off, const int32_t **mem,
                                int *coarse) const = 0;
    // The coarse level's LU factor (rows x rows doubles, row-major, and the
    // pivot row of each step), rows = 0 when the coarse solve is Jacobi.
    virtual void coarse_factor(int *rows, const double **lu, const int32_t **pivots) const = 0;
    // Kernels launched by one cycle (graph replay counts them too).
    virtual int64_t kernels_per_cycle() const = 0;
    // Writes the hierarchy (restore_hierarchy reads it back).
    virtual void save(tf_ctx *ctx, std::ostream &out) const = 0;

    std::vector<LevelStats> stats;
    std::vector<int64_t> visits;
    std::string stop_reason, coarse_solver;
    // Setup time per phase (ms, CUDA events on the context stream), in the
    // order of setup_phase_names().
    std::vector<double> setup_ms;
};

// Names of the setup phases Hierarchy::setup_ms reports.
const std::vector<std::string> &setup_phase_names();

// Builds the hierarchy from the canonical native fine matrix (Amg::setup,
// include/Preconditioner/Amg.cuh:81-143).  row_weights (optional, per level)
// give per-row Jacobi damping for the smoothers.
std::unique_ptr<Hierarchy> build_hierarchy(tf_ctx *ctx, const AmgConfig &cfg, int storage_type,
                                           const tf_dcsr &native);
// A hierarchy written by Hierarchy::save, for a component of the same types
// and smoothing; the per-level copies, launch shapes and the small-level
// region are derived again as build_hierarchy derives them.
std::unique_ptr<Hierarchy> restore_hierarchy(tf_ctx *ctx, const AmgConfig &cfg, int storage_type,
                                             std::istream &in);

// Krylov solver (kind TF_SOLVER_CG or TF_SOLVER_BICGSTAB) over vectors of T.
class Krylov {
  public:
    virtual ~Krylov() = default;
    virtual void setup(tf_ctx *ctx, const tf_csr &a) = 0;
    // rhs/x are device pointers of T; x holds the initial guess.
    virtual tf_solve_result solve(tf_ctx *ctx, const void *rhs, void *x) = 0;
    // y = A x with the solver's operator as the solve streams it.
    virtual void spmv(tf_ctx *ctx, const void *x, void *y) = 0;
    // 1 when that SpMV streams the sliced copy (entries incl. padding), 0 for CSR.
    virtual int spmv_layout(tf_ctx *ctx, int64_t *entries) const = 0;
    virtual Hierarchy *amg() = 0;
    virtual int64_t rows() const = 0;
    // Batches (tf_batch): the whole solve added to graph g as an independent
    // branch that loads its own initial state; inputs staged into and the
    // result copied out of the solver's buffers around the graph launch.
    virtual void batch_nodes(tf_ctx *ctx, cudaGraph_t g) = 0;
    virtual int64_t batch_launches(int iterations) const = 0;
    virtual void batch_stage(tf_ctx *ctx, const void *rhs, const void *x) = 0;
    virtual void batch_finish(tf_ctx *ctx, void *x, void *state_host) = 0;
    virtual size_t state_bytes() const = 0;
    virtual tf_solve_result batch_result(const void *state_host) const = 0;
    // Incremented by every setup (a batch graph built before is stale).
    virtual int64_t generation() const = 0;
    // 1: the whole solve is one graph with a device-side loop (default);
    // 0: one graph per iteration and a host loop (same kernels; profilers
    // that cannot see inside conditional graph nodes need this).
    int graph_mode{1};
    double last_ms{0};
    // How the last solve ran: 2 one whole-solve graph, 1 one graph per
    // iteration, 0 uncaptured launches, -1 no solve yet.
    int last_execution{-1};
};

std::unique_ptr<Krylov> make_krylov(int kind, int value_type, int index_type, const tf_solver_options &opt,
                                    int precond, const tf_amg_options *amg_opt);
void validate_solver_options(const tf_solver_options &o);

}  // namespace tfb
