/*
 * thermofem_b200.h -- C ABI of the B200 (sm_100a) sparse solve path.
 *
 * Plain pointers and sizes, int status returns (TF_OK == 0, negative codes
 * below), no exceptions across the boundary.  Device pointers are caller
 * owned unless a function returns an opaque handle; every launch goes to the
 * stream of the tf_ctx it is given.  Reference citations are paths inside
 * the Mgepahmge/ThermoFEM project and name the interface each entry point
 * replaces.  Nothing here falls back to the CPU: a missing GPU is an error.
 */
#ifndef THERMOFEM_B200_H
#define THERMOFEM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes ------------------------------------------------------ */
/* Map onto the reference's exception classes (include/DataStructure/
 * Memory.cuh:52-66 CudaError; std::invalid_argument / logic_error /
 * length_error thrown by the component constructors and setup). */
#define TF_OK 0
#define TF_ERR_INVALID (-1)   /* std::invalid_argument */
#define TF_ERR_CUDA (-2)      /* CudaError */
#define TF_ERR_LENGTH (-3)    /* std::length_error / overflow_error */
#define TF_ERR_LOGIC (-4)     /* std::logic_error (e.g. apply before setup) */
#define TF_ERR_TIMEOUT (-5)   /* a bounded device wait gave up */
#define TF_ERR_NOMEM (-6)     /* allocation failure */
#define TF_ERR_RUNTIME (-7)   /* std::runtime_error (I/O, parse) */

/* ---- element types ----------------------------------------------------- */
#define TF_F32 0
#define TF_F64 1
#define TF_I32 2
#define TF_I64 3
/* tf_amg_options.hierarchy_type only: operators stored in FP32, the cycle's
 * vectors and arithmetic in FP64 (no reference counterpart). */
#define TF_F32_VALUES 4

/* Solve status, values of thermofem::SolveStatus (include/Solver/
 * Interfaces.cuh:10). */
#define TF_CONVERGED 0
#define TF_MAX_ITERATIONS 1
#define TF_BREAKDOWN 2
#define TF_NONFINITE 3

/* Cycle kinds, thermofem::multigrid::Cycle (include/Multigrid/Cycle.cuh:10). */
#define TF_CYCLE_V 0
#define TF_CYCLE_W 1
#define TF_CYCLE_F 2

const char *tf_version(void);
/* Message of the last failing call on this thread. */
const char *tf_last_error(void);
/* The cudaError_t behind the last failing call on this thread when it
 * failed with TF_ERR_CUDA or TF_ERR_NOMEM, else 0 (the code the
 * reference's CudaError carries, include/DataStructure/Memory.cuh:52-66). */
int tf_last_cuda_error(void);
const char *tf_status_string(int status);

/* ---- execution context ------------------------------------------------- */
/* Owns (or borrows) a stream and a grow-only scratch arena on one device.
 * Not thread safe; one per solver instance.  Replaces the reference's
 * per-object handles (src/LinearAlgebra/IterationContext.cu:35-122) and the
 * CUB workspace of GpuAggregation (src/Multigrid/GpuAggregation.cu:84-126). */
typedef struct tf_ctx tf_ctx;
int tf_ctx_create(int device, void *stream /* cudaStream_t or NULL */, tf_ctx **out);
int tf_ctx_destroy(tf_ctx *ctx);
int tf_ctx_synchronize(tf_ctx *ctx);
/* Self-check of the failure path of the bounded device waits (no reference
 * counterpart): one CTA waits, with the wait every pipelined kernel uses, on a
 * barrier that nothing completes, gives up after `polls` polls (1..2^20) and
 * raises the context's fault word as a stalled kernel would.  Returns
 * TF_ERR_TIMEOUT, having cleared the word; the context stays usable.  A
 * monitoring caller can run it to check that a stalled wait surfaces as an
 * error instead of a hang. */
int tf_ctx_check_bounded_wait(tf_ctx *ctx, int64_t polls);
void *tf_ctx_stream(tf_ctx *ctx);
int tf_ctx_device(tf_ctx *ctx);
/* Number of kernels this context has launched (all entry points). */
int64_t tf_ctx_launch_count(tf_ctx *ctx);
int tf_device_count(int *count);

/* ---- CSR descriptor ---------------------------------------------------- */
/* Device CSR view (include/DataStructure/CsrMatrix.cuh:36-217): offsets
 * rows+1, indices/values nnz, index_type TF_I32|TF_I64, value_type
 * TF_F32|TF_F64. */
typedef struct {
    int64_t rows, cols, nnz;
    int index_type, value_type;
    const void *offsets;
    const void *indices;
    const void *values;
} tf_csr;

/* Device CSR owned by the library (outputs of setup stages). */
typedef struct tf_dcsr tf_dcsr;
int tf_dcsr_view(const tf_dcsr *m, tf_csr *out);
int tf_dcsr_free(tf_dcsr *m);

/* ---- data-structure checks -------------------------------------------- */
/* Structural validation on the device: offsets monotone and bounded, indices
 * in range.  Replaces detail::validateDeviceCsr (src/DataStructure/
 * CsrMatrix.cu:12-58).  TF_ERR_INVALID when malformed. */
int tf_csr_validate(tf_ctx *ctx, const tf_csr *a);
/* Canonical-form check (src/Multigrid/GpuAggregation.cu:283-304): *flags
 * bit 1 = unsorted/duplicate columns, bit 2 = invalid structure or
 * nonfinite value.  Host int written after a stream sync. */
int tf_csr_check_canonical(tf_ctx *ctx, const tf_csr *a, int *flags);
/* Sorted, duplicate-summed copy, explicit zeros kept
 * (GpuAggregation::canonical, GpuAggregation.cu:991-1007). */
int tf_canonicalize(tf_ctx *ctx, const tf_csr *a, tf_dcsr **out);
/* Element-type conversion of a device array (GpuAggregation.cu:1101-1108). */
int tf_convert(tf_ctx *ctx, int64_t n, int src_type, const void *src, int dst_type, void *dst);

/* ---- SpMV family (IterationContext::multiply/residual/jacobi,
 *      src/LinearAlgebra/IterationContext.cu:140-269) --------------------- */
/* y = A x.  x, y have A's value type; y must not alias x. */
int tf_spmv(tf_ctx *ctx, const tf_csr *a, const void *x, void *y);
int tf_spmv_f64(tf_ctx *ctx, int64_t rows, int64_t cols, int64_t nnz, const int32_t *offsets,
                const int32_t *indices, const double *values, const double *x, double *y);
int tf_spmv_f32(tf_ctx *ctx, int64_t rows, int64_t cols, int64_t nnz, const int32_t *offsets,
                const int32_t *indices, const float *values, const float *x, float *y);
/* SpMV autotuner (replaces the fixed library algorithm choice of
 * cusparseSpMV ALG_DEFAULT, IterationContext.cu:140-159): times the feasible
 * pipelined launch shapes (1 or 2 rows per thread, ring depth 2-3, 1-6
 * resident CTAs per SM, chunk capacity 100% or 125% of the mean tile) on this
 * operator and caches the fastest for every later row-tile launch over an
 * operator of the same shape (rows, nnz, types).  A solver's or hierarchy's
 * own operators that carry a sliced copy also time the sliced kernel (next
 * tile prefetched or not, 2-6 resident CTAs per SM).  Operators larger than
 * half the L2 cache are timed with the cache flushed before every launch, as
 * a solve meets them.  y is overwritten.  Outputs may be NULL; *ms is the
 * best time per launch.  Results never depend on the shape chosen. */
int tf_autotune_spmv(tf_ctx *ctx, const tf_csr *a, const void *x, void *y, int *stages, int *ctas_per_sm,
                     int *cap_pct, int *rows_per_thread, float *ms);
/* Sets the cached launch shape for operators of a's shape without timing
 * (no reference counterpart: the library picks its own algorithm).
 * stages 2-4, ctas_per_sm 1-8, cap_pct 50-400, rows_per_thread 1 or 2;
 * TF_ERR_INVALID otherwise or when the stage ring does not fit in shared
 * memory.  Applies to launches enqueued or captured afterwards. */
int tf_spmv_set_config(tf_ctx *ctx, const tf_csr *a, int stages, int ctas_per_sm, int cap_pct,
                       int rows_per_thread);
/* r = b - A x in one pass (replaces SpMV + scal + axpy, IterationContext.cu:167-175). */
int tf_residual(tf_ctx *ctx, const tf_csr *a, const void *b, const void *x, void *r);
/* One fused weighted-Jacobi sweep x_out = x + w * Dinv (b - A x)
 * (Jacobi.cuh:60-74 with IterationContext.cu:26-32).  row_weight (float,
 * nullable) replaces w per row.  When map/coarse are given the sweep reads
 * x~ = x + coarse[map] (prolongation fused, GpuAggregation.cu:970-976).
 * x_out must not alias x. */
int tf_jacobi_sweep(tf_ctx *ctx, const tf_csr *a, const void *dinv, const void *b, const void *x, void *x_out,
                    double weight, const float *row_weight, const int32_t *map, const void *coarse);
/* Zero-guess sweep x = w * Dinv * b (no SpMV). */
int tf_jacobi_zero(tf_ctx *ctx, int64_t n, int value_type, const void *dinv, const void *b, void *x, double weight,
                   const float *row_weight);
/* The Jacobi update on its own, x += w * dinv * (b - ax) with ax = A x formed
 * by the caller (IterationContext::jacobi, src/LinearAlgebra/
 * IterationContext.cu:26-32,251-269); x must not alias an input. */
int tf_jacobi_update(tf_ctx *ctx, int value_type, int64_t n, double weight, const void *dinv, const void *b,
                     const void *ax, void *x);
/* Inverse diagonal with duplicate diagonals summed; TF_ERR_INVALID on a
 * missing, zero or nonfinite diagonal or reciprocal (LinearAlgebra/
 * Diagonal.cuh:13-36), computed on the device. */
int tf_inverse_diagonal(tf_ctx *ctx, const tf_csr *a, void *dinv);

/* ---- aggregate transfers (GpuAggregation.cu:950-976,1050-1067) --------- */
/* coarse[c] = sum of fine[members] in member order (no float atomics). */
int tf_restrict(tf_ctx *ctx, int value_type, int64_t coarse_rows, const int32_t *offsets, const int32_t *members,
                const void *fine, void *coarse);
/* fine[i] += coarse[map[i]]. */
int tf_prolong(tf_ctx *ctx, int value_type, int64_t fine_rows, const int32_t *map, const void *coarse,
               void *fine);

/* ---- BLAS-1 and fused Krylov steps (IterationContext.cu:161-249) ------- */
/* out[k] = sum_i x_k[i] * y_k[i] for k < count (count <= 4), FP64
 * accumulation with a deterministic two-stage reduction; out is a device
 * double array.  Partial sums live in the context's scratch arena. */
int tf_dot_multi(tf_ctx *ctx, int value_type, int64_t n, int count, const void *const *xs, const void *const *ys,
                 double *out);
/* y = a x + b y (FP64 scalars). */
int tf_axpby(tf_ctx *ctx, int value_type, int64_t n, double a, const void *x, double b, void *y);
/* The Krylov solvers' fused multi-output vector steps, one pass each (the
 * reference performs each as separate IterationContext axpy/scale/norm calls
 * with a host round trip per reduction: Cg.cuh:147-158,172-174,
 * BiCgStab.cuh:170-180,195-198,228-231).  Vectors are device arrays of value_type; the
 * squared norms rr/ss are device doubles, reduced in FP64 over a fixed
 * partition of n (the same bits on any GPU).
 *   cg_update:          x += alpha p;  r -= alpha ap;  *rr = r.r
 *   cg_direction:       p = z + beta p  (p = z with restart != 0)
 *   bicgstab_direction: p = r + beta (p - omega v)  (p = r with restart != 0)
 *   bicgstab_s:         s = r - alpha v;  x += alpha phat;  *ss = s.s
 *   bicgstab_update:    x += omega shat;  r = s - omega t;  *rr = r.r  */
int tf_krylov_cg_update(tf_ctx *ctx, int value_type, int64_t n, double alpha, const void *p, const void *ap,
                        void *x, void *r, double *rr);
int tf_krylov_cg_direction(tf_ctx *ctx, int value_type, int64_t n, double beta, int restart, const void *z, void *p);
int tf_krylov_bicgstab_direction(tf_ctx *ctx, int value_type, int64_t n, double beta, double omega, int restart,
                                 const void *r, const void *v, void *p);
int tf_krylov_bicgstab_s(tf_ctx *ctx, int value_type, int64_t n, double alpha, const void *r, const void *v,
                         const void *phat, void *x, void *s, double *ss);
int tf_krylov_bicgstab_update(tf_ctx *ctx, int value_type, int64_t n, double omega, const void *shat,
                              const void *s, const void *t, void *x, void *r, double *rr);

/* ---- setup stages (GpuAggregation, include/Multigrid/GpuAggregation.cuh:47-64) */
/* Row validation (finite values, nonzero diagonal with finite reciprocal)
 * and row max |offdiag| (GpuAggregation.cu:247-271); *bad set on failure. */
int tf_row_stats(tf_ctx *ctx, const tf_csr *a, double *row_max, int *bad);
/* Symmetric strength graph, max-merged (GpuAggregation.cu:339-390). */
int tf_strength(tf_ctx *ctx, const tf_csr *a, const double *row_max, double threshold, tf_dcsr **graph);
/* Synchronous handshake matching, rounds 1..8 (GpuAggregation.cu:402-505):
 * map[rows] gets consecutive pair ids, *count their number. */
int tf_match(tf_ctx *ctx, const tf_csr *graph, int rounds, int32_t *map, int *count);
/* Graph quotient by map, intra edges dropped, max-merged
 * (GpuAggregation.cu:534-576). */
int tf_contract(tf_ctx *ctx, const tf_csr *graph, const int32_t *map, int count, tf_dcsr **out);

/* Aggregate transfer (AggregateTransfer, GpuAggregation.cuh:13-17). */
typedef struct tf_transfer tf_transfer;
/* Two-stage matching + optional two absorption rounds, compaction, member
 * table and histogram (GpuAggregation::aggregate, GpuAggregation.cu:766-818). */
int tf_aggregate(tf_ctx *ctx, const tf_csr *graph, int rounds, int absorb_singletons, tf_transfer **out);
int tf_transfer_info(const tf_transfer *t, int *fine_rows, int *coarse_rows, int32_t histogram[4]);
/* Device arrays owned by the transfer: map[fine], offsets[coarse+1], members[fine]. */
int tf_transfer_arrays(const tf_transfer *t, const int32_t **map, const int32_t **offsets,
                       const int32_t **members);
int tf_transfer_free(tf_transfer *t);
/* Ac = P^T A P by coordinate mapping and sum (GpuAggregation.cu:136-234). */
int tf_galerkin(tf_ctx *ctx, const tf_csr *a, const tf_transfer *t, tf_dcsr **out);
/* The same product from an aggregate map held by the caller
 * (multigrid::galerkin(a, AggregateTransfer), GpuAggregation.cu:1029-1036):
 * map[rows] (device) gives each fine row's aggregate in 0..coarse_rows-1. */
int tf_galerkin_map(tf_ctx *ctx, const tf_csr *a, const int32_t *map, int coarse_rows, tf_dcsr **out);

/* ---- sort / reduce / scan primitives (replace CUB, GpuAggregation.cu:116-211) */
/* Stable LSD radix sort of (u64 key, f64 value) pairs on bits
 * [0, end_bit).  Outputs must not alias inputs. */
int tf_radix_sort_pairs_u64f64(tf_ctx *ctx, int64_t n, const uint64_t *keys_in, const double *values_in,
                               uint64_t *keys_out, double *values_out, int end_bit);
/* Reduce runs of equal keys left to right: op 0 = sum, 1 = max.
 * *count (host) receives the number of unique keys. */
int tf_reduce_by_key_u64f64(tf_ctx *ctx, int64_t n, const uint64_t *keys, const double *values, int op,
                            uint64_t *keys_out, double *values_out, int64_t *count);
/* Exclusive prefix sum of int32 (out may alias in). */
int tf_scan_exclusive_i32(tf_ctx *ctx, int64_t n, const int32_t *in, int32_t *out);
/* The same exclusive prefix sum without allocating anything (no counterpart
 * in the reference).  For callers that cannot allocate device memory when
 * they need a scan (inside an allocator or memory-pool callback, under a
 * fixed device-memory budget, or where cudaMalloc's implicit device
 * synchronisation is not acceptable) and that may not even hold a tf_ctx.
 * Its scratch is a 256 KB array compiled into the library, held by every
 * device that loads the library until the process exits; n is limited to
 * 134,217,728 (2^27) items, larger n returns TF_ERR_LENGTH.  Runs on `stream`
 * (a cudaStream_t, NULL = legacy default stream) of the current device and
 * returns without synchronising.  The first call on a device loads this
 * library's kernels there if CUDA has not loaded them yet (lazy loading, the
 * default since CUDA 12.2) -- which allocates the array and the code on the
 * device and may synchronise it -- and looks up the array's device address
 * (cudaGetSymbolAddress): make that first call beforehand, where allocating
 * is allowed and outside any stream capture; later calls allocate nothing.
 * Not usable after cudaDeviceReset in the same process (the address is kept
 * per device).  All calls on a device share the array:
 * calls whose kernels may overlap on the GPU race and give undefined results.
 * out may alias in. */
int tf_scan_exclusive_i32_noalloc(void *stream, int64_t n, const int32_t *in, int32_t *out);

/* ---- coarse dense LU (GpuAggregation.cu:827-939,1068-1098) ------------- */
/* Partial-pivot LU of a canonical FP64 CSR with rows <= 256 (reference:
 * <= 64); pivot threshold 64*DBL_EPSILON*max|A|.  lu: rows*rows doubles,
 * pivots: rows ints (device).  *factored = 1 on success, 0 when singular. */
int tf_coarse_lu_factor(tf_ctx *ctx, const tf_csr *a, double *lu, int32_t *pivots, int *factored);
/* x = A^-1 b from the factor; b and x may alias; value_type of b/x. */
int tf_coarse_lu_solve(tf_ctx *ctx, int rows, const double *lu, const int32_t *pivots, int value_type,
                       const void *b, void *x);

/* ---- components (include/Smoother/Jacobi.cuh, include/Preconditioner/
 *      Amg.cuh, include/Solver/{Cg,BiCgStab}.cuh) ------------------------ */
/* AmgOptions (Amg.cuh:14-25) plus the precision extension. */
/* A learned per-row Jacobi damping model (tf_mlp_*, below). */
typedef struct tf_mlp tf_mlp;

typedef struct {
    int max_levels;          /* 1..20, default 20 */
    int coarse_rows;         /* 1..256, default 64 */
    int matching_rounds;     /* 1..8, default 8 */
    int pre_sweeps, post_sweeps; /* default 1, 1 */
    int coarse_sweeps;       /* default 8 */
    double jacobi_weight;    /* default 0.75 */
    double strength_threshold; /* default 0.25 */
    int absorb_singletons;   /* default 1 */
    int compact_sort_keys;   /* default 0; does not change results */
    int cycle;               /* TF_CYCLE_V */
    int hierarchy_type;      /* TF_F64 or TF_F32 storage/arithmetic of the cycle, TF_F32_VALUES (FP32 operators,
                                FP64 cycle); -1 = same as vectors */
    int coarse_lu_rows;      /* LU when the last level has <= this many rows; default 64, max 256 */
    int small_level_rows;    /* levels (below the finest) with <= this many rows run each sub-cycle as one
                                launch out of shared memory (one CTA when they fit, else a thread-block
                                cluster); default 1200, 0 launches every level step separately */
    const tf_mlp *damping_model; /* NULL (default): every smoother sweeps with jacobi_weight; else each row
                                    of each level is damped by the model's omega_i (weights copied at
                                    create time) -- no reference counterpart */
} tf_amg_options;
void tf_amg_options_default(tf_amg_options *o);

typedef struct tf_amg tf_amg;
/* value_type/index_type: the component's T and I (vectors and matrix). */
int tf_amg_create(tf_ctx *ctx, int value_type, int index_type, const tf_amg_options *opt, tf_amg **out);
int tf_amg_destroy(tf_amg *m);
/* Amg::setup (Amg.cuh:81-143); transactional: on failure the previous
 * hierarchy is kept. */
int tf_amg_setup(tf_amg *m, const tf_csr *a);
/* Amg::apply (Amg.cuh:149-161): x = M^-1 rhs from a zero guess; device
 * vectors of the component's T; rhs and x may alias. */
int tf_amg_apply(tf_amg *m, const void *rhs, void *x);
int tf_amg_level_count(const tf_amg *m);
/* Level statistics (AmgLevelStatistics, Amg.cuh:27-31). */
int tf_amg_level_stats(const tf_amg *m, int level, int64_t *rows, int64_t *nnz, int32_t histogram[4]);
const char *tf_amg_stop_reason(const tf_amg *m);
const char *tf_amg_coarse_solver(const tf_amg *m);
/* Visits per level of the last apply (Amg::lastCycleVisits). */
int tf_amg_last_visits(const tf_amg *m, int64_t *visits, int capacity);
/* Setup time per phase of the last setup, in ms from CUDA events on the
 * context stream (no reference counterpart; the reference driver times the
 * whole setup with std::chrono, example/solve-matrix.cu:125-128): up to
 * `capacity` of tf_amg_setup_phase_count() values, named by
 * tf_amg_setup_phase_name (level copies and diagonals, column and sliced
 * copies, SpMV shape tuning, strength graphs, aggregation, Galerkin
 * products, coarse LU, small-level region, layout selection). */
int tf_amg_setup_phases(const tf_amg *m, double *ms, int capacity);
int tf_amg_setup_phase_count(void);
const char *tf_amg_setup_phase_name(int phase);
/* Level operator and transfer of the hierarchy (read-only device views). */
int tf_amg_level_matrix(const tf_amg *m, int level, tf_csr *out);
/* y = A_level x with the level's operator as the cycle streams it (its
 * storage type and column stream); x, y device vectors of the hierarchy's
 * storage type, not aliased. */
int tf_amg_level_spmv(const tf_amg *amg, int level, const void *x, void *y);
/* The storage that SpMV streams (no reference counterpart): *sliced = 1
 * for the operator's sliced copy (32-row slices, entries column-major,
 * 2-byte column offsets; *entries counts its padding too), 2 for a sliced
 * copy whose rows are ordered longest first within each 256-row tile, 3 for
 * a banded copy (32-row slices whose rows share one column offset per entry
 * slot: values plus one 8-byte {offset, padding mask} pair per 32 entries),
 * 0 for the CSR arrays with 2-byte column offsets, 4 for the CSR arrays with
 * their 4-byte column indices (*entries = nnz for 0 and 4). */
int tf_amg_level_spmv_layout(const tf_amg *m, int level, int *sliced, int64_t *entries);
int tf_amg_level_transfer(const tf_amg *m, int level, const int32_t **map, const int32_t **offsets,
                          const int32_t **members, int *coarse_rows);

/* The coarse level's factor (CoarseFactor, include/Multigrid/
 * GpuAggregation.cuh:19-25, which the reference's tests read directly):
 * *rows x *rows FP64 LU, row-major, unit lower part below the diagonal, and
 * the pivot row chosen at each step, both device arrays owned by the
 * hierarchy; *rows = 0 (NULL arrays) when the coarse solve is Jacobi. */
int tf_amg_coarse_factor(const tf_amg *m, int *rows, const double **lu, const int32_t **pivots);
/* Hierarchy checkpoint (no reference counterpart; the reference rebuilds
 * the hierarchy on every setup): tf_amg_save writes the built hierarchy --
 * every level's operator in its storage type, its damped inverse diagonal,
 * the aggregates, the coarse factor and the level statistics -- to a file;
 * tf_amg_load restores it into a component created with the same value,
 * index and hierarchy types and the same smoothing (TF_ERR_INVALID
 * otherwise, and for a truncated or foreign file), re-deriving the column
 * copies, launch shapes and small-level region as setup does, so that the
 * restored component applies with the same bits.  Load is transactional:
 * on failure the previous hierarchy is kept. */
int tf_amg_save(const tf_amg *m, const char *path);
int tf_amg_load(tf_amg *m, const char *path);

/* Jacobi smoother component (Jacobi.cuh:26-93). */
typedef struct tf_jacobi tf_jacobi;
int tf_jacobi_create(tf_ctx *ctx, int value_type, int index_type, int sweeps, double weight, tf_jacobi **out);
int tf_jacobi_destroy(tf_jacobi *j);
int tf_jacobi_setup(tf_jacobi *j, const tf_csr *a);
/* x updated from its current value; rhs and x may alias. */
int tf_jacobi_apply(tf_jacobi *j, const void *rhs, void *x);

/* Solver components: kind 0 = PCG (Cg.cuh), 1 = right-preconditioned
 * BiCGStab (BiCgStab.cuh).  precond 0 = Identity, 1 = AMG with amg_opt. */
typedef struct {
    int max_iterations;          /* default 1000 */
    double relative_tolerance;   /* default 1e-8 (f64) / 1e-5 (f32) */
    double absolute_tolerance;   /* default 0 */
    int residual_refresh_interval; /* default 50 */
} tf_solver_options;
void tf_solver_options_default(int value_type, tf_solver_options *o);

typedef struct {
    int status;      /* TF_CONVERGED ... */
    int iterations;
    double residual_norm;
    double relative_residual;
} tf_solve_result;

#define TF_SOLVER_CG 0
#define TF_SOLVER_BICGSTAB 1
#define TF_PRECOND_IDENTITY 0
#define TF_PRECOND_AMG 1
typedef struct tf_solver tf_solver;
int tf_solver_create(tf_ctx *ctx, int kind, int value_type, int index_type, const tf_solver_options *opt,
                     int precond, const tf_amg_options *amg_opt, tf_solver **out);
int tf_solver_destroy(tf_solver *s);
/* Solver::setup (Cg.cuh:63-70, BiCgStab.cuh:70-77); a failed setup leaves
 * the solver unusable until the next successful setup. */
int tf_solver_setup(tf_solver *s, const tf_csr *a);
/* Solver::apply: x holds the initial guess on entry; rhs and x may alias.
 * Device or host pointers: host_buffers != 0 means rhs/x are host memory
 * (pinned or pageable) and the copies run inside the call. */
int tf_solver_apply(tf_solver *s, const void *rhs, void *x, int host_buffers, tf_solve_result *result);
/* Execution mode of apply: 1 (default) runs the whole solve as one CUDA
 * graph whose iteration loop is a conditional WHILE node (no host round trip
 * per iteration); 0 launches one graph per iteration from a host loop that
 * reads a 4-byte running flag.  Same kernels, same results; mode 0 exists for
 * profilers that cannot look inside conditional graph nodes. */
int tf_solver_set_graph_mode(tf_solver *s, int mode);
/* y = A x with the solver's own copy of the operator, as its iterations
 * stream it (IterationContext::multiply, IterationContext.cu:140-159, on the
 * snapshot taken by setup); x, y device vectors of the solver's value type,
 * not aliased.  TF_ERR_LOGIC before setup. */
int tf_solver_spmv(tf_solver *s, const void *x, void *y);
/* The storage tf_solver_spmv streams, as tf_amg_level_spmv_layout says;
 * TF_ERR_LOGIC before setup. */
int tf_solver_spmv_layout(const tf_solver *s, int *sliced, int64_t *entries);
/* How the last apply ran: 2 as one whole-solve graph, 1 as one graph per
 * iteration, 0 as uncaptured launches (a step CUDA refused to
 * capture), -1 before the first apply or for a NULL solver.  No reference
 * counterpart (the reference launches from the host). */
int tf_solver_last_execution(const tf_solver *s);
/* The AMG preconditioner owned by the solver, or NULL for Identity. */
tf_amg *tf_solver_amg(tf_solver *s);
/* Device time of the last apply in milliseconds (CUDA events on the ctx stream). */
double tf_solver_last_apply_ms(const tf_solver *s);

/* ---- Batched solves (no reference counterpart) ---------------------------
 * Many independent systems solved together: every solver's whole solve
 * (its own hierarchy, Krylov loop and convergence test) becomes one branch
 * of a single CUDA graph, so one apply is one graph launch in which the
 * systems run concurrently -- the transient use case of many small problems
 * per time step.  The batch borrows set-up solvers that share its context
 * (they must outlive it); a solver set up again after the graph was built
 * makes the next apply rebuild it.  rhs[k] / x[k] are device vectors of
 * solver k (x[k] is its initial guess and receives its solution);
 * results[k] is its report.  Each system's iterations and results are those
 * of tf_solver_apply on it alone. */
typedef struct tf_batch tf_batch;
int tf_batch_create(tf_ctx *ctx, int count, tf_solver *const *solvers, tf_batch **out);
int tf_batch_destroy(tf_batch *b);
int tf_batch_apply(tf_batch *b, const void *const *rhs, void *const *x, tf_solve_result *results);

/* ---- Learned per-row damping (no reference counterpart) -----------------
 * A 2-layer MLP (4 row features -> 32 ReLU units -> 1, BF16 weights, FP32
 * accumulation) maps each row of a level operator to a Jacobi damping
 * omega_i = omega_min + (omega_max - omega_min) * sigmoid(z).  Features
 * (tf_row_features, n x 4 floats, row-major): log(|a_ii| / mean_j |a_jj|),
 * sum_j!=i |a_ij| / |a_ii|, row nonzeros / 8, level index / 10.  Training is
 * on the GPU with the library's own kernels: tf_mlp_backward accumulates the
 * gradient of the mean squared error to per-row targets (deterministic,
 * fixed reduction order), tf_mlp_sgd takes a momentum step on the FP32
 * master weights with the mean gradient and clears it.  A new model starts
 * near omega = 2/3 (the fixed-weight smoother) for every row.  Parameters
 * (TF_MLP_PARAMS floats): W1[32][4], b1[32], w2[32], b2. */
#define TF_MLP_FEATURES 4
#define TF_MLP_HIDDEN 32
#define TF_MLP_PARAMS (TF_MLP_HIDDEN * TF_MLP_FEATURES + 2 * TF_MLP_HIDDEN + 1)
int tf_mlp_create(tf_ctx *ctx, uint64_t seed, double omega_min, double omega_max, tf_mlp **out);
int tf_mlp_destroy(tf_mlp *m);
int tf_mlp_get_params(const tf_mlp *m, float *host_params);
int tf_mlp_set_params(tf_mlp *m, const float *host_params);
int tf_mlp_bounds(const tf_mlp *m, double *omega_min, double *omega_max);
int tf_row_features(tf_ctx *ctx, const tf_csr *a, int level, float *features);
/* omega (n floats, device) from features (n x 4, device); BF16 weights. */
int tf_mlp_forward(tf_mlp *m, int64_t n, const float *features, float *omega);
/* Adds the gradient of sum_i (omega_i - target_i)^2 over the batch to the
 * model's accumulator; *loss (nullable) = the batch's mean squared error. */
int tf_mlp_backward(tf_mlp *m, int64_t n, const float *features, const float *target, double *loss);
/* The accumulated gradient sums (TF_MLP_PARAMS doubles, host). */
int tf_mlp_get_gradient(const tf_mlp *m, double *host_gradient);
int tf_mlp_sgd(tf_mlp *m, double lr, double momentum);

/* ---- Matrix Market input (include/IO/MatrixMarket.cuh:14-31) ----------- */
typedef struct {
    int rows, cols;
    int64_t nnz;
    int32_t *offsets;
    int32_t *indices;
    double *values;
} tf_host_csr;
/* Parses coordinate real|integer general|symmetric text; duplicates kept in
 * input order, symmetric triangles expanded (src/IO/MatrixMarket.cu:35-122).
 * TF_ERR_RUNTIME with tf_last_error() on malformed input. */
int tf_read_matrix_market(const char *text, size_t length, tf_host_csr *out);
int tf_read_matrix_market_file(const char *path, tf_host_csr *out);
/* The same reader over a caller's byte source (the std::istream overload of
 * io::readMatrixMarket, include/IO/MatrixMarket.cuh:30): read() fills up to
 * `capacity` bytes of buf and returns how many, 0 at the end of the input,
 * (size_t)-1 on a read error ("Matrix Market input read failure"). */
int tf_read_matrix_market_stream(size_t (*read)(void *user, char *buf, size_t capacity), void *user,
                                 tf_host_csr *out);
void tf_host_csr_free(tf_host_csr *m);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
