/*
 * oracle.h -- CPU restatement of ThermoFEM's sparse solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle the CUDA path is tested against:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it.  Nothing in the product (thermofem_b200/) links, imports or calls it.
 *
 * Every function restates the reference behaviour cited beside it
 * (paths are inside the Mgepahmge/ThermoFEM project):
 *   - aggregation setup: src/Multigrid/GpuAggregation.cu and the host
 *     statement of the same algorithm in test/support/NativeAggregationOracle.cu
 *   - V/W/F cycle: include/Multigrid/Cycle.cuh:35-63, Amg.cuh:81-257
 *   - Jacobi: include/Smoother/Jacobi.cuh:60-74, IterationContext.cu:26-32
 *   - PCG: include/Solver/Cg.cuh:105-189
 *   - BiCGStab: include/Solver/BiCgStab.cuh:122-247
 *
 * Parity is pinned: tests/test_oracle_pin.py checks this restatement against
 * the reference's own NativeAggregationOracle compiled from its sources
 * (oracle/Makefile -> oracle/_ref/) and against committed golden fixtures
 * under tests/golden/ generated from that build.
 *
 * Floating point: compiled with -ffp-contract=off; sums run left to right in
 * the stable-sorted entry order the reference host oracle uses.
 */
#ifndef THERMOFEM_ORACLE_H
#define THERMOFEM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (same values as the product C-ABI for readability). */
#define OR_OK 0
#define OR_INVALID (-1)
#define OR_NONFINITE (-7)
#define OR_LENGTH (-3)

/* Host CSR owned by the oracle (malloc'd arrays, free with or_csr_free). */
typedef struct {
    int rows, cols;
    int64_t nnz;
    int *offsets;
    int *indices;
    double *values;
} or_csr;

void or_csr_free(or_csr *a);
void or_free(void *p);

/* --- aggregation setup (GpuAggregation.cu:991-1025; oracle :119-318) ---- */
int or_canonical(int n, const int *rp, const int *ci, const double *v, int64_t nnz, or_csr *out);
/* Row max |offdiag| and diagonal validity (GpuAggregation.cu:247-271). */
int or_validate(const or_csr *a, double *row_max);
int or_strength(const or_csr *a, double theta, or_csr *graph);
int or_match_pairs(const or_csr *g, int rounds, int *map, int *count);
int or_contract(const or_csr *g, const int *map, int count, or_csr *out);
/* aggregate: map[n], offsets[n+1], members[n], *coarse, hist[4]. */
int or_aggregate(const or_csr *g, int rounds, int absorb, int *map, int *offsets, int *members, int *coarse,
                 int64_t hist[4]);
int or_galerkin(const or_csr *a, const int *map, int coarse, or_csr *out);

/* --- dense coarse LU (GpuAggregation.cu:827-939) ------------------------ */
/* lu[n*n] row major, pivots[n]; returns 1 when factored, 0 when singular. */
int or_lu_factor(const or_csr *a, double *lu, int *pivots);
void or_lu_solve(int n, const double *lu, const int *pivots, const double *b, double *x);

/* --- kernels of the iteration (IterationContext.cu) --------------------- */
void or_spmv(const or_csr *a, const double *x, double *y);
double or_dot(int64_t n, const double *x, const double *y);
double or_norm(int64_t n, const double *x);

/* --- AMG hierarchy + cycle (Amg.cuh:81-257, Cycle.cuh:35-63) ----------- */
typedef struct {
    int max_levels, coarse_rows, matching_rounds, pre_sweeps, post_sweeps, coarse_sweeps;
    double jacobi_weight, strength_threshold;
    int absorb_singletons;
    int cycle;         /* 0 V, 1 W, 2 F */
    int coarse_lu_rows; /* LU used when the last level has <= this many rows (reference: 64) */
} or_amg_options;

typedef struct or_amg or_amg;
/* Builds the hierarchy; *status = OR_OK or an error code. */
or_amg *or_amg_setup(const or_csr *a, const or_amg_options *opt, int *status);
void or_amg_free(or_amg *m);
int or_amg_levels(const or_amg *m);
/* rows, nnz, hist[4] of level d; stop reason / coarse solver strings. */
void or_amg_level_info(const or_amg *m, int d, int64_t *rows, int64_t *nnz, int64_t hist[4]);
const char *or_amg_stop_reason(const or_amg *m);
const char *or_amg_coarse_solver(const or_amg *m);
/* Transfer of level d (map into level d+1): returns pointers owned by m. */
const int *or_amg_map(const or_amg *m, int d);
const or_csr *or_amg_matrix(const or_amg *m, int d);
/* One preconditioner application from a zero guess; visits[levels] out (may be NULL). */
void or_amg_apply(or_amg *m, const double *rhs, double *x, int64_t *visits);

/* --- Krylov solvers (Cg.cuh, BiCgStab.cuh) ------------------------------ */
typedef struct {
    int status; /* 0 Converged, 1 MaxIterations, 2 Breakdown, 3 NonFinite */
    int iterations;
    double residual_norm, relative_residual;
} or_solve_result;

typedef struct {
    int max_iterations;
    double relative_tolerance, absolute_tolerance;
    int refresh_interval;
} or_solver_options;

/* precond == NULL means Identity.  x holds the initial guess on entry. */
or_solve_result or_cg(const or_csr *a, or_amg *precond, const double *b, double *x, const or_solver_options *opt);
or_solve_result or_bicgstab(const or_csr *a, or_amg *precond, const double *b, double *x,
                            const or_solver_options *opt);

/* --- Jacobi smoother (Jacobi.cuh:60-74) -------------------------------- */
int or_jacobi(const or_csr *a, int sweeps, double weight, const double *b, double *x);

/* --- test input generators --------------------------------------------- */
/* sample(n) of the reference's aggregation sweep (amg_native_test.cpp:28-52),
 * driven by the MT19937 32-bit generator seeded with 173+n. */
int or_sample_matrix(int n, or_csr *out);
/* Raw MT19937 stream, for pinning the generator against std::mt19937. */
void or_mt19937(uint32_t seed, int count, uint32_t *out);

int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
