// coarse.cu -- coarsest-level direct solve.
//
// Factor: the reference's partial-pivot LU (src/Multigrid/GpuAggregation.cu:
// 827-893) on one CTA, with the same pivot rule (first largest |a_ik|, full
// row swaps) and the same singularity threshold 64 * DBL_EPSILON * max|A|,
// but for up to 256 rows: the dense matrix lives in shared memory up to 160
// rows (200 KB of the 227 KB per CTA) and in L2-resident global memory above.
// The elimination of step k is spread over all (row, column) pairs of the
// trailing block instead of one thread per row.
//
// Solve: the reference permutes and substitutes with a __syncthreads per
// row (GpuAggregation.cu:904-939), i.e. 2n barriers on every coarse visit.
// tf_coarse_lu_solve keeps that algorithm; the AMG cycle instead applies an
// explicit inverse built once from the factor (n independent substitutions
// at setup), a dense mat-vec that costs one pass over n^2 doubles in L2.
#include "ops.cuh"

#include <cfloat>

namespace tfb {
namespace {

constexpr int kLuThreads = 1024;
constexpr int kSmemRows = 160;

__global__ void __launch_bounds__(kLuThreads) lu_factor_kernel(int n, const int32_t *__restrict__ rp,
                                                                 const int32_t *__restrict__ ci,
                                                                 const double *__restrict__ a, double *lu,
                                                                 int32_t *pivots, int *bad, int use_smem) {
    pdl_enter();
    extern __shared__ __align__(16) double dyn[];
    __shared__ double red_v[kLuThreads / 32];
    __shared__ int red_i[kLuThreads / 32];
    __shared__ double scale;
    __shared__ int pivot, failed;
    double *m = use_smem ? dyn : lu;
    const int tid = threadIdx.x;
    const int nn = n * n;
    for (int e = tid; e < nn; e += blockDim.x) m[e] = 0.0;
    __syncthreads();
    double mx = 0;
    for (int r = tid; r < n; r += blockDim.x)
        for (int32_t j = rp[r]; j < rp[r + 1]; ++j) {
            m[r * n + ci[j]] = a[j];
            mx = fmax(mx, fabs(a[j]));
        }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((tid & 31) == 0) red_v[tid >> 5] = mx;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s = fmax(s, red_v[w]);
        scale = s;
        failed = 0;
        *bad = 0;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        // Pivot: largest |m[i][k]|, smallest i on ties (the sequential
        // "strictly greater" scan of the reference).
        double bv = -1.0;
        int bi = n;
        for (int i = k + tid; i < n; i += blockDim.x) {
            const double v = fabs(m[i * n + k]);
            if (v > bv) {
                bv = v;
                bi = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if ((tid & 31) == 0) {
            red_v[tid >> 5] = bv;
            red_i[tid >> 5] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double v = red_v[0];
            int p = red_i[0];
            for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w)
                if (red_v[w] > v || (red_v[w] == v && red_i[w] < p)) {
                    v = red_v[w];
                    p = red_i[w];
                }
            if (p >= n) p = k;  // every candidate was NaN: keep k (sequential rule)
            const double pv = m[p * n + k];
            if (!isfinite(pv) || fabs(pv) <= 64 * DBL_EPSILON * scale) failed = 1;
            pivot = p;
            pivots[k] = p;
        }
        __syncthreads();
        if (failed) {
            if (tid == 0) *bad = 1;
            return;
        }
        const int p = pivot;
        if (p != k)
            for (int j = tid; j < n; j += blockDim.x) {
                const double t = m[p * n + j];
                m[p * n + j] = m[k * n + j];
                m[k * n + j] = t;
            }
        __syncthreads();
        for (int r = k + 1 + tid; r < n; r += blockDim.x) m[r * n + k] /= m[k * n + k];
        __syncthreads();
        const int w = n - k - 1;
        for (int e = tid; e < w * w; e += blockDim.x) {
            const int r = k + 1 + e / w, j = k + 1 + e % w;
            m[r * n + j] -= m[r * n + k] * m[k * n + j];
        }
        __syncthreads();
    }
    for (int e = tid; e < nn; e += blockDim.x) {
        if (use_smem) lu[e] = m[e];
        if (!isfinite(m[e])) atomicExch(bad, 1);
    }
}

// Reference triangular solve (GpuAggregation.cu:904-939): permutation, then
// column-oriented forward and back substitution; b and x may alias.
template <class T>
__global__ void lu_solve_kernel(int n, const double *__restrict__ lu, const int32_t *__restrict__ pivots, const T *b,
                                T *x) {
    pdl_enter();
    __shared__ double v[256];
    const int row = threadIdx.x;
    if (row < n) v[row] = static_cast<double>(b[row]);
    __syncthreads();
    if (row == 0)
        for (int k = 0; k < n; ++k) {
            const double t = v[k];
            v[k] = v[pivots[k]];
            v[pivots[k]] = t;
        }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (row > k && row < n) v[row] -= lu[row * n + k] * v[k];
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
        if (row == k) v[row] /= lu[row * n + row];
        __syncthreads();
        if (row < k) v[row] -= lu[row * n + k] * v[k];
        __syncthreads();
    }
    if (row < n) x[row] = static_cast<T>(v[row]);
}

// Column c of A^-1 = U^-1 L^-1 P e_c, one thread per column.
__global__ void lu_inverse_kernel(int n, const double *__restrict__ lu, const int32_t *__restrict__ pivots,
                                  double *__restrict__ inv /* row major */, double *__restrict__ work) {
    pdl_enter();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double *v = work + static_cast<int64_t>(c) * n;
    for (int i = 0; i < n; ++i) v[i] = (i == c) ? 1.0 : 0.0;
    for (int k = 0; k < n; ++k) {
        const double t = v[k];
        v[k] = v[pivots[k]];
        v[pivots[k]] = t;
    }
    for (int k = 0; k < n; ++k)
        for (int r = k + 1; r < n; ++r) v[r] -= lu[r * n + k] * v[k];
    for (int k = n - 1; k >= 0; --k) {
        v[k] /= lu[k * n + k];
        for (int r = 0; r < k; ++r) v[r] -= lu[r * n + k] * v[k];
    }
    for (int i = 0; i < n; ++i) inv[static_cast<int64_t>(i) * n + c] = v[i];
}

// x = inv * b, one warp per row, FP64 accumulation.
template <class T>
__global__ void dense_apply_kernel(int n, const double *__restrict__ inv, const T *__restrict__ b, T *__restrict__ x) {
    pdl_enter();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    double s = 0;
    for (int j = lane; j < n; j += 32) s += inv[static_cast<int64_t>(warp) * n + j] * static_cast<double>(b[j]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) x[warp] = static_cast<T>(s);
}

// dense_apply_kernel between a restriction and a prolongation.  Every CTA
// restricts all n (<= 256) coarse values itself (restrict_kernel's order);
// CTA 0 stores them.
template <class T>
__global__ void dense_fused_kernel(int n, const double *__restrict__ inv, T *__restrict__ b, T *__restrict__ x,
                                   const T *__restrict__ rfine, const int32_t *__restrict__ roff,
                                   const int32_t *__restrict__ rmem, const int32_t *__restrict__ soff,
                                   const int32_t *__restrict__ smem, T *__restrict__ fine) {
    pdl_enter();
    __shared__ T sb[256];
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        T v;
        if (rfine) {
            v = 0;
            for (int32_t j = roff[c]; j < roff[c + 1]; ++j) v += rfine[rmem[j]];
            if (blockIdx.x == 0) b[c] = v;
        } else {
            v = b[c];
        }
        sb[c] = v;
    }
    __syncthreads();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    double s = 0;
    for (int j = lane; j < n; j += 32) s += inv[static_cast<int64_t>(warp) * n + j] * static_cast<double>(sb[j]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const T v = static_cast<T>(__shfl_sync(0xffffffffu, s, 0));
    if (lane == 0) x[warp] = v;
    if (fine)
        for (int32_t k = soff[warp] + lane; k < soff[warp + 1]; k += 32) fine[smem[k]] += v;
}

}  // namespace

bool coarse_lu_factor(tf_ctx *ctx, const Csr<double, int32_t> &a, double *lu, int32_t *pivots) {
    const int n = static_cast<int>(a.rows);
    require(n >= 1 && n <= 256 && a.rows == a.cols, "GPU LU requires order 1..256");
    const bool smem = n <= kSmemRows;
    const size_t bytes = smem ? static_cast<size_t>(n) * n * sizeof(double) : 0;
    // the attribute is per function and device for the whole process: set
    // it to the largest size any order needs, so no caller lowers it under
    // another thread's launch
    constexpr size_t kMaxBytes = static_cast<size_t>(kSmemRows) * kSmemRows * sizeof(double);
    if (bytes > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(lu_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kMaxBytes)),
                   "LU shared memory");
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    launch_kernel(ctx, "lu_factor", lu_factor_kernel, 1, kLuThreads, bytes, n, a.rp, a.ci, a.val, lu, pivots, bad,
                  smem ? 1 : 0);
    return read_scalar(ctx, bad) == 0;
}

template <class T>
void coarse_lu_solve(tf_ctx *ctx, int n, const double *lu, const int32_t *pivots, const T *b, T *x) {
    require(n >= 1 && n <= 256, "Invalid GPU coarse solve");
    launch_kernel(ctx, "lu_solve", lu_solve_kernel<T>, 1, 256, 0, n, lu, pivots, b, x);
}

void coarse_inverse(tf_ctx *ctx, int n, const double *lu, const int32_t *pivots, double *inv) {
    double *work = static_cast<double *>(ctx->arena(static_cast<size_t>(n) * n * sizeof(double), 1));
    launch_kernel(ctx, "lu_inverse", lu_inverse_kernel, grid_for(n, 64), 64, 0, n, lu, pivots, inv, work);
}

template <class T>
void coarse_dense_apply(tf_ctx *ctx, int n, const double *inv, const T *b, T *x) {
    launch_kernel(ctx, "coarse_apply", dense_apply_kernel<T>, grid_for(static_cast<int64_t>(n) * 32), kBlock, 0, n, inv,
                  b, x);
}

template <class T>
void coarse_dense_apply_fused(tf_ctx *ctx, int n, const double *inv, T *b, T *x, const T *rfine, const int32_t *roff,
                              const int32_t *rmem, const int32_t *soff, const int32_t *smem, T *fine) {
    require(n >= 1 && n <= 256, "dense coarse solve requires order 1..256");
    launch_kernel(ctx, "coarse_apply_fused", dense_fused_kernel<T>, grid_for(static_cast<int64_t>(n) * 32), kBlock, 0,
                  n, inv, b, x, rfine, roff, rmem, soff, smem, fine);
}

template void coarse_dense_apply_fused<float>(tf_ctx *, int, const double *, float *, float *, const float *,
                                              const int32_t *, const int32_t *, const int32_t *, const int32_t *,
                                              float *);
template void coarse_dense_apply_fused<double>(tf_ctx *, int, const double *, double *, double *, const double *,
                                               const int32_t *, const int32_t *, const int32_t *, const int32_t *,
                                               double *);
template void coarse_lu_solve<float>(tf_ctx *, int, const double *, const int32_t *, const float *, float *);
template void coarse_lu_solve<double>(tf_ctx *, int, const double *, const int32_t *, const double *, double *);
template void coarse_dense_apply<float>(tf_ctx *, int, const double *, const float *, float *);
template void coarse_dense_apply<double>(tf_ctx *, int, const double *, const double *, double *);

}  // namespace tfb
