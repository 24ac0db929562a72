// spmv.cu -- the SpMV family on the row-tile kernels (tile.cuh) and the
// vector kernels around it.
//
// The epilogue is a template parameter, so the residual, the weighted-Jacobi
// sweep and the prolongation-fused sweep read A exactly once per pass: the
// reference does SpMV + scal + axpy (src/LinearAlgebra/IterationContext.cu:
// 167-175) and SpMV + update (:26-32,251-269) as separate passes.  Each
// epilogue's pre() loads the row's own operands (issued at the start of the
// row's tile so their latency overlaps the gathers).
#include <cstdlib>
#include <cstring>

#include "tile.cuh"

namespace tfb {
namespace {

using tile::PlainX;
using tile::ProlongX;

template <class T>
struct StoreY {
    static constexpr int kReduce = 0;
    struct Pre {};
    T *__restrict__ y;
    double *partial{nullptr};
    __device__ __forceinline__ bool skip() const { return false; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t, const XS &) const {
        return {};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &, double (&)[1]) const { y[i] = acc; }
};

template <class T>
struct ResidualOut {
    static constexpr int kReduce = 0;
    struct Pre {
        T b;
    };
    const T *__restrict__ b;
    T *__restrict__ r;
    double *partial{nullptr};
    __device__ __forceinline__ bool skip() const { return false; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &) const {
        return {b[i]};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&)[1]) const {
        r[i] = p.b - acc;
    }
};

// x_out = x~ + (w Dinv) (b - A x~), the reference's update expression
// x += w * d * (b - a) (IterationContext.cu:26-32).
template <class T>
struct JacobiOut {
    static constexpr int kReduce = 0;
    struct Pre {
        T x, d, b, w;
    };
    const T *__restrict__ dinv;
    const T *__restrict__ b;
    T *__restrict__ xo;
    const float *__restrict__ row_w;
    T w;
    double *partial{nullptr};
    __device__ __forceinline__ bool skip() const { return false; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &xs) const {
        return {xs(i), dinv[i], b[i], row_w ? static_cast<T>(row_w[i]) : w};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&)[1]) const {
        xo[i] = p.x + p.w * p.d * (p.b - acc);
    }
};

// A post-smoothing sweep of a coarse level that also applies the
// prolongation of its result to the fine level: row c's new value is added
// to x_fine at every member of aggregate c (fine[m] += coarse[c], the same
// addition as prolong_kernel; each fine row belongs to one aggregate, so the
// scatter has no conflicts and no ordering to fix).
template <class T>
struct JacobiScatter {
    static constexpr int kReduce = 0;
    struct Pre {
        T x, d, b;
        int32_t m0, m1;
    };
    const T *__restrict__ dinv;
    const T *__restrict__ b;
    T *__restrict__ xo;
    T w;
    const int32_t *__restrict__ off;  // aggregate -> members (fine rows)
    const int32_t *__restrict__ mem;
    T *__restrict__ fine;
    double *partial{nullptr};
    __device__ __forceinline__ bool skip() const { return false; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &xs) const {
        return {xs(i), dinv[i], b[i], off[i], off[i + 1]};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&)[1]) const {
        const T v = p.x + w * p.d * (p.b - acc);
        xo[i] = v;
        for (int32_t k = p.m0; k < p.m1; ++k) fine[mem[k]] += v;
    }
};

template <class T, class I, class V, class XS, class Epi>
void launch_tile(tf_ctx *ctx, const Csr<T, I, V> &a, const XS &xs, const Epi &epi, const char *name) {
    tile::launch(ctx, a, xs, epi, name);
}


template <class T>
__global__ void jacobi_zero_kernel(int64_t n, const T *__restrict__ dinv, const T *__restrict__ b, T *__restrict__ x,
                                   T w, const float *__restrict__ row_w) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const T wi = row_w ? static_cast<T>(row_w[i]) : w;
        // x = 0 + w d (b - 0), the reference update from a zero guess.
        x[i] = wi * dinv[i] * b[i];
    }
}

// *bad = 1 when some idx[i] lies outside [0, limit).
__global__ void index_range_kernel(int64_t n, const int32_t *__restrict__ idx, int32_t limit, int *bad) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (idx[i] < 0 || idx[i] >= limit) atomicExch(bad, 1);
}

// x += w d (b - ax) with ax = A x computed before (IterationContext::jacobi,
// src/LinearAlgebra/IterationContext.cu:26-32,251-269): the Jacobi update on
// its own, for callers that form A x themselves.
template <class T>
__global__ void jacobi_update_kernel(int64_t n, T w, const T *__restrict__ dinv, const T *__restrict__ b,
                                     const T *__restrict__ ax, T *__restrict__ x) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[i] += w * dinv[i] * (b[i] - ax[i]);
}

template <class T, class I, class V>
__global__ void inverse_diagonal_kernel(int64_t n, const I *__restrict__ rp, const I *__restrict__ ci,
                                        const V *__restrict__ val, T *__restrict__ dinv, int *bad) {
    pdl_enter();
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    T d = 0;
    for (I j = rp[i]; j < rp[i + 1]; ++j)
        if (static_cast<int64_t>(ci[j]) == i) d += val[j];
    const T inv = T(1) / d;
    if (!isfinite(d) || d == T(0) || !isfinite(inv)) atomicExch(bad, 1);
    dinv[i] = inv;
}

template <class T>
__global__ void restrict_kernel(int64_t nc, const int32_t *__restrict__ off, const int32_t *__restrict__ mem,
                                const T *__restrict__ fine, T *__restrict__ coarse) {
    pdl_enter();
    const int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (c >= nc) return;
    T s = 0;
    for (int32_t j = off[c]; j < off[c + 1]; ++j) s += fine[mem[j]];
    coarse[c] = s;
}

// Restriction of a fine vector into the coarse right-hand side fused with
// the zero-guess sweep that follows it: b[c] = sum of fine[m] over the
// members of aggregate c (restrict_kernel's order), x[c] = w d[c] b[c]
// (jacobi_zero_kernel's expression).
template <class T>
__global__ void restrict_jacobi_zero_kernel(int64_t nc, const int32_t *__restrict__ off,
                                            const int32_t *__restrict__ mem, const T *__restrict__ fine,
                                            T *__restrict__ b, const T *__restrict__ dinv, T *__restrict__ x, T w) {
    pdl_enter();
    const int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (c >= nc) return;
    T s = 0;
    for (int32_t j = off[c]; j < off[c + 1]; ++j) s += fine[mem[j]];
    b[c] = s;
    x[c] = w * dinv[c] * s;
}

template <class I>
__global__ void delta_columns_kernel(int64_t n, const I *__restrict__ rp, const I *__restrict__ ci,
                                     int16_t *__restrict__ cd, int *bad) {
    pdl_enter();
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    for (I j = rp[i]; j < rp[i + 1]; ++j) {
        const int64_t d = static_cast<int64_t>(ci[j]) - i;
        if (d < -32767 || d > 32767) {
            atomicExch(bad, 1);
            return;
        }
        cd[j] = static_cast<int16_t>(d);
    }
}

// Row order of the sorted sliced layout: within each 256-row tile, rows by
// decreasing length, ties by row (a rank by counting; one CTA per tile).
template <class I>
__global__ void slice_sort_kernel(int64_t rows, const I *__restrict__ rp, int32_t *__restrict__ perm) {
    pdl_enter();
    __shared__ int64_t len[256];
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * 256;
    const int nr = static_cast<int>(rows - r0 < 256 ? rows - r0 : 256);
    const int t = threadIdx.x;
    if (t < nr) len[t] = static_cast<int64_t>(rp[r0 + t + 1] - rp[r0 + t]);
    __syncthreads();
    if (t >= nr) return;
    const int64_t mine = len[t];
    int rank = 0;
    for (int k = 0; k < nr; ++k) rank += (len[k] > mine || (len[k] == mine && k < t)) ? 1 : 0;
    perm[r0 + rank] = static_cast<int32_t>(r0 + t);
}

// Entries of each 32-row slice of the sliced layout (32 x its longest row),
// one warp per slice, and their total.  Position t holds row perm[t] (or t).
template <class I>
__global__ void slice_entries_kernel(int64_t rows, int64_t nslices, const I *__restrict__ rp,
                                     const int32_t *__restrict__ perm, int32_t *__restrict__ entries,
                                     unsigned long long *total) {
    pdl_enter();
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t s = t >> 5;  // uniform across the warp
    if (s >= nslices) return;
    const int lane = static_cast<int>(t & 31);
    int64_t len = 0;
    if (t < rows) {
        const int64_t row = perm ? perm[t] : t;
        len = static_cast<int64_t>(rp[row + 1] - rp[row]);
    }
    for (int o = 16; o > 0; o >>= 1) len = max(len, static_cast<int64_t>(__shfl_xor_sync(0xffffffffu, len, o)));
    if (lane == 0) {
        const int64_t e = len * 32;
        entries[s] = e > INT32_MAX ? INT32_MAX : static_cast<int32_t>(e);
        atomicAdd(total, static_cast<unsigned long long>(e));
    }
}

// The entries of the row at position t into its slice (column-major,
// padding after its last entry).
template <class T, class I>
__global__ void slice_fill_kernel(int64_t rows, int64_t nslices, const I *__restrict__ rp,
                                  const T *__restrict__ val, const int16_t *__restrict__ cd,
                                  const int32_t *__restrict__ perm, const int32_t *__restrict__ sp,
                                  T *__restrict__ sv, int16_t *__restrict__ sc) {
    pdl_enter();
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t s = t >> 5;
    if (s >= nslices) return;
    const int lane = static_cast<int>(t & 31);
    const int64_t base = sp[s];
    const int64_t width = (static_cast<int64_t>(sp[s + 1]) - base) >> 5;
    int64_t j0 = 0, len = 0;
    if (t < rows) {
        const int64_t row = perm ? perm[t] : t;
        j0 = rp[row];
        len = static_cast<int64_t>(rp[row + 1]) - j0;
    }
    for (int64_t j = 0; j < width; ++j) {
        const int64_t k = base + j * 32 + lane;
        if (j < len) {
            sv[k] = val[j0 + j];
            sc[k] = cd[j0 + j];
        } else {
            sv[k] = T(0);
            sc[k] = kSlicePad;
        }
    }
}

// Banded copy.  A warp walks one slice: lane l holds row 32 s + l and a
// cursor into its (sorted) entries; at each step the warp takes the smallest
// column offset among the lanes' next entries as the slot's shared offset,
// and the lanes whose next entry has it advance.  The slot count is the
// number of distinct offsets of the slice.  bad: 1 a row with unsorted or
// repeated columns, 2 a slice wider than kBandMaxSlots.
constexpr int kBandMaxSlots = 32;

__device__ __forceinline__ int band_next(int64_t p, int64_t e, const int32_t *__restrict__ ci, int row) {
    return p < e ? ci[p] - row : INT_MAX;
}

__global__ void band_width_kernel(int64_t rows, int64_t nslices, const int32_t *__restrict__ rp,
                                  const int32_t *__restrict__ ci, int32_t *__restrict__ entries,
                                  unsigned long long *total, int *bad) {
    pdl_enter();
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t s = t >> 5;  // uniform across the warp
    if (s >= nslices) return;
    const int lane = static_cast<int>(t & 31);
    const int row = static_cast<int>(t);
    int64_t p = 0, e = 0;
    if (t < rows) {
        p = rp[t];
        e = rp[t + 1];
        for (int64_t k = p + 1; k < e; ++k)
            if (ci[k] <= ci[k - 1]) atomicOr(bad, 1);
    }
    int slots = 0;
    for (;;) {
        const int mine = band_next(p, e, ci, row);
        int m = mine;
        for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (m == INT_MAX) break;
        if (mine == m) ++p;
        if (++slots > kBandMaxSlots) {
            if (lane == 0) atomicOr(bad, 2);
            return;
        }
    }
    if (lane == 0) {
        entries[s] = slots * 32;
        atomicAdd(total, static_cast<unsigned long long>(slots) * 32ull);
    }
}

template <class T>
__global__ void band_fill_kernel(int64_t rows, int64_t nslices, const int32_t *__restrict__ rp,
                                 const int32_t *__restrict__ ci, const T *__restrict__ val,
                                 const int32_t *__restrict__ sp, T *__restrict__ sv, int2 *__restrict__ bd) {
    pdl_enter();
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t s = t >> 5;
    if (s >= nslices) return;
    const int lane = static_cast<int>(t & 31);
    const int row = static_cast<int>(t);
    int64_t p = 0, e = 0;
    if (t < rows) {
        p = rp[t];
        e = rp[t + 1];
    }
    const int64_t base = sp[s];
    for (int j = 0;; ++j) {
        const int mine = band_next(p, e, ci, row);
        int m = mine;
        for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (m == INT_MAX) break;
        const bool has = mine == m;
        const unsigned pad = __ballot_sync(0xffffffffu, !has);
        sv[base + j * 32 + lane] = has ? val[p] : T(0);
        if (lane == 0) bd[(base >> 5) + j] = make_int2(m, static_cast<int>(pad));
        if (has) ++p;
    }
}

template <class T>
__global__ void prolong_kernel(int64_t nf, const int32_t *__restrict__ map, const T *__restrict__ coarse,
                               T *__restrict__ fine) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < nf;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        fine[i] += coarse[map[i]];
}

// Deterministic block reduction of up to 4 sums (fixed tree order).
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *shm /* [K][32] */) {
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) shm[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            v[k] = lane < nw ? shm[k * 32 + lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
    }
}

struct DotArgs {
    const void *x[4];
    const void *y[4];
};

template <class T, int K>
__global__ void __launch_bounds__(256) dot_partial_kernel(int64_t n, DotArgs args, double *partial) {
    pdl_enter();
    __shared__ double shm[K * 32];
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            v[k] += static_cast<double>(static_cast<const T *>(args.x[k])[i]) *
                    static_cast<double>(static_cast<const T *>(args.y[k])[i]);
    }
    block_sum<K>(v, shm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) partial[k * gridDim.x + blockIdx.x] = v[k];
}

template <int K>
__global__ void __launch_bounds__(256) dot_final_kernel(int parts, const double *partial, double *out) {
    pdl_enter();
    __shared__ double shm[K * 32];
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        v[k] = 0.0;
        for (int p = threadIdx.x; p < parts; p += blockDim.x) v[k] += partial[k * parts + p];
    }
    block_sum<K>(v, shm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = v[k];
}

// ---- the Krylov solvers' fused vector steps as standalone operations ----
// (the same arithmetic as the solvers' own kernels in krylov.cu; squared
// norms in FP64 over the fixed dot_multi partition, then dot_final_kernel)

// x += alpha p; r -= alpha ap; partial sums of r_i^2 (Cg.cuh:172-174)
template <class T>
__global__ void __launch_bounds__(256) cg_update_kernel(int64_t n, T alpha, const T *__restrict__ p,
                                                        const T *__restrict__ ap, T *__restrict__ x,
                                                        T *__restrict__ r, double *partial) {
    pdl_enter();
    __shared__ double shm[32];
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        x[i] += alpha * p[i];
        const T ri = r[i] - alpha * ap[i];
        r[i] = ri;
        v[0] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    block_sum<1>(v, shm);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// p = z + beta p, or p = z when restarting (Cg.cuh:147-158)
template <class T>
__global__ void cg_direction_kernel(int64_t n, T beta, int restart, const T *__restrict__ z, T *__restrict__ p) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        p[i] = restart ? z[i] : z[i] + beta * p[i];
}

// p = r + beta (p - omega v), or p = r when restarting (BiCgStab.cuh:170-180)
template <class T>
__global__ void bicgstab_direction_kernel(int64_t n, T beta, T omega, int restart, const T *__restrict__ r,
                                          const T *__restrict__ v, T *__restrict__ p) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (restart) {
            p[i] = r[i];
        } else {
            const T t = p[i] - omega * v[i];
            p[i] = r[i] + beta * t;
        }
    }
}

// s = r - alpha v; x += alpha phat; partial sums of s_i^2 (BiCgStab.cuh:195-198)
template <class T>
__global__ void __launch_bounds__(256) bicgstab_s_kernel(int64_t n, T alpha, const T *__restrict__ r,
                                                         const T *__restrict__ v, const T *__restrict__ ph,
                                                         T *__restrict__ x, T *__restrict__ sv, double *partial) {
    pdl_enter();
    __shared__ double shm[32];
    double acc[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const T si = r[i] - alpha * v[i];
        sv[i] = si;
        x[i] += alpha * ph[i];
        acc[0] += static_cast<double>(si) * static_cast<double>(si);
    }
    block_sum<1>(acc, shm);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

// x += omega shat; r = s - omega t; partial sums of r_i^2 (BiCgStab.cuh:228-231)
template <class T>
__global__ void __launch_bounds__(256) bicgstab_update_kernel(int64_t n, T omega, const T *__restrict__ sh,
                                                              const T *__restrict__ sv, const T *__restrict__ t,
                                                              T *__restrict__ x, T *__restrict__ r,
                                                              double *partial) {
    pdl_enter();
    __shared__ double shm[32];
    double acc[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        x[i] += omega * sh[i];
        const T ri = sv[i] - omega * t[i];
        r[i] = ri;
        acc[0] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    block_sum<1>(acc, shm);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

template <class T>
__global__ void axpby_kernel(int64_t n, double a, const T *__restrict__ x, double b, T *__restrict__ y) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const T ta = static_cast<T>(a), tb = static_cast<T>(b);
        y[i] = tb == T(0) ? ta * x[i] : ta * x[i] + tb * y[i];
    }
}

template <class S, class D>
__global__ void convert_kernel(int64_t n, const S *__restrict__ src, D *__restrict__ dst) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<D>(src[i]);
}

template <class I>
__global__ void csr_structure_kernel(int64_t rows, int64_t cols, int64_t nnz, const I *__restrict__ rp,
                                     const I *__restrict__ ci, int *bad) {
    pdl_enter();
    const int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (r == 0 && (rp[0] != 0 || static_cast<int64_t>(rp[rows]) != nnz)) atomicExch(bad, 1);
    if (r >= rows) return;
    const int64_t s = rp[r], e = rp[r + 1];
    if (s < 0 || e < s || e > nnz) {
        atomicExch(bad, 1);
        return;
    }
    for (int64_t j = s; j < e; ++j)
        if (ci[j] < 0 || static_cast<int64_t>(ci[j]) >= cols) atomicExch(bad, 1);
}

// Canonical-form flags (src/Multigrid/GpuAggregation.cu:283-304).
template <class T, class I>
__global__ void canonical_flags_kernel(int64_t n, int64_t nnz, const I *__restrict__ rp, const I *__restrict__ ci,
                                       const T *__restrict__ val, int *flags) {
    pdl_enter();
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    if (rp[0] != 0 || static_cast<int64_t>(rp[n]) != nnz || rp[i] < 0 || rp[i] > rp[i + 1] ||
        static_cast<int64_t>(rp[i + 1]) > nnz) {
        atomicOr(flags, 2);
        return;
    }
    int64_t previous = -1;
    for (I j = rp[i]; j < rp[i + 1]; ++j) {
        const int64_t c = ci[j];
        if (c < 0 || c >= n || !isfinite(val[j])) atomicOr(flags, 2);
        if (c <= previous) atomicOr(flags, 1);
        previous = c;
    }
}

// Level validation and row max |offdiag| (GpuAggregation.cu:247-271).
__global__ void row_stats_kernel(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                 const double *__restrict__ a, int *bad, double *__restrict__ row_max) {
    pdl_enter();
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    double diag = 0, mx = 0;
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
        if (!isfinite(a[j])) atomicExch(bad, 1);
        if (ci[j] == i) diag = a[j];
        else mx = fmax(mx, fabs(a[j]));
    }
    if (diag == 0 || !isfinite(diag) || !isfinite(1.0 / diag)) atomicExch(bad, 1);
    if (row_max) row_max[i] = mx;
}

unsigned stride_grid(tf_ctx *ctx, int64_t n) {
    const int64_t want = (n + kBlock - 1) / kBlock;
    const int64_t cap = static_cast<int64_t>(ctx->sm_count) * 16;
    return static_cast<unsigned>(want < 1 ? 1 : (want > cap ? cap : want));
}

}  // namespace

// One row per thread; the staged chunk holds a typical tile (mean row
// length x 256 rows, +25%) so short-row operators keep up to 8 CTAs per SM
// resident, capped at 48 KB of shared memory for long rows (which then take
// several chunks).  A pure function of (rows, nnz): the Krylov kernels size
// their per-tile partial sums from it.
SpmvShape spmv_shape(int64_t rows, int64_t nnz, size_t value_size, size_t index_size) {
    SpmvShape s;
    s.rows_per_thread = 1;
    const int64_t cap = static_cast<int64_t>(49152 / (value_size + index_size)) & ~int64_t(63);
    const int64_t mean_tile = rows > 0 ? (nnz * 256 + rows - 1) / rows : 0;
    int64_t chunk = (mean_tile + mean_tile / 4 + 63) & ~int64_t(63);
    if (chunk < 512) chunk = 512;
    if (chunk > cap) chunk = cap;
    s.chunk = static_cast<int>(chunk);
    return s;
}

template <class T, class I, class V>
void spmv(tf_ctx *ctx, const Csr<T, I, V> &a, const T *x, T *y) {
    launch_tile(ctx, a, PlainX<T>{x}, StoreY<T>{y, nullptr}, "spmv");
}

template <class T, class I>
void autotune_spmv(tf_ctx *ctx, const Csr<T, I> &a, const T *x, T *y, int *stages, int *ctas_per_sm, int *cap_pct,
                   int *rows_per_thread, float *ms) {
    const tile::PipeConfig c = tile::autotune(ctx, a, x, y, ms);
    if (stages) *stages = c.stages;
    if (ctas_per_sm) *ctas_per_sm = c.ctas_per_sm;
    if (cap_pct) *cap_pct = c.cap_pct;
    if (rows_per_thread) *rows_per_thread = c.rpt;
}

template <class T, class I, class V>
void tune_spmv(tf_ctx *ctx, const Csr<T, I, V> &a, const T *x, T *y) {
    if (!std::getenv("THERMOFEM_B200_SLICED_SHAPE") && tile::tuned(ctx, a)) return;
    tile::autotune(ctx, a, x, y, nullptr);
}

template <class T, class I, class V>
bool streams_sliced(tf_ctx *ctx, const Csr<T, I, V> &a, int64_t entries_if_sliced, int64_t *entries) {
    bool sliced = false;
    if constexpr (std::is_same_v<I, int32_t>) {
        if (a.sp && (a.cd || a.bd)) sliced = tile::copy_config(ctx, a).sliced != 0;
    }
    *entries = sliced ? entries_if_sliced : a.nnz;
    return sliced;
}

template <class T, class I>
void set_spmv_config(tf_ctx *ctx, const Csr<T, I> &a, int stages, int ctas_per_sm, int cap_pct, int rows_per_thread) {
    tile::configure(ctx, a, tile::PipeConfig{stages, ctas_per_sm, cap_pct, rows_per_thread});
}

template <class T, class I, class V>
void residual(tf_ctx *ctx, const Csr<T, I, V> &a, const T *b, const T *x, T *r) {
    launch_tile(ctx, a, PlainX<T>{x}, ResidualOut<T>{b, r, nullptr}, "residual");
}

template <class T, class I, class V>
void jacobi_sweep(tf_ctx *ctx, const Csr<T, I, V> &a, const T *dinv, const T *b, const T *x, T *xo, T w,
                  const float *row_w, const int32_t *map, const T *e) {
    JacobiOut<T> epi{dinv, b, xo, row_w, w, nullptr};
    if (map)
        launch_tile(ctx, a, ProlongX<T>{x, map, e}, epi, "jacobi_prolong");
    else
        launch_tile(ctx, a, PlainX<T>{x}, epi, "jacobi");
}

template <class T, class I, class V>
void jacobi_sweep_scatter(tf_ctx *ctx, const Csr<T, I, V> &a, const T *dinv, const T *b, const T *x, T *xo, T w,
                          const int32_t *off, const int32_t *mem, T *fine) {
    launch_tile(ctx, a, PlainX<T>{x}, JacobiScatter<T>{dinv, b, xo, w, off, mem, fine, nullptr}, "jacobi_scatter");
}

template <class T>
void restrict_jacobi_zero(tf_ctx *ctx, int64_t nc, const int32_t *off, const int32_t *mem, const T *fine, T *b,
                          const T *dinv, T *x, T w) {
    if (!nc) return;
    launch_kernel(ctx, "restrict_jacobi_zero", restrict_jacobi_zero_kernel<T>, grid_for(nc), kBlock, 0, nc, off, mem,
                  fine, b, dinv, x, w);
}

bool indices_out_of_range(tf_ctx *ctx, int64_t n, const int32_t *idx, int32_t limit) {
    if (!n) return false;
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, bad, 0, sizeof(int));
    launch_kernel(ctx, "index_range", index_range_kernel, stride_grid(ctx, n), kBlock, 0, n, idx, limit, bad);
    return read_scalar(ctx, bad) != 0;
}

template <class T>
void jacobi_update(tf_ctx *ctx, int64_t n, T w, const T *dinv, const T *b, const T *ax, T *x) {
    if (!n) return;
    launch_kernel(ctx, "jacobi_update", jacobi_update_kernel<T>, stride_grid(ctx, n), kBlock, 0, n, w, dinv, b, ax, x);
}
template void jacobi_update<float>(tf_ctx *, int64_t, float, const float *, const float *, const float *, float *);
template void jacobi_update<double>(tf_ctx *, int64_t, double, const double *, const double *, const double *,
                                    double *);

template <class T>
void jacobi_zero(tf_ctx *ctx, int64_t n, const T *dinv, const T *b, T *x, T w, const float *row_w) {
    if (!n) return;
    launch_kernel(ctx, "jacobi_zero", jacobi_zero_kernel<T>, stride_grid(ctx, n), kBlock, 0, n, dinv, b, x, w, row_w);
}

// b = S(in), x = w Dinv b: the conversion of a cycle's right-hand side into
// the finest level's storage fused with its zero-guess sweep (the same
// values as convert followed by jacobi_zero).
template <class S, class T>
__global__ void jacobi_zero_convert_kernel(int64_t n, const S *__restrict__ dinv, const T *__restrict__ in,
                                           S *__restrict__ b, S *__restrict__ x, S w) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const S bi = static_cast<S>(in[i]);
        b[i] = bi;
        x[i] = w * dinv[i] * bi;
    }
}

template <class S, class T>
void jacobi_zero_convert(tf_ctx *ctx, int64_t n, const S *dinv, const T *in, S *b, S *x, S w) {
    if (!n) return;
    launch_kernel(ctx, "jacobi_zero_convert", jacobi_zero_convert_kernel<S, T>, stride_grid(ctx, n), kBlock, 0, n,
                  dinv, in, b, x, w);
}
template void jacobi_zero_convert<float, double>(tf_ctx *, int64_t, const float *, const double *, float *, float *,
                                                 float);
template void jacobi_zero_convert<float, float>(tf_ctx *, int64_t, const float *, const float *, float *, float *,
                                                float);
template void jacobi_zero_convert<double, double>(tf_ctx *, int64_t, const double *, const double *, double *,
                                                  double *, double);
template void jacobi_zero_convert<double, float>(tf_ctx *, int64_t, const double *, const float *, double *,
                                                 double *, double);

template <class T, class I, class V>
void inverse_diagonal(tf_ctx *ctx, const Csr<T, I, V> &a, T *dinv) {
    require(a.rows > 0 && a.rows == a.cols, "Inverse diagonal requires a nonempty square matrix");
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, bad, 0, sizeof(int));
    launch_kernel(ctx, "inverse_diagonal", inverse_diagonal_kernel<T, I, V>, grid_for(a.rows), kBlock, 0, a.rows, a.rp,
                  a.ci, a.val, dinv, bad);
    if (read_scalar(ctx, bad)) fail(TF_ERR_INVALID, "Missing or invalid diagonal");
}

bool delta_columns_enabled() {
    const char *v = std::getenv("THERMOFEM_B200_DELTA16");
    return !(v && v[0] == '0');
}

template <class I>
bool delta_columns(tf_ctx *ctx, int64_t rows, const I *rp, const I *ci, int16_t *cd) {
    if (!rows) return false;
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, bad, 0, sizeof(int));
    launch_kernel(ctx, "delta_columns", delta_columns_kernel<I>, grid_for(rows), kBlock, 0, rows, rp, ci, cd, bad);
    return read_scalar(ctx, bad) == 0;
}
template bool delta_columns<int32_t>(tf_ctx *, int64_t, const int32_t *, const int32_t *, int16_t *);
template bool delta_columns<int64_t>(tf_ctx *, int64_t, const int64_t *, const int64_t *, int16_t *);

// One CTA waits, with the pipelined kernels' bounded wait, on an mbarrier
// that nothing completes, and raises the fault word as they do when a wait
// expires (no copy is in flight, so there is nothing to drain).
__global__ void wait_check_kernel(long long polls, int *fault) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        tile::mbar_init(&bar, 1);
        tile::mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !tile::mbar_wait(&bar, 0, polls)) atomicExch(fault, 1);
}

void bounded_wait_check(tf_ctx *ctx, int64_t polls) {
    require(polls >= 1 && polls <= tile::kWaitLimit, "polls must be 1..2^20");
    launch_kernel(ctx, "wait_check", wait_check_kernel, 1, 32, 0, static_cast<long long>(polls), ctx->fault);
    cuda_check(cudaStreamSynchronize(ctx->stream), "wait check");
    check_faults(ctx);  // TF_ERR_TIMEOUT, fault word cleared
}

bool banded_enabled() {
    const char *v = std::getenv("THERMOFEM_B200_BANDED");
    return !(v && v[0] == '0');
}

bool sliced_enabled() {
    const char *v = std::getenv("THERMOFEM_B200_SLICED");
    return !(v && v[0] == '0');
}

static bool sorted_slices_enabled() {
    const char *v = std::getenv("THERMOFEM_B200_SLICED");
    return v && std::strcmp(v, "sorted") == 0;
}

// Slice entry counts for the given row order; returns their total.
static int64_t slice_entries(tf_ctx *ctx, int64_t rows, int64_t nslices, const int32_t *rp, const int32_t *perm,
                             int32_t *entries) {
    DeviceBuffer<unsigned long long> total(1);
    memset_async(ctx, entries, 0, (nslices + 1) * sizeof(int32_t));
    memset_async(ctx, total.data(), 0, sizeof(unsigned long long));
    launch_kernel(ctx, "slice_entries", slice_entries_kernel<int32_t>, grid_for(nslices * 32), kBlock, 0, rows,
                  nslices, rp, perm, entries, total.data());
    return static_cast<int64_t>(read_scalar(ctx, total.data()));
}

// Most entries of any 256-row tile (8 consecutive slices) of a sliced copy.
__global__ void slice_tile_max_kernel(int64_t nslices, const int32_t *__restrict__ sp,
                                      unsigned long long *tile_max) {
    pdl_enter();
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t s0 = t * 8;
    if (s0 >= nslices) return;
    const int64_t s1 = s0 + 8 < nslices ? s0 + 8 : nslices;
    atomicMax(tile_max, static_cast<unsigned long long>(sp[s1] - sp[s0]));
}

template <class T>
bool build_sliced(tf_ctx *ctx, const Csr<T, int32_t> &a, SlicedCopy<T> &out, bool allow_sort) {
    out.release();
    if (!a.rows || !a.nnz || !a.cd) return false;
    const int64_t nslices = (a.rows + 31) / 32;
    // padding of at most THERMOFEM_B200_SLICED_PAD percent of nnz (tiny
    // operators excepted; int32 entry starts).  Default 50 for FP64 values,
    // where the row-tile kernel's per-row work outweighs the padded bytes on
    // the aggregated levels (30-45 % padding), 25 for FP32, where it does not
    // (128^3 PCG, one B200: FP64 36.1-36.8 vs 37.9-38.5 ms with 50 vs 25;
    // mixed 30.6 vs 29.4-29.8 ms).
    int pad_pct = sizeof(T) == 8 ? 50 : 25;
    if (const char *v = std::getenv("THERMOFEM_B200_SLICED_PAD")) pad_pct = std::atoi(v);
    auto fits = [&](int64_t n) { return n < INT32_MAX && (n <= a.nnz + a.nnz * pad_pct / 100 || n <= 4096); };
    DeviceBuffer<int32_t> entries(static_cast<size_t>(nslices) + 1);
    int64_t n = slice_entries(ctx, a.rows, nslices, a.rp, nullptr, entries.data());
    if (!fits(n)) {
        if (!allow_sort || !sorted_slices_enabled()) return false;
        out.perm.allocate(static_cast<size_t>(a.rows));
        launch_kernel(ctx, "slice_sort", slice_sort_kernel<int32_t>, grid_for(a.rows, 256), 256, 0, a.rows, a.rp,
                      out.perm.data());
        n = slice_entries(ctx, a.rows, nslices, a.rp, out.perm.data(), entries.data());
        if (!fits(n)) {
            out.release();
            return false;
        }
    }
    out.sp.allocate(static_cast<size_t>(nslices) + 1);
    scan_exclusive(ctx, nslices + 1, entries.data(), out.sp.data());
    out.val.allocate(static_cast<size_t>(n));
    out.col.allocate(static_cast<size_t>(n));
    launch_kernel(ctx, "slice_fill", slice_fill_kernel<T, int32_t>, grid_for(nslices * 32), kBlock, 0, a.rows,
                  nslices, a.rp, a.val, a.cd, out.perm.data(), out.sp.data(), out.val.data(), out.col.data());
    DeviceBuffer<unsigned long long> tmax(1);
    memset_async(ctx, tmax.data(), 0, sizeof(unsigned long long));
    launch_kernel(ctx, "slice_tile_max", slice_tile_max_kernel, grid_for((nslices + 7) / 8), kBlock, 0, nslices,
                  out.sp.data(), tmax.data());
    out.tile_max = static_cast<int64_t>(read_scalar(ctx, tmax.data()));
    out.entries = n;
    return true;
}
template bool build_sliced<float>(tf_ctx *, const Csr<float, int32_t> &, SlicedCopy<float> &, bool);
template bool build_sliced<double>(tf_ctx *, const Csr<double, int32_t> &, SlicedCopy<double> &, bool);

template <class T>
bool build_banded(tf_ctx *ctx, const Csr<T, int32_t> &a, SlicedCopy<T> &out) {
    out.release();
    if (!a.rows || !a.nnz || a.rows >= INT32_MAX) return false;
    const int64_t nslices = (a.rows + 31) / 32;
    int pad_pct = 10;
    if (const char *v = std::getenv("THERMOFEM_B200_BANDED_PAD")) pad_pct = std::atoi(v);
    DeviceBuffer<int32_t> entries(static_cast<size_t>(nslices) + 1);
    DeviceBuffer<unsigned long long> total(1);
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, entries.data(), 0, (nslices + 1) * sizeof(int32_t));
    memset_async(ctx, total.data(), 0, sizeof(unsigned long long));
    memset_async(ctx, bad, 0, sizeof(int));
    launch_kernel(ctx, "band_width", band_width_kernel, grid_for(nslices * 32), kBlock, 0, a.rows, nslices, a.rp,
                  a.ci, entries.data(), total.data(), bad);
    if (read_scalar(ctx, bad)) return false;
    const int64_t n = static_cast<int64_t>(read_scalar(ctx, total.data()));
    if (n >= INT32_MAX || n > a.nnz + a.nnz * pad_pct / 100) return false;
    out.sp.allocate(static_cast<size_t>(nslices) + 1);
    scan_exclusive(ctx, nslices + 1, entries.data(), out.sp.data());
    out.val.allocate(static_cast<size_t>(n));
    // an even number of slots: the staged kernel copies whole 16-byte pairs
    const int64_t slots = n / 32, slots_even = (slots + 1) & ~int64_t(1);
    out.band.allocate(static_cast<size_t>(slots_even));
    if (slots_even > slots) memset_async(ctx, out.band.data() + slots, 0, sizeof(int2));
    launch_kernel(ctx, "band_fill", band_fill_kernel<T>, grid_for(nslices * 32), kBlock, 0, a.rows, nslices, a.rp,
                  a.ci, a.val, out.sp.data(), out.val.data(), out.band.data());
    DeviceBuffer<unsigned long long> tmax(1);
    memset_async(ctx, tmax.data(), 0, sizeof(unsigned long long));
    launch_kernel(ctx, "slice_tile_max", slice_tile_max_kernel, grid_for((nslices + 7) / 8), kBlock, 0, nslices,
                  out.sp.data(), tmax.data());
    out.tile_max = static_cast<int64_t>(read_scalar(ctx, tmax.data()));
    out.entries = n;
    return true;
}
template bool build_banded<float>(tf_ctx *, const Csr<float, int32_t> &, SlicedCopy<float> &);
template bool build_banded<double>(tf_ctx *, const Csr<double, int32_t> &, SlicedCopy<double> &);

template <class T>
void restrict_sum(tf_ctx *ctx, int64_t nc, const int32_t *off, const int32_t *mem, const T *fine, T *coarse) {
    if (!nc) return;
    launch_kernel(ctx, "restrict", restrict_kernel<T>, grid_for(nc), kBlock, 0, nc, off, mem, fine, coarse);
}

template <class T>
void prolong_add(tf_ctx *ctx, int64_t nf, const int32_t *map, const T *coarse, T *fine) {
    if (!nf) return;
    launch_kernel(ctx, "prolong", prolong_kernel<T>, stride_grid(ctx, nf), kBlock, 0, nf, map, coarse, fine);
}

template <class T>
void dot_multi(tf_ctx *ctx, int64_t n, int count, const T *const *xs, const T *const *ys, double *out) {
    require(count >= 1 && count <= 4, "dot count must be 1..4");
    DotArgs args{};
    for (int k = 0; k < count; ++k) {
        args.x[k] = xs[k];
        args.y[k] = ys[k];
    }
    // Fixed partition for a given n: the result does not depend on the GPU.
    int64_t parts64 = (n + 2047) / 2048;
    if (parts64 < 1) parts64 = 1;
    if (parts64 > 1184) parts64 = 1184;
    const int parts = static_cast<int>(parts64);
    double *partial = static_cast<double *>(ctx->arena(sizeof(double) * 4 * parts));
    switch (count) {
        case 1: launch_kernel(ctx, "dot_partial", dot_partial_kernel<T, 1>, parts, 256, 0, n, args, partial); break;
        case 2: launch_kernel(ctx, "dot_partial", dot_partial_kernel<T, 2>, parts, 256, 0, n, args, partial); break;
        case 3: launch_kernel(ctx, "dot_partial", dot_partial_kernel<T, 3>, parts, 256, 0, n, args, partial); break;
        default: launch_kernel(ctx, "dot_partial", dot_partial_kernel<T, 4>, parts, 256, 0, n, args, partial); break;
    }
    switch (count) {
        case 1: launch_kernel(ctx, "dot_final", dot_final_kernel<1>, 1, 256, 0, parts, partial, out); break;
        case 2: launch_kernel(ctx, "dot_final", dot_final_kernel<2>, 1, 256, 0, parts, partial, out); break;
        case 3: launch_kernel(ctx, "dot_final", dot_final_kernel<3>, 1, 256, 0, parts, partial, out); break;
        default: launch_kernel(ctx, "dot_final", dot_final_kernel<4>, 1, 256, 0, parts, partial, out); break;
    }
}

// The fixed partition of dot_multi: a reduction's value does not depend on the GPU.
static int reduction_parts(int64_t n) {
    int64_t parts = (n + 2047) / 2048;
    return static_cast<int>(parts < 1 ? 1 : (parts > 1184 ? 1184 : parts));
}

template <class T>
void krylov_cg_update(tf_ctx *ctx, int64_t n, double alpha, const T *p, const T *ap, T *x, T *r, double *rr) {
    const int parts = reduction_parts(n);
    double *partial = static_cast<double *>(ctx->arena(sizeof(double) * parts));
    launch_kernel(ctx, "krylov_cg_update", cg_update_kernel<T>, parts, 256, 0, n, static_cast<T>(alpha), p, ap, x, r,
                  partial);
    launch_kernel(ctx, "dot_final", dot_final_kernel<1>, 1, 256, 0, parts, partial, rr);
}

template <class T>
void krylov_cg_direction(tf_ctx *ctx, int64_t n, double beta, int restart, const T *z, T *p) {
    if (!n) return;
    launch_kernel(ctx, "krylov_cg_direction", cg_direction_kernel<T>, stride_grid(ctx, n), kBlock, 0, n,
                  static_cast<T>(beta), restart, z, p);
}

template <class T>
void krylov_bicgstab_direction(tf_ctx *ctx, int64_t n, double beta, double omega, int restart, const T *r,
                               const T *v, T *p) {
    if (!n) return;
    launch_kernel(ctx, "krylov_bicgstab_direction", bicgstab_direction_kernel<T>, stride_grid(ctx, n), kBlock, 0, n,
                  static_cast<T>(beta), static_cast<T>(omega), restart, r, v, p);
}

template <class T>
void krylov_bicgstab_s(tf_ctx *ctx, int64_t n, double alpha, const T *r, const T *v, const T *phat, T *x, T *s,
                       double *ss) {
    const int parts = reduction_parts(n);
    double *partial = static_cast<double *>(ctx->arena(sizeof(double) * parts));
    launch_kernel(ctx, "krylov_bicgstab_s", bicgstab_s_kernel<T>, parts, 256, 0, n, static_cast<T>(alpha), r, v,
                  phat, x, s, partial);
    launch_kernel(ctx, "dot_final", dot_final_kernel<1>, 1, 256, 0, parts, partial, ss);
}

template <class T>
void krylov_bicgstab_update(tf_ctx *ctx, int64_t n, double omega, const T *shat, const T *s, const T *t, T *x, T *r,
                            double *rr) {
    const int parts = reduction_parts(n);
    double *partial = static_cast<double *>(ctx->arena(sizeof(double) * parts));
    launch_kernel(ctx, "krylov_bicgstab_update", bicgstab_update_kernel<T>, parts, 256, 0, n, static_cast<T>(omega),
                  shat, s, t, x, r, partial);
    launch_kernel(ctx, "dot_final", dot_final_kernel<1>, 1, 256, 0, parts, partial, rr);
}

template <class T>
void axpby(tf_ctx *ctx, int64_t n, double a, const T *x, double b, T *y) {
    if (!n) return;
    launch_kernel(ctx, "axpby", axpby_kernel<T>, stride_grid(ctx, n), kBlock, 0, n, a, x, b, y);
}

template <class S, class D>
void convert(tf_ctx *ctx, int64_t n, const S *src, D *dst) {
    if (!n) return;
    launch_kernel(ctx, "convert", convert_kernel<S, D>, stride_grid(ctx, n), kBlock, 0, n, src, dst);
}

template <class T>
void fill_zero(tf_ctx *ctx, int64_t n, T *x) {
    memset_async(ctx, x, 0, static_cast<size_t>(n) * sizeof(T));
}

template <class I>
bool csr_structure_ok(tf_ctx *ctx, int64_t rows, int64_t cols, int64_t nnz, const I *rp, const I *ci) {
    if (rows == 0 && rp == nullptr) return nnz == 0;  // an empty matrix may come without offsets
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, bad, 0, sizeof(int));
    launch_kernel(ctx, "csr_validate", csr_structure_kernel<I>, grid_for(rows > 0 ? rows : 1), kBlock, 0, rows, cols,
                  nnz, rp, ci, bad);
    return read_scalar(ctx, bad) == 0;
}

template <class T, class I>
int csr_canonical_flags(tf_ctx *ctx, const Csr<T, I> &a) {
    int *flags = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, flags, 0, sizeof(int));
    if (a.rows) {
        launch_kernel(ctx, "check_canonical", canonical_flags_kernel<T, I>, grid_for(a.rows), kBlock, 0, a.rows, a.nnz,
                      a.rp, a.ci, a.val, flags);
    }
    return read_scalar(ctx, flags);
}

bool row_stats(tf_ctx *ctx, const Csr<double, int32_t> &a, double *row_max) {
    int *bad = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, bad, 0, sizeof(int));
    if (a.rows) {
        launch_kernel(ctx, "row_stats", row_stats_kernel, grid_for(a.rows), kBlock, 0, a.rows, a.rp, a.ci, a.val, bad,
                      row_max);
    }
    return read_scalar(ctx, bad) == 0;
}

#define TF_SPMV_INST(T, I)                                                                                     \
    template void spmv<T, I>(tf_ctx *, const Csr<T, I> &, const T *, T *);                                     \
    template void autotune_spmv<T, I>(tf_ctx *, const Csr<T, I> &, const T *, T *, int *, int *, int *, int *, float *); \
    template void set_spmv_config<T, I>(tf_ctx *, const Csr<T, I> &, int, int, int, int); \
    template void tune_spmv<T, I>(tf_ctx *, const Csr<T, I> &, const T *, T *);                                \
    template bool streams_sliced<T, I>(tf_ctx *, const Csr<T, I> &, int64_t, int64_t *);                      \
    template void residual<T, I>(tf_ctx *, const Csr<T, I> &, const T *, const T *, T *);                      \
    template void jacobi_sweep<T, I>(tf_ctx *, const Csr<T, I> &, const T *, const T *, const T *, T *, T,     \
                                     const float *, const int32_t *, const T *);                               \
    template void jacobi_sweep_scatter<T, I>(tf_ctx *, const Csr<T, I> &, const T *, const T *, const T *, T *, T, \
                                             const int32_t *, const int32_t *, T *);                           \
    template void inverse_diagonal<T, I>(tf_ctx *, const Csr<T, I> &, T *);                                    \
    template int csr_canonical_flags<T, I>(tf_ctx *, const Csr<T, I> &);
TF_SPMV_INST(float, int32_t)
TF_SPMV_INST(double, int32_t)
TF_SPMV_INST(float, int64_t)
TF_SPMV_INST(double, int64_t)
#undef TF_SPMV_INST

// FP32 values under FP64 vectors (the hierarchy whose operators are stored
// in FP32 and whose cycle runs in FP64).
template void spmv<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &, const double *, double *);
template void tune_spmv<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &, const double *,
                                               double *);
template bool streams_sliced<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &, int64_t,
                                                    int64_t *);
template void residual<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &, const double *,
                                              const double *, double *);
template void jacobi_sweep<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &, const double *,
                                                  const double *, const double *, double *, double, const float *,
                                                  const int32_t *, const double *);
template void jacobi_sweep_scatter<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &,
                                                          const double *, const double *, const double *, double *,
                                                          double, const int32_t *, const int32_t *, double *);
template void inverse_diagonal<double, int32_t, float>(tf_ctx *, const Csr<double, int32_t, float> &, double *);

#define TF_VEC_INST(T)                                                                                        \
    template void jacobi_zero<T>(tf_ctx *, int64_t, const T *, const T *, T *, T, const float *);              \
    template void restrict_sum<T>(tf_ctx *, int64_t, const int32_t *, const int32_t *, const T *, T *);        \
    template void restrict_jacobi_zero<T>(tf_ctx *, int64_t, const int32_t *, const int32_t *, const T *, T *,  \
                                          const T *, T *, T);                                                  \
    template void prolong_add<T>(tf_ctx *, int64_t, const int32_t *, const T *, T *);                          \
    template void dot_multi<T>(tf_ctx *, int64_t, int, const T *const *, const T *const *, double *);           \
    template void axpby<T>(tf_ctx *, int64_t, double, const T *, double, T *);                                 \
    template void krylov_cg_update<T>(tf_ctx *, int64_t, double, const T *, const T *, T *, T *, double *);     \
    template void krylov_cg_direction<T>(tf_ctx *, int64_t, double, int, const T *, T *);                      \
    template void krylov_bicgstab_direction<T>(tf_ctx *, int64_t, double, double, int, const T *, const T *, T *); \
    template void krylov_bicgstab_s<T>(tf_ctx *, int64_t, double, const T *, const T *, const T *, T *, T *,     \
                                       double *);                                                              \
    template void krylov_bicgstab_update<T>(tf_ctx *, int64_t, double, const T *, const T *, const T *, T *, T *, \
                                            double *);                                                         \
    template void fill_zero<T>(tf_ctx *, int64_t, T *);
TF_VEC_INST(float)
TF_VEC_INST(double)
#undef TF_VEC_INST

template void convert<float, double>(tf_ctx *, int64_t, const float *, double *);
template void convert<double, float>(tf_ctx *, int64_t, const double *, float *);
template void convert<int32_t, int64_t>(tf_ctx *, int64_t, const int32_t *, int64_t *);
template void convert<int64_t, int32_t>(tf_ctx *, int64_t, const int64_t *, int32_t *);
template void convert<float, float>(tf_ctx *, int64_t, const float *, float *);
template void convert<double, double>(tf_ctx *, int64_t, const double *, double *);
template void convert<int32_t, int32_t>(tf_ctx *, int64_t, const int32_t *, int32_t *);
template void convert<int64_t, int64_t>(tf_ctx *, int64_t, const int64_t *, int64_t *);
template bool csr_structure_ok<int32_t>(tf_ctx *, int64_t, int64_t, int64_t, const int32_t *, const int32_t *);
template bool csr_structure_ok<int64_t>(tf_ctx *, int64_t, int64_t, int64_t, const int64_t *, const int64_t *);

}  // namespace tfb
