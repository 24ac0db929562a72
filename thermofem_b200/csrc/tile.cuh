// tile.cuh -- the row-tile CSR kernel shared by the SpMV family (spmv.cu)
// and the fused Krylov steps (krylov.cu).
//
// One CTA owns 256 * RPT consecutive rows.  Their nonzeros form one
// contiguous range of values and column indices, which is staged into
// shared memory with 16-byte vector loads (every HBM sector read once and
// fully); each thread then reduces its rows from shared memory left to right
// with x gathered through L1/L2.  Long tiles are processed in chunks.  The
// epilogue is a template parameter: it writes the row result, may read the
// row's own x~ (XS), may accumulate up to four per-row products that the CTA
// reduces into per-tile partial sums (deterministic: fixed tile partition and
// fixed reduction tree), and may gate the whole launch on a device flag.
#pragma once
#include "ops.cuh"

namespace tfb {
namespace tile {

constexpr int kThreads = 256;

// Copies n consecutive elements src[0..n) into dst[0..n) with all threads of
// the block: 16-byte vector loads over the aligned interior, scalar loads for
// the ragged head and tail.  No element outside [0, n) is read.
template <class E>
__device__ __forceinline__ void stage(E *dst, const E *__restrict__ src, int n) {
    constexpr int kVec = 16 / sizeof(E);
    const uintptr_t addr = reinterpret_cast<uintptr_t>(src);
    const int misaligned = static_cast<int>((addr & 15u) / sizeof(E));
    int head = misaligned ? kVec - misaligned : 0;
    if (head > n) head = n;
    if (static_cast<int>(threadIdx.x) < head) dst[threadIdx.x] = src[threadIdx.x];
    const int body = (n - head) / kVec;
    const uint4 *sv = reinterpret_cast<const uint4 *>(src + head);
    E *d = dst + head;
#pragma unroll 4
    for (int v = threadIdx.x; v < body; v += blockDim.x) {
        const uint4 q = __ldg(sv + v);
        E tmp[kVec];
        memcpy(tmp, &q, 16);
#pragma unroll
        for (int e = 0; e < kVec; ++e) d[v * kVec + e] = tmp[e];
    }
    const int tail = head + body * kVec;
    if (tail + static_cast<int>(threadIdx.x) < n) dst[tail + threadIdx.x] = src[tail + threadIdx.x];
}

template <class T>
struct PlainX {
    const T *__restrict__ x;
    __device__ __forceinline__ T operator()(int64_t j) const { return __ldg(x + j); }
};

// x~_j = x_j + e[map_j]: the prolongation x += P e read on the fly.
template <class T>
struct ProlongX {
    const T *__restrict__ x;
    const int32_t *__restrict__ map;
    const T *__restrict__ e;
    __device__ __forceinline__ T operator()(int64_t j) const { return __ldg(x + j) + __ldg(e + __ldg(map + j)); }
};

// Deterministic block reduction of K doubles; thread 0 holds the result.
template <int K>
__device__ __forceinline__ void block_reduce(double (&v)[K]) {
    __shared__ double shm[K > 0 ? K * 32 : 1];
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

// Epilogue requirements:
//   static constexpr int kReduce;           number of reduced products (0..4)
//   __device__ bool skip() const;           true: the whole launch is gated off
//   __device__ void operator()(int64_t i, T acc, const XS &xs, double (&red)[kReduce or 1]) const;
//   double *partial;                        [kReduce][gridDim.x] when kReduce > 0
template <class T, class I, int RPT, class XS, class Epi>
__global__ void __launch_bounds__(kThreads) csr_tile_kernel(int64_t rows, const I *__restrict__ rp,
                                                             const I *__restrict__ ci, const T *__restrict__ val,
                                                             int chunk, XS xs, Epi epi) {
    constexpr int K = Epi::kReduce;
    if (epi.skip()) return;
    extern __shared__ __align__(16) unsigned char smem[];
    T *sval = reinterpret_cast<T *>(smem);
    I *scol = reinterpret_cast<I *>(smem + static_cast<size_t>(chunk) * sizeof(T));
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * (kThreads * RPT);
    const int64_t rend = min(r0 + static_cast<int64_t>(kThreads * RPT), rows);
    const int64_t t0 = rp[r0], t1 = rp[rend];
    int64_t rs[RPT], re[RPT];
    T acc[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int64_t r = r0 + threadIdx.x + k * kThreads;
        rs[k] = r < rows ? static_cast<int64_t>(rp[r]) : 0;
        re[k] = r < rows ? static_cast<int64_t>(rp[r + 1]) : 0;
        acc[k] = T(0);
    }
    for (int64_t c0 = t0; c0 < t1; c0 += chunk) {
        const int cnt = static_cast<int>(min(static_cast<int64_t>(chunk), t1 - c0));
        if (c0 != t0) __syncthreads();
        stage(sval, val + c0, cnt);
        stage(scol, ci + c0, cnt);
        __syncthreads();
        // The first kGather entries of every row of this thread are gathered
        // together (independent x loads in flight) before any accumulation;
        // the sum itself stays left to right.  Padding lanes add +0.
        constexpr int kGather = 8;
        T xv[RPT][kGather];
        int lo[RPT], hi[RPT];  // chunk-relative
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            lo[k] = static_cast<int>(max(rs[k], c0) - c0);
            hi[k] = static_cast<int>(min(re[k], c0 + cnt) - c0);
#pragma unroll
            for (int u = 0; u < kGather; ++u) {
                const int o = lo[k] + u;
                xv[k][u] = o < hi[k] ? xs(static_cast<int64_t>(scol[o])) : T(0);
            }
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            T s = acc[k];
#pragma unroll
            for (int u = 0; u < kGather; ++u) {
                const int o = lo[k] + u;
                s += (o < hi[k] ? sval[o] : T(0)) * xv[k][u];
            }
            for (int o0 = lo[k] + kGather; o0 < hi[k]; o0 += kGather) {
                T y[kGather];
#pragma unroll
                for (int u = 0; u < kGather; ++u) {
                    const int o = o0 + u;
                    y[u] = o < hi[k] ? xs(static_cast<int64_t>(scol[o])) : T(0);
                }
#pragma unroll
                for (int u = 0; u < kGather; ++u) {
                    const int o = o0 + u;
                    s += (o < hi[k] ? sval[o] : T(0)) * y[u];
                }
            }
            acc[k] = s;
        }
    }
    double red[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); ++k) red[k] = 0.0;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int64_t r = r0 + threadIdx.x + k * kThreads;
        if (r < rows) epi(r, acc[k], xs, red);
    }
    if constexpr (K > 0) {
        block_reduce<K>(red);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < K; ++k) epi.partial[k * gridDim.x + blockIdx.x] = red[k];
    }
}

// Number of CTAs (= partial sums) of a tile launch over these rows.
inline unsigned grid(const SpmvShape &shape, int64_t rows) {
    const int64_t tile_rows = static_cast<int64_t>(kThreads) * shape.rows_per_thread;
    return static_cast<unsigned>((rows + tile_rows - 1) / tile_rows);
}

// Opts the instantiation into the dynamic shared memory it is launched with
// (the staged chunk plus the epilogue's static reduction buffer can exceed
// the 48 KB default); done once per instantiation and device.
template <auto Kernel>
void allow_smem(size_t bytes) {
    static thread_local int configured_device = -1;
    static thread_local size_t configured_bytes = 0;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev == configured_device && bytes <= configured_bytes) return;
    cuda_check(cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
               "tile shared memory");
    configured_device = dev;
    configured_bytes = bytes;
}

template <class T, class I, class XS, class Epi>
void launch(tf_ctx *ctx, const Csr<T, I> &a, const XS &xs, const Epi &epi, const char *name) {
    if (a.rows == 0) return;
    const SpmvShape shape = spmv_shape(a.rows, a.nnz, sizeof(T), sizeof(I));
    const unsigned g = grid(shape, a.rows);
    const size_t smem = static_cast<size_t>(shape.chunk) * (sizeof(T) + sizeof(I));
    if (shape.rows_per_thread == 2) {
        allow_smem<csr_tile_kernel<T, I, 2, XS, Epi>>(smem);
        csr_tile_kernel<T, I, 2><<<g, kThreads, smem, ctx->stream>>>(a.rows, a.rp, a.ci, a.val, shape.chunk, xs, epi);
    } else {
        allow_smem<csr_tile_kernel<T, I, 1, XS, Epi>>(smem);
        csr_tile_kernel<T, I, 1><<<g, kThreads, smem, ctx->stream>>>(a.rows, a.rp, a.ci, a.val, shape.chunk, xs, epi);
    }
    launched(ctx, name);
}

}  // namespace tile
}  // namespace tfb
