// tile.cuh -- the SpMV kernels shared by the SpMV family (spmv.cu) and the
// fused Krylov steps (krylov.cu): the staged row-tile kernel (unaligned
// arrays), the pipelined row-tile kernel (csr_pipe_kernel: CSR chunks
// bulk-copied into a shared-memory ring), and the two kernels over an
// operator's sliced copy (sliced_kernel: coalesced loads per 32-row slice;
// sliced_pipe_kernel: whole tiles bulk-copied into a ring).  All of them take
// the same epilogues and gather functors, reduce every row left to right and
// write partial sums per 256-row block, so they give the same bits;
// tile::launch picks one by the operator's storage and its tuned shape.
//
// Staged row-tile kernel: one CTA owns 256 * RPT consecutive rows.  Their nonzeros form one
// contiguous range of values and column indices, which is staged into
// shared memory with 16-byte vector loads (every HBM sector read once and
// fully); each thread then reduces its rows from shared memory left to right
// with x gathered through L1/L2.  Long tiles are processed in chunks.  The
// epilogue is a template parameter: it writes the row result, may read the
// row's own x~ (XS), may accumulate up to four per-row products that the CTA
// reduces into per-tile partial sums (deterministic: fixed tile partition and
// fixed reduction tree), and may gate the whole launch on a device flag.
#pragma once
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

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

// Gather functors: xs(j) is x~_j; xs.row(i) is a view of x~ around row i,
// view(c) = x~_{i+c}, for kernels that gather by column offsets (one 32-bit
// offset per entry instead of a 64-bit index).
template <class T>
struct PlainX {
    const T *__restrict__ x;
    __device__ __forceinline__ T operator()(int64_t j) const { return __ldg(x + j); }
    struct View {
        const T *__restrict__ p;
        __device__ __forceinline__ T operator()(int c) const { return __ldg(p + c); }
    };
    __device__ __forceinline__ View row(int64_t i) const { return {x + i}; }
};

// x~_j = x_j + e[map_j]: the prolongation x += P e read on the fly.
template <class T>
struct ProlongX {
    const T *__restrict__ x;
    const int32_t *__restrict__ map;
    const T *__restrict__ e;
    __device__ __forceinline__ T operator()(int64_t j) const { return __ldg(x + j) + __ldg(e + __ldg(map + j)); }
    struct View {
        const T *__restrict__ p;
        const int32_t *__restrict__ m;
        const T *__restrict__ e;
        __device__ __forceinline__ T operator()(int c) const { return __ldg(p + c) + __ldg(e + __ldg(m + c)); }
    };
    __device__ __forceinline__ View row(int64_t i) const { return {x + i, map + i, e}; }
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

// Last-CTA handoff.  Every CTA of a reducing launch calls last_cta() once,
// after its partial sums are written; it returns true in the CTA that comes
// last (a device-wide ticket), which then sees every partial sum and runs the
// scalar step that consumes them, in place of a separate one-CTA launch.  The
// ticket is reset for the next launch.  All threads of the CTA must call it.
__device__ __forceinline__ bool last_cta(unsigned *ticket) {
    __shared__ unsigned is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's partial sums before its ticket
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = t == gridDim.x - 1 ? 1u : 0u;
        if (is_last) {
            atomicExch(ticket, 0u);
            __threadfence();
        }
    }
    __syncthreads();
    return is_last != 0;
}

// No scalar step after the reduction.
struct NoFinal {
    static constexpr bool kActive = false;
    unsigned *ticket{nullptr};
    __device__ void operator()(const double *, int) const {}
};

// Runs fin (when active) in the last CTA over `parts` partial sums.
template <class Fin>
__device__ __forceinline__ void finish(const Fin &fin, const double *part, int parts) {
    if constexpr (Fin::kActive) {
        if (last_cta(fin.ticket)) fin(part, parts);
    }
}

// Epilogue requirements:
//   static constexpr int kReduce;           number of reduced products (0..4)
//   __device__ bool skip() const;           true: the whole launch is gated off
//   __device__ void operator()(int64_t i, T acc, const XS &xs, double (&red)[kReduce or 1]) const;
//   double *partial;                        [kReduce][gridDim.x] when kReduce > 0
// (the pipelined kernel also needs `fin`, a tile::finish step, when kReduce > 0)
template <class T, class I, int RPT, class XS, class Epi, class V = T>
__global__ void __launch_bounds__(kThreads) csr_tile_kernel(int64_t rows, const I *__restrict__ rp,
                                                             const I *__restrict__ ci, const V *__restrict__ val,
                                                             int chunk, XS xs, Epi epi) {
    constexpr int K = Epi::kReduce;
    pdl_enter();
    if (epi.skip()) return;
    extern __shared__ __align__(128) unsigned char smem[];
    V *sval = reinterpret_cast<V *>(smem);
    I *scol = reinterpret_cast<I *>(smem + static_cast<size_t>(chunk) * sizeof(V));
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
        if (r < rows) epi(r, acc[k], epi.pre(r, xs), red);
    }
    if constexpr (K > 0) {
        block_reduce<K>(red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) epi.partial[k * gridDim.x + blockIdx.x] = red[k];
        }
    }
}

// ---------------------------------------------------------------------------
// Pipelined persistent variant (sm_100a).
//
// A persistent CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...  One
// producer warp (warp 8, lane 0) streams each tile's row offsets, values and
// column indices into a ring of shared-memory stages with cp.async.bulk
// (TMA bulk copies, completion counted in bytes on an mbarrier), staying up
// to `stages - 1` chunks ahead; the eight consumer warps wait on the stage's
// "full" barrier, reduce one row per thread exactly as above, and release the
// stage on its "empty" barrier.  Bulk copies start and end on 16-byte
// boundaries: a chunk [cs, ce) is copied from align_down(cs) to align_up(ce)
// (the over-read lies inside the arrays except at their very end, where the
// ragged tail is fetched with plain loads before the barrier is armed).
// Every wait is bounded: on expiry the kernel raises *fault, skips its
// remaining work, drains its own copies (bounded) and returns.
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 4;
constexpr int kPipeCtasPerSm = 2;
constexpr long long kWaitLimit = 1ll << 20;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit = kWaitLimit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Shared-memory layout of one stage: row offsets (I), values (T), column
// entries (C).
template <class T, class I, class C = I>
struct StageLayout {
    static constexpr int kVT = 16 / sizeof(T), kVI = 16 / sizeof(I), kVC = 16 / sizeof(C);
    int rp_bytes, val_bytes, col_bytes, bytes;
    __host__ __device__ StageLayout(int cap, int tile_rows) {
        rp_bytes = ((tile_rows + 1 + kVI) * static_cast<int>(sizeof(I)) + 15) & ~15;
        val_bytes = ((cap + 2 * kVT) * static_cast<int>(sizeof(T)) + 15) & ~15;
        col_bytes = ((cap + 2 * kVC) * static_cast<int>(sizeof(C)) + 15) & ~15;
        bytes = (rp_bytes + val_bytes + col_bytes + 127) & ~127;
    }
};

// One range [lo, hi) of an array of length len, staged at dst[j - align_down(lo)].
template <class E>
struct Range {
    int64_t a0{0}, bulk_end{0}, hi{0};
    __device__ __forceinline__ void plan(int64_t lo, int64_t hi_, int64_t len) {
        constexpr int64_t V = 16 / sizeof(E);
        hi = hi_;
        a0 = lo - (lo % V);
        const int64_t a1 = (hi_ + V - 1) / V * V;
        bulk_end = hi_ <= lo ? a0 : (a1 <= len ? a1 : hi_ - (hi_ % V));
        if (bulk_end < a0) bulk_end = a0;
    }
    __device__ __forceinline__ void plain(E *dst, const E *src) const {
        for (int64_t j = bulk_end; j < hi; ++j) dst[j - a0] = src[j];
    }
    __device__ __forceinline__ uint32_t bytes() const { return static_cast<uint32_t>((bulk_end - a0) * sizeof(E)); }
    __device__ __forceinline__ void issue(E *dst, const E *src, uint64_t *bar) const {
        if (bulk_end > a0) bulk_load(dst, src + a0, bytes(), bar);
    }
};

// RPT rows per consumer thread: a tile is 256 * RPT rows, thread t owns rows
// t, t + 256, ... of it, and issues the first gathers of all its rows before
// accumulating any (more loads in flight per register).  Partial sums stay
// per 256-row block in the same warp and lane order, so reductions do not
// depend on RPT.
//
// Column entries are stored as C: the column itself (C == I) or, for
// int16_t, its offset from the row (column = row + entry), which cuts the
// index stream from 4 to 2 bytes per nonzero for operators whose couplings
// lie within 32767 rows of the diagonal.
//
// With early != 0 (the matrix is not written by any kernel still in flight)
// the producer fills the first `stages` chunks before waiting for the
// previous kernel of the stream (programmatic dependent launch), so the
// matrix stream overlaps that kernel's tail; the consumers, which read x and
// the epilogue operands, always wait first.
template <class C>
__device__ __forceinline__ int64_t column_of(int64_t row, C entry) {
    if constexpr (std::is_same_v<C, int16_t>) return row + entry;
    else return static_cast<int64_t>(entry);
}

template <class T, class I, class C, int RPT, class XS, class Epi, class V = T>
__global__ void __launch_bounds__(kThreads + 32) csr_pipe_kernel(int64_t rows, int64_t nnz, const I *__restrict__ rp,
                                                                  const C *__restrict__ ci,
                                                                  const V *__restrict__ val, int cap, int stages,
                                                                  int early, XS xs, Epi epi, int *fault) {
    constexpr int K = Epi::kReduce;
    constexpr int KK = K > 0 ? K : 1;
    constexpr int kVT = 16 / sizeof(V), kVC = 16 / sizeof(C);
    constexpr int kTileRows = kThreads * RPT;
    constexpr int kWarps = kThreads / 32;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t full_bar[kMaxStages], empty_bar[kMaxStages];
    __shared__ double warp_sums[kMaxStages + 1][RPT][kWarps][KK];
    __shared__ int warp_done[kMaxStages + 1];
    __shared__ int skipped_cta;
    const StageLayout<V, I, C> L(cap, kTileRows);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kWarps);
        }
        for (int s = 0; s < kMaxStages + 1; ++s) warp_done[s] = 0;
        mbar_fence_init();
    }
    __syncthreads();
    auto stage_rp = [&](int s) { return reinterpret_cast<I *>(smem + static_cast<size_t>(s) * L.bytes); };
    auto stage_val = [&](int s) {
        return reinterpret_cast<V *>(smem + static_cast<size_t>(s) * L.bytes + L.rp_bytes);
    };
    auto stage_col = [&](int s) {
        return reinterpret_cast<C *>(smem + static_cast<size_t>(s) * L.bytes + L.rp_bytes + L.val_bytes);
    };
    const int64_t ntiles = (rows + kTileRows - 1) / kTileRows;
    const int64_t nblocks = (rows + kThreads - 1) / kThreads;  // 256-row blocks = partial sums
    bool ok = true;
    uint32_t armed[kMaxStages] = {0, 0, 0, 0};  // producer: completions requested per stage

    if (tid == kThreads) {
        // ---- producer ----
        uint32_t it = 0;
        bool entered = false, stop = false;
        auto enter = [&] {
            if (!entered) {
                entered = true;
                pdl_enter();
                stop = epi.skip();
            }
            return stop;
        };
        if (!early) enter();
        for (int64_t tile = blockIdx.x; tile < ntiles && ok && !stop; tile += gridDim.x) {
            const int64_t r0 = tile * kTileRows;
            const int nr = static_cast<int>(min(static_cast<int64_t>(kTileRows), rows - r0));
            const int64_t s = rp[r0], e = rp[r0 + nr];
            const int64_t nch = e > s ? (e - s + cap - 1) / cap : 1;
            for (int64_t c = 0; c < nch && ok; ++c, ++it) {
                const int st = static_cast<int>(it % stages);
                if (it >= static_cast<uint32_t>(stages)) {
                    if (enter()) break;
                    if (!mbar_wait(&empty_bar[st], ((it / stages) + 1) & 1)) {
                        ok = false;
                        break;
                    }
                }
                const int64_t cs = s + c * cap, ce = min(e, cs + cap);
                Range<I> rr;
                if (c == 0) rr.plan(r0, r0 + nr + 1, rows + 1);
                else rr.plan(r0, r0, rows + 1);
                Range<V> rv;
                rv.plan(cs, ce, nnz);
                Range<C> rc;
                rc.plan(cs, ce, nnz);
                rr.plain(stage_rp(st), rp);
                rv.plain(stage_val(st), val);
                rc.plain(stage_col(st), ci);
                mbar_arrive_expect_tx(&full_bar[st], rr.bytes() + rv.bytes() + rc.bytes());
                ++armed[st];
                rr.issue(stage_rp(st), rp, &full_bar[st]);
                rv.issue(stage_val(st), val, &full_bar[st]);
                rc.issue(stage_col(st), ci, &full_bar[st]);
            }
        }
        enter();
        if (!ok) atomicExch(fault, 1);
    } else if (tid < kThreads) {
        // ---- consumers: RPT rows per thread ----
        pdl_enter();
        const int lane = tid & 31, warp = tid >> 5;
        uint32_t it = 0, local_tile = 0;
        double red[RPT][KK];
        const bool skipped = epi.skip();
        if (tid == 0) skipped_cta = skipped ? 1 : 0;
        const int64_t first = skipped ? ntiles : blockIdx.x;
        // entry offsets in the index type's width (32-bit arithmetic for int32 CSR)
        using Off = std::conditional_t<sizeof(I) == 4, int32_t, int64_t>;
        for (int64_t tile = first; tile < ntiles && ok; tile += gridDim.x) {
            const int64_t r0 = tile * kTileRows;
            const int nr = static_cast<int>(min(static_cast<int64_t>(kTileRows), rows - r0));
            Off rs[RPT], re[RPT], s = 0, e = 0;
            int nch = 1;
            T acc[RPT];
            // x~ around each of this thread's rows (gathers by column offset)
            decltype(xs.row(0)) xv[RPT];
#pragma unroll
            for (int k = 0; k < RPT; ++k) xv[k] = xs.row(r0 + tid + k * kThreads);
            // The rows' own epilogue operands (b, D^-1, x_i, ...) are loaded
            // now, so their latency overlaps the stage wait and the gathers.
            typename Epi::Pre pre[RPT];
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                rs[k] = re[k] = 0;
                acc[k] = T(0);
                pre[k] = typename Epi::Pre{};
                if (tid + k * kThreads < nr) pre[k] = epi.pre(r0 + tid + k * kThreads, xs);
#pragma unroll
                for (int q = 0; q < KK; ++q) red[k][q] = 0.0;
            }
            for (int c = 0; c < nch; ++c, ++it) {
                const int st = static_cast<int>(it % stages);
                // warp-uniform decision, so __syncwarp below never waits on a lane that left
                if (__any_sync(0xffffffffu, !mbar_wait(&full_bar[st], (it / stages) & 1))) {
                    ok = false;
                    if (lane == 0) atomicExch(fault, 1);
                    break;
                }
                if (c == 0) {
                    const I *srp = stage_rp(st);
                    s = static_cast<Off>(srp[0]);
                    e = static_cast<Off>(srp[nr]);
                    nch = e > s ? static_cast<int>((static_cast<int64_t>(e) - s + cap - 1) / cap) : 1;
#pragma unroll
                    for (int k = 0; k < RPT; ++k)
                        if (tid + k * kThreads < nr) {
                            rs[k] = srp[tid + k * kThreads];
                            re[k] = srp[tid + k * kThreads + 1];
                        }
                }
                const Off cs = s + static_cast<Off>(c) * cap, ce = min(e, cs + static_cast<Off>(cap));
                const V *sv = stage_val(st) + (cs % kVT);  // sv[j - cs]
                const C *sc = stage_col(st) + (cs % kVC);  // sc[j - cs]
                constexpr int kGather = 8;
                int lo[RPT], hi[RPT];
                T y[RPT][kGather];
                // x~_j of entry o of row k: through the row's view when the
                // entries are column offsets (a 32-bit offset per gather)
                auto gather = [&](int k, int o) {
                    if constexpr (std::is_same_v<C, int16_t>) return xv[k](sc[o]);
                    else return xs(column_of(r0 + tid + k * kThreads, sc[o]));
                };
#pragma unroll
                for (int k = 0; k < RPT; ++k) {
                    lo[k] = static_cast<int>(max(rs[k], cs) - cs);
                    hi[k] = static_cast<int>(max(min(re[k], ce) - cs, Off(0)));
#pragma unroll
                    for (int u = 0; u < kGather; ++u) {
                        const int o = lo[k] + u;
                        y[k][u] = o < hi[k] ? gather(k, o) : T(0);
                    }
                }
#pragma unroll
                for (int k = 0; k < RPT; ++k) {
                    T a = acc[k];
#pragma unroll
                    for (int u = 0; u < kGather; ++u) {
                        const int o = lo[k] + u;
                        a += (o < hi[k] ? sv[o] : T(0)) * y[k][u];
                    }
                    for (int o0 = lo[k] + kGather; o0 < hi[k]; o0 += kGather) {
                        T z[kGather];
#pragma unroll
                        for (int u = 0; u < kGather; ++u) {
                            const int o = o0 + u;
                            z[u] = o < hi[k] ? gather(k, o) : T(0);
                        }
#pragma unroll
                        for (int u = 0; u < kGather; ++u) {
                            const int o = o0 + u;
                            a += (o < hi[k] ? sv[o] : T(0)) * z[u];
                        }
                    }
                    acc[k] = a;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_bar[st]);
            }
            if (!ok) break;
#pragma unroll
            for (int k = 0; k < RPT; ++k)
                if (tid + k * kThreads < nr) epi(r0 + tid + k * kThreads, acc[k], pre[k], red[k]);
            if constexpr (K > 0) {
                // Per-256-row-block partial sums, independent of the grid and
                // of RPT: each warp reduces its rows of every block, the last
                // warp of the tile to finish adds the eight warp sums in warp
                // order.  Warps are at most `stages` tiles apart, so a ring of
                // kMaxStages + 1 slots never overwrites a slot still being read.
                const int slot = static_cast<int>(local_tile % (kMaxStages + 1));
#pragma unroll
                for (int k = 0; k < RPT; ++k)
#pragma unroll
                    for (int q = 0; q < K; ++q)
                        for (int o = 16; o > 0; o >>= 1) red[k][q] += __shfl_down_sync(0xffffffffu, red[k][q], o);
                if (lane == 0) {
#pragma unroll
                    for (int k = 0; k < RPT; ++k)
#pragma unroll
                        for (int q = 0; q < K; ++q) warp_sums[slot][k][warp][q] = red[k][q];
                    __threadfence_block();
                    if (atomicAdd(&warp_done[slot], 1) == kWarps - 1) {
                        __threadfence_block();
                        for (int k = 0; k < RPT; ++k) {
                            const int64_t block = tile * RPT + k;
                            if (block >= nblocks) break;
#pragma unroll
                            for (int q = 0; q < K; ++q) {
                                double v = 0.0;
                                for (int w = 0; w < kWarps; ++w) v += warp_sums[slot][k][w][q];
                                epi.partial[q * nblocks + block] = v;
                            }
                        }
                        warp_done[slot] = 0;
                    }
                }
            }
            ++local_tile;
        }
    }
    __syncthreads();
    pdl_trigger();  // the main loop is done: the next kernel may be scheduled
    if (tid == kThreads) {
        // No copy of this CTA may still be in flight when it exits: wait
        // (bounded; immediate when the consumers consumed everything) for the
        // last phase armed on every stage.
        for (int st = 0; st < stages; ++st)
            if (armed[st]) mbar_wait(&full_bar[st], (armed[st] - 1) & 1);
    }
    if constexpr (K > 0) {
        // the scalar step that consumes the partial sums, in the last CTA
        // (the gate is the same in every CTA: all count or none does)
        __syncthreads();
        if (!skipped_cta) finish(epi.fin, epi.partial, static_cast<int>(nblocks));
    }
}

// ---------------------------------------------------------------------------
// Sliced kernel (operators that carry a sliced copy, Csr::sp).
//
// A CTA of eight warps walks 256-row tiles (the same tiles, and so the same
// 256-row blocks of partial sums, as the kernels above); warp w of a tile
// owns slice 8 tile + w, lane l its row 32 s + l.  Entry j of every row of
// a slice is one coalesced load across the warp (values and 2-byte column
// offsets), so no staging, no per-row chunk bounds and no shared memory are
// needed.  The first G entries of a slice are loaded ahead: for the launch's
// first tile before the dependency wait when the matrix is stable (early),
// and with PF for the CTA's next tile while the current one gathers x.  A
// row accumulates its entries left to right from +0 exactly as the
// row-per-thread kernels do (padding adds 0 * 0, which leaves any sum that
// starts at +0 unchanged), so every output and partial sum is bit-identical.
// A sorted copy (perm) orders the rows of each tile longest first, so a
// slice's rows have similar lengths; lane l then computes row perm[slot]
// (every output is still the same bits; only epilogues without partial sums
// are launched on it).
// ---------------------------------------------------------------------------
// Where a slice entry's column offset comes from.  c = cols.at(base, j,
// lane) is the offset from the lane's row of entry j of the slice that
// starts at entry base, or kColPad for a padding entry (no gather).
constexpr int kColPad = INT_MIN;

// Sliced copy: one 2-byte offset per entry, loaded with the values.
struct OffsetCols {
    const int16_t *__restrict__ sc;
    __device__ __forceinline__ int at(int base, int j, int lane) const {
        const int16_t c = __ldcs(sc + base + j * 32 + lane);
        return c == kSlicePad ? kColPad : c;
    }
};

// Banded copy: one {offset, padding mask} pair per slot, shared by the
// slice's 32 rows (a broadcast load per warp, cached).
struct BandCols {
    const int2 *__restrict__ bd;
    __device__ __forceinline__ int at(int base, int j, int lane) const {
        const int2 q = __ldg(bd + (base >> 5) + j);
        return (static_cast<unsigned>(q.y) >> lane) & 1u ? kColPad : q.x;
    }
};

template <class T, int G>
struct SliceHead {
    T v[G];
    int c[G];
    int32_t base, width;
};

template <class T, int G, class Cols>
__device__ __forceinline__ void load_slice_head(SliceHead<T, G> &h, int64_t slice, int64_t nslices,
                                                const int32_t *__restrict__ sp, const T *__restrict__ sv,
                                                const Cols &cols, int lane) {
    h.base = 0;
    h.width = 0;
    if (slice < nslices) {
        h.base = __ldg(sp + slice);
        h.width = (__ldg(sp + slice + 1) - h.base) >> 5;
    }
    const T *pv = sv + h.base + lane;  // entry g of this lane's row at pv[32 g]
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (g < h.width) {
            h.v[g] = __ldcs(pv + g * 32);
            h.c[g] = cols.at(h.base, g, lane);
        } else {
            h.v[g] = T(0);
            h.c[g] = kColPad;
        }
    }
}

template <class T, int G, bool PF, class XS, class Epi, class Cols, class V = T>
__global__ void __launch_bounds__(kThreads) sliced_kernel(int64_t rows, const int32_t *__restrict__ sp,
                                                          const V *__restrict__ sv, Cols cols,
                                                          const int32_t *__restrict__ perm, int early, XS xs,
                                                          Epi epi) {
    constexpr int K = Epi::kReduce;
    constexpr int KK = K > 0 ? K : 1;
    constexpr int kWarps = kThreads / 32;
    // warp sums, double-buffered by tile parity: one barrier per tile suffices
    __shared__ double warp_sums[2][kWarps][KK];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // sliced copies exist for int32 operators only: 32-bit row arithmetic
    const int nrows = static_cast<int>(rows);
    const int ntiles = (nrows + kThreads - 1) / kThreads;  // = 256-row blocks of partial sums
    const int nslices = (nrows + 31) / 32;
    int tile = blockIdx.x;
    SliceHead<V, G> h;
    if (early) load_slice_head(h, tile * kWarps + warp, nslices, sp, sv, cols, lane);
    pdl_enter();
    if (epi.skip()) return;  // the gate reads the same device word in every CTA
    if (!early) load_slice_head(h, tile * kWarps + warp, nslices, sp, sv, cols, lane);
    for (int parity = 0; tile < ntiles; tile += gridDim.x, parity ^= 1) {
        const int slot = tile * kThreads + threadIdx.x;  // position in the sliced order
        const bool live = slot < nrows;
        const int row = live && perm ? __ldg(perm + slot) : slot;
        typename Epi::Pre pre{};
        if (live) pre = epi.pre(row, xs);
        SliceHead<V, G> next;
        if constexpr (PF) load_slice_head(next, (tile + gridDim.x) * kWarps + warp, nslices, sp, sv, cols, lane);
        const auto xr = xs.row(row);  // x~ around this lane's row, indexed by column offset
        T y[G];
#pragma unroll
        for (int g = 0; g < G; ++g) y[g] = h.c[g] != kColPad ? xr(h.c[g]) : T(0);
        T acc = T(0);
#pragma unroll
        for (int g = 0; g < G; ++g) acc += h.v[g] * y[g];
        for (int j0 = G; j0 < h.width; j0 += G) {
            V v[G];
            int c[G];
            const V *pv = sv + h.base + lane + j0 * 32;
#pragma unroll
            for (int g = 0; g < G; ++g) {
                if (j0 + g < h.width) {
                    v[g] = __ldcs(pv + g * 32);
                    c[g] = cols.at(h.base, j0 + g, lane);
                } else {
                    v[g] = V(0);
                    c[g] = kColPad;
                }
            }
#pragma unroll
            for (int g = 0; g < G; ++g) y[g] = c[g] != kColPad ? xr(c[g]) : T(0);
#pragma unroll
            for (int g = 0; g < G; ++g) acc += v[g] * y[g];
        }
        double red[KK];
#pragma unroll
        for (int q = 0; q < KK; ++q) red[q] = 0.0;
        if (live) epi(row, acc, pre, red);
        if constexpr (K > 0) {
#pragma unroll
            for (int q = 0; q < K; ++q)
                for (int o = 16; o > 0; o >>= 1) red[q] += __shfl_down_sync(0xffffffffu, red[q], o);
            if (lane == 0)
#pragma unroll
                for (int q = 0; q < K; ++q) warp_sums[parity][warp][q] = red[q];
            // a warp writes this parity's slots again two tiles later, past
            // the next barrier, which thread q reaches only after this read
            __syncthreads();
            if (threadIdx.x < K) {
                double v = 0.0;
                for (int w = 0; w < kWarps; ++w) v += warp_sums[parity][w][threadIdx.x];
                epi.partial[threadIdx.x * static_cast<int64_t>(ntiles) + tile] = v;
            }
        }
        if constexpr (PF) h = next;
        else if (tile + static_cast<int>(gridDim.x) < ntiles)
            load_slice_head(h, (tile + gridDim.x) * kWarps + warp, nslices, sp, sv, cols, lane);
    }
    pdl_trigger();  // the main loop is done: the next kernel may be scheduled
    if constexpr (K > 0) finish(epi.fin, epi.partial, ntiles);
}

// ---------------------------------------------------------------------------
// Staged sliced kernel: the sliced or banded copy streamed through shared
// memory.
//
// A group of R tiles (8 R slices, 256 R rows) is contiguous in the copy
// (entries [sp[8 R g], sp[8 R (g + 1)]) of the values and of the column
// source), so the producer thread (warp 8, lane 0) moves a whole group with
// two bulk copies into a ring stage.  Slice starts are multiples of 32
// entries, so the value copy starts and ends on 16-byte boundaries (the
// column sources keep theirs, see below).  The producer also writes the
// group's 8 R + 1 slice starts into the stage header before arming the
// stage.  Consumer warp w owns slice w of each of the group's tiles, lane l
// its row, and reads its slices from shared memory lane by lane (consecutive
// addresses: no bank conflicts); only the x gathers leave the SM.  R amortises
// the per-stage work (the waits, the header, the producer's copies) over R
// slices per warp.  Row sums, epilogues and the per-256-row-block partial
// sums are those of the kernels above: the same bits.  Every wait is bounded
// as in csr_pipe_kernel (fault word, drain of the CTA's own copies).
// ---------------------------------------------------------------------------
// Column sources of the staged kernel: what the producer copies next to a
// group's values (entries [e0, e1) of the copy) and how a consumer lane
// reads slot j of its slice from the stage: take(j, c) is false for a
// padding entry, else sets c to the column offset from the lane's row.
//
// Sliced copy: the group's 2-byte offsets, one per entry.
struct StagedOffsets {
    const int16_t *__restrict__ sc;
    static __host__ __device__ int stage_bytes(int cap) { return (cap * 2 + 127) & ~127; }
    __device__ __forceinline__ uint32_t bytes(int64_t e0, int64_t e1) const {
        return static_cast<uint32_t>((e1 - e0) * 2);
    }
    __device__ __forceinline__ void copy(void *dst, int64_t e0, int64_t e1, uint64_t *bar) const {
        bulk_load(dst, sc + e0, bytes(e0, e1), bar);
    }
    struct View {
        const int16_t *p;
        __device__ __forceinline__ bool take(int j, int &c) const {
            const int16_t v = p[j * 32];
            c = v;
            return v != kSlicePad;
        }
    };
    // base: the slice's first entry, relative to e0
    __device__ __forceinline__ View view(const void *stage, int64_t, int base, int lane) const {
        return {static_cast<const int16_t *>(stage) + base + lane};
    }
};

// Banded copy: the group's {offset, padding mask} slots (one per 32
// entries), copied from the even slot at or below e0 / 32 to the even slot
// at or above e1 / 32, so that both ends sit on 16-byte boundaries (the band
// array is allocated to an even number of slots).  A lane reads the slot as
// a broadcast (one shared-memory word for the whole warp) and tests its own
// bit of the mask.
struct StagedBand {
    const int2 *__restrict__ bd;
    static __host__ __device__ int stage_bytes(int cap) { return ((cap / 32 + 2) * 8 + 127) & ~127; }
    static __device__ __forceinline__ int64_t lo(int64_t e0) { return (e0 >> 5) & ~int64_t(1); }
    static __device__ __forceinline__ int64_t hi(int64_t e1) { return ((e1 >> 5) + 1) & ~int64_t(1); }
    __device__ __forceinline__ uint32_t bytes(int64_t e0, int64_t e1) const {
        return static_cast<uint32_t>((hi(e1) - lo(e0)) * 8);
    }
    __device__ __forceinline__ void copy(void *dst, int64_t e0, int64_t e1, uint64_t *bar) const {
        bulk_load(dst, bd + lo(e0), bytes(e0, e1), bar);
    }
    struct View {
        const int2 *q;
        unsigned bit;
        __device__ __forceinline__ bool take(int j, int &c) const {
            const int2 v = q[j];
            c = v.x;
            return (static_cast<unsigned>(v.y) & bit) == 0u;
        }
    };
    __device__ __forceinline__ View view(const void *stage, int64_t e0, int base, int lane) const {
        return {static_cast<const int2 *>(stage) + ((e0 >> 5) - lo(e0)) + (base >> 5), 1u << lane};
    }
};

// One ring stage: the header of R * 8 + 1 slice starts, the values, the
// column source.  cap: the stage's entry capacity.
template <class T, class Cols, int R>
struct SlicedStage {
    static constexpr int kHeader = ((R * 8 + 1) * 4 + 63) & ~63;
    int val_bytes, col_bytes, bytes;
    __host__ __device__ explicit SlicedStage(int cap) {
        val_bytes = (cap * static_cast<int>(sizeof(T)) + 127) & ~127;
        col_bytes = Cols::stage_bytes(cap);
        bytes = (kHeader + val_bytes + col_bytes + 127) & ~127;
    }
};

// Four values of a stage, 16-byte aligned, into registers.
template <class T>
__device__ __forceinline__ void load4(T (&v)[4], const T *p) {
    if constexpr (sizeof(T) == 4) {
        const float4 t = *reinterpret_cast<const float4 *>(p);
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else {
        const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
}

// Four consecutive x values from global memory, 16-byte aligned, through
// the read-only path.
template <class T>
__device__ __forceinline__ void load4_ldg(T (&v)[4], const T *p) {
    if constexpr (sizeof(T) == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else {
        const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p + 2));
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
}

// kQuad (banded copies, R = 4, epilogues without partial sums): consumer
// lanes take four consecutive rows each instead of one -- warp w owns
// slices 4w..4w+3 of the group, lane 8q + p rows 4p..4p+3 of slice 4w + q.
// Per slot a lane reads the slot pair once for its four rows, their four
// values with one 16-byte load (slices start on 32-entry boundaries, so a
// row quad's values are 16-byte aligned in the stage) and gathers x at four
// consecutive addresses, which cuts the instructions per entry about in
// half; each row still adds its products slot by slot from +0.
template <class T, int R, class XS, class Epi, class Cols, bool kQuad = false, class V = T>
__global__ void __launch_bounds__(kThreads + 32)
    sliced_pipe_kernel(int64_t rows, const int32_t *__restrict__ sp, const V *__restrict__ sv, Cols cols, int cap,
                       int stages, int early, XS xs, Epi epi, int *fault) {
    static_assert(!kQuad || (R == 4 && Epi::kReduce == 0 && std::is_same_v<Cols, StagedBand>),
                  "the four-rows-per-lane form serves banded copies in groups of 4 tiles without partial sums");
    constexpr int K = Epi::kReduce;
    constexpr int KK = K > 0 ? K : 1;
    constexpr int kWarps = kThreads / 32;
    constexpr int kSlices = kWarps * R;  // slices per group
    constexpr int kRing = kMaxStages * R + 1;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t full_bar[kMaxStages], empty_bar[kMaxStages];
    __shared__ double warp_sums[kRing][kWarps][KK];
    __shared__ int warp_done[kRing];
    __shared__ int skipped_cta;
    using Stage = SlicedStage<V, Cols, R>;
    const Stage L(cap);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int st = 0; st < stages; ++st) {
            mbar_init(&full_bar[st], 1);
            mbar_init(&empty_bar[st], kWarps);
        }
        for (int st = 0; st < kRing; ++st) warp_done[st] = 0;
        mbar_fence_init();
    }
    __syncthreads();
    auto stage_hdr = [&](int st) { return reinterpret_cast<int32_t *>(smem + static_cast<size_t>(st) * L.bytes); };
    auto stage_val = [&](int st) {
        return reinterpret_cast<V *>(smem + static_cast<size_t>(st) * L.bytes + Stage::kHeader);
    };
    auto stage_col = [&](int st) {
        return static_cast<void *>(smem + static_cast<size_t>(st) * L.bytes + Stage::kHeader + L.val_bytes);
    };
    const int64_t ntiles = (rows + kThreads - 1) / kThreads;  // = 256-row blocks of partial sums
    const int64_t ngroups = (ntiles + R - 1) / R;
    const int64_t nslices = (rows + 31) / 32;
    bool ok = true;
    uint32_t armed[kMaxStages] = {0, 0, 0, 0};  // producer: completions requested per stage

    if (tid == kThreads) {
        // ---- producer ----
        uint32_t it = 0;
        bool entered = false, stop = false;
        auto enter = [&] {
            if (!entered) {
                entered = true;
                pdl_enter();
                stop = epi.skip();
            }
            return stop;
        };
        if (!early) enter();
        // the group's first and last slice starts are loaded one group
        // ahead, so their latency overlaps the wait for a free stage; the
        // others are loaded before that wait
        auto start_at = [&](int64_t s) { return __ldg(sp + (s < nslices ? s : nslices)); };
        int32_t next0 = 0, next1 = 0;
        if (static_cast<int64_t>(blockIdx.x) < ngroups) {
            next0 = start_at(blockIdx.x * static_cast<int64_t>(kSlices));
            next1 = start_at((blockIdx.x + 1) * static_cast<int64_t>(kSlices));
        }
        for (int64_t grp = blockIdx.x; grp < ngroups && ok && !stop; grp += gridDim.x, ++it) {
            const int64_t e0 = next0, e1 = next1;
            const int64_t s0 = grp * kSlices;
            if (grp + gridDim.x < ngroups) {
                next0 = start_at((grp + gridDim.x) * kSlices);
                next1 = start_at((grp + gridDim.x + 1) * kSlices);
            }
            int32_t mid[kSlices - 1];
#pragma unroll
            for (int k = 1; k < kSlices; ++k) mid[k - 1] = start_at(s0 + k);
            const int st = static_cast<int>(it % stages);
            if (it >= static_cast<uint32_t>(stages)) {
                if (enter()) break;
                if (!mbar_wait(&empty_bar[st], ((it / stages) + 1) & 1)) {
                    ok = false;
                    break;
                }
            }
            int32_t *hdr = stage_hdr(st);
            hdr[0] = static_cast<int32_t>(e0);
#pragma unroll
            for (int k = 1; k < kSlices; ++k) hdr[k] = mid[k - 1];
            hdr[kSlices] = static_cast<int32_t>(e1);
            const uint32_t nv = static_cast<uint32_t>((e1 - e0) * static_cast<int64_t>(sizeof(V)));
            const uint32_t nc = e1 > e0 ? cols.bytes(e0, e1) : 0;
            mbar_arrive_expect_tx(&full_bar[st], nv + nc);
            ++armed[st];
            if (e1 > e0) {
                bulk_load(stage_val(st), sv + e0, nv, &full_bar[st]);
                cols.copy(stage_col(st), e0, e1, &full_bar[st]);
            }
        }
        enter();
        if (!ok) atomicExch(fault, 1);
    } else if (kQuad && tid < kThreads) {
        if constexpr (kQuad) {
            // ---- consumers, four rows per lane ----
            pdl_enter();
            const int lane = tid & 31, warp = tid >> 5;
            const int q = lane >> 3, p = lane & 7;
            const int s = warp * 4 + q;  // the lane's slice within the group
            uint32_t it = 0;
            const bool skipped = epi.skip();
            if (tid == 0) skipped_cta = skipped ? 1 : 0;
            const int64_t first = skipped ? ngroups : blockIdx.x;
            for (int64_t grp = first; grp < ngroups && ok; grp += gridDim.x, ++it) {
                const int64_t row0 = grp * (R * kThreads) + s * 32 + 4 * p;
                typename Epi::Pre pre[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    pre[k] = typename Epi::Pre{};
                    if (row0 + k < rows) pre[k] = epi.pre(row0 + k, xs);
                }
                const int st = static_cast<int>(it % stages);
                if (__any_sync(0xffffffffu, !mbar_wait(&full_bar[st], (it / stages) & 1))) {
                    ok = false;
                    if (lane == 0) atomicExch(fault, 1);
                    break;
                }
                const int32_t *hdr = stage_hdr(st);
                const int base = hdr[s] - hdr[0];
                const int width = (hdr[s + 1] - hdr[s]) >> 5;
                const int2 *band = static_cast<const int2 *>(stage_col(st)) +
                                   static_cast<int>((hdr[0] >> 5) - StagedBand::lo(hdr[0])) + (base >> 5);
                const V *vs = stage_val(st) + base + 4 * p;
                const auto xr = xs.row(row0);
                T acc[4] = {T(0), T(0), T(0), T(0)};
                for (int j0 = 0; j0 < width; j0 += 8) {
                    T y[8][4];
#pragma unroll
                    for (int g = 0; g < 8; ++g) {
                        int c = 0;
                        unsigned pad = 0xFu;  // bit k: row 4p + k has no entry in this slot
                        if (j0 + g < width) {
                            const int2 v = band[j0 + g];
                            c = v.x;
                            pad = (static_cast<unsigned>(v.y) >> (4 * p)) & 0xFu;
                        }
                        if constexpr (std::is_same_v<std::remove_cv_t<decltype(xr)>, typename PlainX<T>::View>) {
                            // the four rows' x values in one 16-byte load when they
                            // are all entries (no index outside x) and their address
                            // is 16-byte aligned; else one load per entry
                            if (pad == 0u && (reinterpret_cast<uintptr_t>(xr.p + c) & 15u) == 0) {
                                load4_ldg(y[g], xr.p + c);
                                continue;
                            }
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) y[g][k] = (pad >> k) & 1u ? T(0) : xr(c + k);
                    }
#pragma unroll
                    for (int g = 0; g < 8; ++g) {
                        if (j0 + g < width) {
                            V v[4];
                            load4(v, vs + (j0 + g) * 32);
#pragma unroll
                            for (int k = 0; k < 4; ++k) acc[k] += v[k] * y[g][k];
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_bar[st]);
                double red[1] = {0.0};
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (row0 + k < rows) epi(row0 + k, acc[k], pre[k], red);
            }
        }
    } else if (tid < kThreads) {
        // ---- consumers: warp w owns slice w of each tile of the group ----
        pdl_enter();
        const int lane = tid & 31, warp = tid >> 5;
        uint32_t it = 0, local_block = 0;
        const bool skipped = epi.skip();
        if (tid == 0) skipped_cta = skipped ? 1 : 0;
        const int64_t first = skipped ? ngroups : blockIdx.x;
        for (int64_t grp = first; grp < ngroups && ok; grp += gridDim.x, ++it) {
            typename Epi::Pre pre[R];
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int64_t row = (grp * R + k) * kThreads + tid;
                pre[k] = typename Epi::Pre{};
                if (row < rows) pre[k] = epi.pre(row, xs);
            }
            const int st = static_cast<int>(it % stages);
            if (__any_sync(0xffffffffu, !mbar_wait(&full_bar[st], (it / stages) & 1))) {
                ok = false;
                if (lane == 0) atomicExch(fault, 1);
                break;
            }
            const int32_t *hdr = stage_hdr(st);
            // The first 8 slots of all R slices are gathered before any
            // product is added (8 R loads in flight per lane: the x gathers'
            // L2 latency, not the bytes, bounds this loop), then each row
            // adds its products left to right, slots past 8 in a second loop.
            // A padding entry (value 0 in the copy) gathers nothing and adds
            // 0 * 0 = +0: a row sum starts at +0 and never becomes -0 (an
            // exact cancellation rounds to +0), so adding +0 leaves every
            // bit of it as the entry-by-entry sum of the CSR kernels.
            T acc[R];
            T y[R][8];
            int base[R], width[R];
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int s = k * kWarps + warp;
                base[k] = hdr[s] - hdr[0];
                width[k] = (hdr[s + 1] - hdr[s]) >> 5;
                const auto cs = cols.view(stage_col(st), hdr[0], base[k], lane);
                const auto xr = xs.row((grp * R + k) * kThreads + tid);
#pragma unroll
                for (int g = 0; g < 8; ++g) {
                    int c = 0;
                    y[k][g] = g < width[k] && cs.take(g, c) ? xr(c) : T(0);
                }
            }
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const V *vs = stage_val(st) + base[k] + lane;
                T a = T(0);
#pragma unroll
                for (int g = 0; g < 8; ++g) a += (g < width[k] ? vs[g * 32] : T(0)) * y[k][g];
                if (width[k] > 8) {
                    const auto cs = cols.view(stage_col(st), hdr[0], base[k], lane);
                    const auto xr = xs.row((grp * R + k) * kThreads + tid);
                    for (int j0 = 8; j0 < width[k]; j0 += 8) {
                        T z[8];
#pragma unroll
                        for (int g = 0; g < 8; ++g) {
                            int c = 0;
                            z[g] = j0 + g < width[k] && cs.take(j0 + g, c) ? xr(c) : T(0);
                        }
#pragma unroll
                        for (int g = 0; g < 8; ++g) a += (j0 + g < width[k] ? vs[(j0 + g) * 32] : T(0)) * z[g];
                    }
                }
                acc[k] = a;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty_bar[st]);
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int64_t block = grp * R + k;
                const int64_t row = block * kThreads + tid;
                double red[KK];
#pragma unroll
                for (int q = 0; q < KK; ++q) red[q] = 0.0;
                if (row < rows) epi(row, acc[k], pre[k], red);
                if constexpr (K > 0) {
                    // as in csr_pipe_kernel: the last warp of the block adds
                    // the eight warp sums in warp order; warps are at most
                    // `stages` groups apart, so a ring of kMaxStages R + 1
                    // slots never overwrites a slot still being read
                    const int slot = static_cast<int>(local_block % kRing);
#pragma unroll
                    for (int q = 0; q < K; ++q)
                        for (int o = 16; o > 0; o >>= 1) red[q] += __shfl_down_sync(0xffffffffu, red[q], o);
                    if (lane == 0 && block < ntiles) {
#pragma unroll
                        for (int q = 0; q < K; ++q) warp_sums[slot][warp][q] = red[q];
                        __threadfence_block();
                        if (atomicAdd(&warp_done[slot], 1) == kWarps - 1) {
                            __threadfence_block();
#pragma unroll
                            for (int q = 0; q < K; ++q) {
                                double v = 0.0;
                                for (int w = 0; w < kWarps; ++w) v += warp_sums[slot][w][q];
                                epi.partial[q * ntiles + block] = v;
                            }
                            warp_done[slot] = 0;
                        }
                    }
                }
                ++local_block;
            }
        }
    }
    __syncthreads();
    pdl_trigger();  // the main loop is done: the next kernel may be scheduled
    if (tid == kThreads) {
        for (int st = 0; st < stages; ++st)
            if (armed[st]) mbar_wait(&full_bar[st], (armed[st] - 1) & 1);
    }
    if constexpr (K > 0) {
        __syncthreads();
        if (!skipped_cta) finish(epi.fin, epi.partial, static_cast<int>(ntiles));
    }
}

// Pipelined launch shape: rows per thread, entries per chunk, stages in the
// ring, resident CTAs per SM (the persistent grid is ctas_per_sm x SMs, at
// most one CTA per tile).
struct PipeShape {
    int rpt, cap, stages, ctas_per_sm, grid;
    size_t smem;
};

// Tunable part of the shape: rows per thread, ring depth, resident CTAs per
// SM and the chunk capacity as a percentage of the mean tile.  The result
// does not depend on it (rows are reduced left to right in any chunking,
// partial sums are per 256-row block), only the speed does.
struct PipeConfig {
    int stages{2}, ctas_per_sm{4}, cap_pct{125}, rpt{1};
    // Operators with a sliced copy: stream it with sliced_ctas resident CTAs
    // per SM, sliced = 1 directly (sliced_kernel, next-tile prefetch when
    // set), sliced = 2 through a ring of sliced_stages shared-memory stages
    // (sliced_pipe_kernel, sliced_group tiles per stage: 1, 2 or 4), sliced =
    // 3 the same with four rows per consumer lane (banded copies, 4 tiles
    // per stage).
    int sliced{0}, sliced_ctas{4}, prefetch{1}, sliced_stages{2}, sliced_group{1};
};

// Stage capacity (entries) of the staged sliced kernel for a's copy in
// groups of R tiles: R times its largest tile, or 0 when a stage would
// exceed 96 KB.
template <class T, class Cols, int R>
int sliced_stage_cap_for(int64_t tile_max) {
    const int64_t cap = (tile_max * R + 255) & ~int64_t(255);
    if (cap <= 0 || cap > (int64_t(96) << 10)) return 0;
    return SlicedStage<T, Cols, R>(static_cast<int>(cap)).bytes <= (96 << 10) ? static_cast<int>(cap) : 0;
}
template <class T, class I, class V>
int sliced_stage_cap(const Csr<T, I, V> &a, int group) {
    switch (group) {
        case 4: return a.bd ? sliced_stage_cap_for<V, StagedBand, 4>(a.sl_tile_max)
                            : sliced_stage_cap_for<V, StagedOffsets, 4>(a.sl_tile_max);
        case 2: return a.bd ? sliced_stage_cap_for<V, StagedBand, 2>(a.sl_tile_max)
                            : sliced_stage_cap_for<V, StagedOffsets, 2>(a.sl_tile_max);
        default: return a.bd ? sliced_stage_cap_for<V, StagedBand, 1>(a.sl_tile_max)
                             : sliced_stage_cap_for<V, StagedOffsets, 1>(a.sl_tile_max);
    }
}

// Dynamic shared memory the staged kernel's ring may take (the per-block
// opt-in limit, 227 KB on B200, less its static barriers and sums).
constexpr size_t kStagedSmemMax = size_t(200) << 10;

// Shared memory of one stage of the staged kernel over a's copy.
template <class T, class I, class V>
size_t sliced_stage_bytes(const Csr<T, I, V> &a, int group, int cap) {
    auto bytes = [&](auto cols) -> size_t {
        using Cols = decltype(cols);
        switch (group) {
            case 4: return SlicedStage<V, Cols, 4>(cap).bytes;
            case 2: return SlicedStage<V, Cols, 2>(cap).bytes;
            default: return SlicedStage<V, Cols, 1>(cap).bytes;
        }
    };
    return a.bd ? bytes(StagedBand{}) : bytes(StagedOffsets{});
}

// A kernel as a type, for the helpers that take it as a template argument.
template <auto K>
struct KernelTag {
    static constexpr auto kernel = K;
};

// Calls f(KernelTag<kernel>, cols) with the staged kernel instantiation for
// a's column source and the group size; quad: the four-rows-per-lane form,
// where it applies (a banded copy, an epilogue without partial sums; group
// 4 is then implied).
template <class T, class I, class XS, class Epi, class F, class V>
decltype(auto) with_staged_kernel(const Csr<T, I, V> &a, int group, F &&f, bool quad = false) {
    auto pick = [&](auto cols) -> decltype(auto) {
        using Cols = decltype(cols);
        if constexpr (std::is_same_v<Cols, StagedBand> && Epi::kReduce == 0)
            if (quad) return f(KernelTag<sliced_pipe_kernel<T, 4, XS, Epi, Cols, true, V>>{}, cols);
        switch (group) {
            case 4: return f(KernelTag<sliced_pipe_kernel<T, 4, XS, Epi, Cols, false, V>>{}, cols);
            case 2: return f(KernelTag<sliced_pipe_kernel<T, 2, XS, Epi, Cols, false, V>>{}, cols);
            default: return f(KernelTag<sliced_pipe_kernel<T, 1, XS, Epi, Cols, false, V>>{}, cols);
        }
    };
    if (a.bd) return pick(StagedBand{a.bd});
    return pick(StagedOffsets{a.sc});
}

template <class T, class I, class C = I>
PipeShape pipe_shape(int64_t rows, int64_t nnz, int sm_count, const PipeConfig &cfg) {
    PipeShape p;
    p.rpt = cfg.rpt == 2 ? 2 : 1;
    const int tile_rows = kThreads * p.rpt;
    const int rp_bytes = ((tile_rows + 1 + 16 / static_cast<int>(sizeof(I))) * static_cast<int>(sizeof(I)) + 15) & ~15;
    const int stage_limit = 32768 * p.rpt;
    const int max_cap = ((stage_limit - rp_bytes) / static_cast<int>(sizeof(T) + sizeof(C)) - 8) & ~63;
    const int64_t mean_tile = rows > 0 ? (nnz * tile_rows + rows - 1) / rows : 0;
    int64_t cap = (mean_tile * cfg.cap_pct / 100 + 63) & ~int64_t(63);
    if (cap < 256) cap = 256;
    if (cap > max_cap) cap = max_cap;
    p.cap = static_cast<int>(cap);
    p.stages = cfg.stages;
    p.ctas_per_sm = cfg.ctas_per_sm;
    p.smem = static_cast<size_t>(StageLayout<T, I, C>(p.cap, tile_rows).bytes) * p.stages;
    const int64_t ntiles = (rows + tile_rows - 1) / tile_rows;
    const int64_t g = static_cast<int64_t>(sm_count) * cfg.ctas_per_sm;
    p.grid = static_cast<int>(ntiles < g ? (ntiles < 1 ? 1 : ntiles) : g);
    return p;
}

// Number of partial sums a reducing launch writes: one per 256-row block.
inline int partials(int64_t rows) { return static_cast<int>(rows > 0 ? (rows + kThreads - 1) / kThreads : 1); }

// Process-wide cache of tuned configurations, keyed by the operator's shape
// and storage (value, row offset and column entry sizes).
struct TuneKey {
    int64_t rows, nnz;
    int vsize, isize, csize, sm_count;
    bool operator<(const TuneKey &o) const {
        return std::tie(rows, nnz, vsize, isize, csize, sm_count) <
               std::tie(o.rows, o.nnz, o.vsize, o.isize, o.csize, o.sm_count);
    }
};
inline std::mutex &tune_mutex() {
    static std::mutex m;
    return m;
}
inline std::map<TuneKey, PipeConfig> &tune_cache() {
    static std::map<TuneKey, PipeConfig> m;
    return m;
}
// (values of type V under vectors of type T: V's size, plus 100 when the
// two differ, so FP32 values under FP64 vectors keep shapes of their own)
template <class T, class I, class C, class V = T>
TuneKey tune_key(int64_t rows, int64_t nnz, int sm_count) {
    return TuneKey{rows, nnz, static_cast<int>(sizeof(V)) + (std::is_same_v<T, V> ? 0 : 100),
                   static_cast<int>(sizeof(I)), static_cast<int>(sizeof(C)), sm_count};
}
template <class T, class I, class C, class V = T>
PipeConfig tuned_config(int64_t rows, int64_t nnz, int sm_count) {
    std::lock_guard<std::mutex> lock(tune_mutex());
    auto it = tune_cache().find(tune_key<T, I, C, V>(rows, nnz, sm_count));
    return it == tune_cache().end() ? PipeConfig{} : it->second;
}
template <class T, class I, class C, class V = T>
bool has_config(int64_t rows, int64_t nnz, int sm_count) {
    std::lock_guard<std::mutex> lock(tune_mutex());
    return tune_cache().count(tune_key<T, I, C, V>(rows, nnz, sm_count)) != 0;
}
template <class T, class I, class C, class V = T>
void store_config(int64_t rows, int64_t nnz, int sm_count, const PipeConfig &cfg) {
    std::lock_guard<std::mutex> lock(tune_mutex());
    tune_cache()[tune_key<T, I, C, V>(rows, nnz, sm_count)] = cfg;
}

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Calls f(cols) with the column stream the pipelined kernel reads for a:
// the 2-byte row offsets when the operator carries them, else the indices.
template <class T, class I, class F, class V>
decltype(auto) with_columns(const Csr<T, I, V> &a, F &&f) {
    if constexpr (std::is_same_v<I, int32_t>) {
        if (a.cd && aligned16(a.cd)) return f(a.cd);
    }
    return f(a.ci);
}

// Validates and caches a launch shape for operators of a's shape.
template <class T, class I, class V>
void configure(tf_ctx *ctx, const Csr<T, I, V> &a, const PipeConfig &cfg) {
    require(cfg.rpt == 1 || cfg.rpt == 2, "rows_per_thread must be 1 or 2");
    require(cfg.stages >= 2 && cfg.stages <= kMaxStages, "stages must be 2..4");
    require(cfg.ctas_per_sm >= 1 && cfg.ctas_per_sm <= 8, "ctas_per_sm must be 1..8");
    require(cfg.cap_pct >= 50 && cfg.cap_pct <= 400, "cap_pct must be 50..400");
    with_columns(a, [&](auto cols) {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(cols)>>;
        const PipeShape p = pipe_shape<V, I, C>(a.rows, a.nnz, ctx->sm_count, cfg);
        require(p.smem <= 200 * 1024, "stage ring exceeds shared memory");
        store_config<T, I, C, V>(a.rows, a.nnz, ctx->sm_count, cfg);
    });
}

// Resident CTAs per SM of an instantiation at this block size and dynamic
// shared memory (cached per instantiation, device and size).  Persistent
// grids are clamped to it at launch: an epilogue that needs more registers
// than the one a shape was tuned with must not spill CTAs into a second wave.
template <auto Kernel>
int resident_ctas(int threads, size_t smem) {
    static thread_local int dev_c = -1, threads_c = 0, res = 0;
    static thread_local size_t smem_c = 0;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != dev_c || threads != threads_c || smem != smem_c) {
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res, Kernel, threads, smem), "occupancy");
        dev_c = dev;
        threads_c = threads;
        smem_c = smem;
    }
    return res;
}

// Bytes written between timed tuning launches to push the operator out of
// the L2 cache (126 MB on B200).
constexpr size_t kTuneFlushBytes = size_t(192) << 20;

// Opts the instantiation into the dynamic shared memory it is launched with
// (the staged chunk plus the epilogue's static reduction buffer can exceed
// the 48 KB default).  The attribute belongs to the function on a device,
// for every thread of the process, so it only ever grows: per device the
// largest size any thread asked for (a thread that lowered it could make
// another thread's launch fail).
template <auto Kernel>
void allow_smem(size_t bytes) {
    static thread_local int seen_device = -1;
    static thread_local size_t seen_bytes = 0;  // known granted on seen_device
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev == seen_device && bytes <= seen_bytes) return;
    static std::mutex m;
    static std::map<int, size_t> granted;
    std::lock_guard<std::mutex> lock(m);
    size_t &g = granted[dev];
    if (bytes > g) {
        cuda_check(cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
                   "tile shared memory");
        g = bytes;
    }
    seen_device = dev;
    seen_bytes = g;
}

// Epilogues whose launches are usually skipped say so (rarely_runs()).
template <class E>
auto rarely_runs(const E &e, int) -> decltype(e.rarely_runs()) {
    return e.rarely_runs();
}
template <class E>
bool rarely_runs(const E &, long) {
    return false;
}

template <class T, class I, class C, class XS, class Epi, class V>
void launch_pipe(tf_ctx *ctx, const Csr<T, I, V> &a, const C *cols, const XS &xs, const Epi &epi, const char *name,
                 const PipeConfig *force) {
    const PipeConfig cfg = force ? *force : tuned_config<T, I, C, V>(a.rows, a.nnz, ctx->sm_count);
    const PipeShape p = pipe_shape<V, I, C>(a.rows, a.nnz, ctx->sm_count, cfg);
    const int early = ctx->stable && !rarely_runs(epi, 0) ? 1 : 0;
    auto grid = [&](int resident) {
        const int64_t g = static_cast<int64_t>(ctx->sm_count) * (resident > 0 ? resident : 1);
        return static_cast<int>(p.grid < g ? p.grid : g);
    };
    if (p.rpt == 2) {
        allow_smem<csr_pipe_kernel<T, I, C, 2, XS, Epi, V>>(p.smem);
        const int g = grid(resident_ctas<csr_pipe_kernel<T, I, C, 2, XS, Epi, V>>(kThreads + 32, p.smem));
        launch_kernel(ctx, name, csr_pipe_kernel<T, I, C, 2, XS, Epi, V>, g, kThreads + 32, p.smem, a.rows, a.nnz, a.rp,
                      cols, a.val, p.cap, p.stages, early, xs, epi, ctx->fault);
    } else {
        allow_smem<csr_pipe_kernel<T, I, C, 1, XS, Epi, V>>(p.smem);
        const int g = grid(resident_ctas<csr_pipe_kernel<T, I, C, 1, XS, Epi, V>>(kThreads + 32, p.smem));
        launch_kernel(ctx, name, csr_pipe_kernel<T, I, C, 1, XS, Epi, V>, g, kThreads + 32, p.smem, a.rows, a.nnz, a.rp,
                      cols, a.val, p.cap, p.stages, early, xs, epi, ctx->fault);
    }
}

template <class T, class I, class XS, class Epi, class V>
void launch_sliced(tf_ctx *ctx, const Csr<T, I, V> &a, const XS &xs, const Epi &epi, const char *name,
                   const PipeConfig &cfg) {
    const int64_t ntiles = (a.rows + kThreads - 1) / kThreads;
    const int early = ctx->stable && !rarely_runs(epi, 0) ? 1 : 0;
    if (cfg.sliced >= 2 && !a.perm) {
        // sliced = 3: four rows per lane over a banded copy (epilogues with
        // partial sums take the one-row form with the same stages)
        const bool quad = cfg.sliced == 3 && a.bd && Epi::kReduce == 0;
        const int group = cfg.sliced == 3 ? 4 : cfg.sliced_group;
        const int cap = sliced_stage_cap(a, group);
        const size_t stage = cap > 0 ? sliced_stage_bytes(a, group, cap) : 0;
        // a ring deeper than the shared memory holds runs with fewer stages
        // (the stage count changes the speed only)
        const int stages = stage ? std::min<int>(cfg.sliced_stages, static_cast<int>(kStagedSmemMax / stage)) : 0;
        if (stages >= 2) {
            const size_t smem = stage * stages;
            const int64_t ngroups = (ntiles + group - 1) / group;
            with_staged_kernel<T, I, XS, Epi>(a, group, [&](auto tag, auto cols) {
                constexpr auto kernel = decltype(tag)::kernel;
                allow_smem<kernel>(smem);
                const int resident = resident_ctas<kernel>(kThreads + 32, smem);
                const int per_sm = cfg.sliced_ctas < resident || resident < 1 ? cfg.sliced_ctas : resident;
                const int64_t g = static_cast<int64_t>(ctx->sm_count) * per_sm;
                launch_kernel(ctx, name, kernel, static_cast<int>(ngroups < g ? ngroups : g), kThreads + 32, smem,
                              a.rows, a.sp, a.sv, cols, cap, stages, early, xs, epi, ctx->fault);
            }, quad);
            return;
        }
    }
    auto grid = [&](int resident) {
        const int per_sm = cfg.sliced_ctas < resident || resident < 1 ? cfg.sliced_ctas : resident;
        const int64_t g = static_cast<int64_t>(ctx->sm_count) * per_sm;
        return static_cast<int>(ntiles < g ? ntiles : g);
    };
    auto go = [&](auto cols) {
        using Cols = decltype(cols);
        if (cfg.prefetch)
            launch_kernel(ctx, name, sliced_kernel<T, 8, true, XS, Epi, Cols, V>,
                          grid(resident_ctas<sliced_kernel<T, 8, true, XS, Epi, Cols, V>>(kThreads, 0)), kThreads, 0,
                          a.rows, a.sp, a.sv, cols, a.perm, early, xs, epi);
        else
            launch_kernel(ctx, name, sliced_kernel<T, 8, false, XS, Epi, Cols, V>,
                          grid(resident_ctas<sliced_kernel<T, 8, false, XS, Epi, Cols, V>>(kThreads, 0)), kThreads, 0,
                          a.rows, a.sp, a.sv, cols, a.perm, early, xs, epi);
    };
    if (a.bd) go(BandCols{a.bd});
    else go(OffsetCols{a.sc});
}

// The launch shape cached for an operator's sliced or banded copy: it is
// stored under the column stream its row-tile kernel reads (2-byte offsets
// when the operator has them, else its indices).
template <class T, class I, class V>
PipeConfig copy_config(tf_ctx *ctx, const Csr<T, I, V> &a) {
    return a.cd ? tuned_config<T, I, int16_t, V>(a.rows, a.nnz, ctx->sm_count)
                : tuned_config<T, I, I, V>(a.rows, a.nnz, ctx->sm_count);
}

// Launches the sliced kernel when the operator carries a sliced copy and its
// tuned configuration picks it, else the pipelined kernel when the arrays
// start on 16-byte boundaries (every buffer this library allocates does),
// the staged kernel otherwise.  Reducing epilogues need one of the first
// two: they write their partial sums per 256-row block (tile::partials).
template <class T, class I, class XS, class Epi, class V>
void launch(tf_ctx *ctx, const Csr<T, I, V> &a, const XS &xs, const Epi &epi, const char *name,
            const PipeConfig *force = nullptr) {
    if (a.rows == 0) return;
    if constexpr (std::is_same_v<I, int32_t>) {
        // a sorted copy permutes rows within their tile, which would change
        // the order of a reducing epilogue's partial sums: row tiles then
        if (a.sp && (a.cd || a.bd) && (!a.perm || Epi::kReduce == 0)) {
            const PipeConfig cfg = force ? *force : copy_config(ctx, a);
            if (cfg.sliced) {
                launch_sliced(ctx, a, xs, epi, name, cfg);
                return;
            }
        }
    }
    const bool pipe = aligned16(a.rp) && (a.nnz == 0 || (aligned16(a.ci) && aligned16(a.val)));
    if (pipe) {
        with_columns(a, [&](auto cols) { launch_pipe(ctx, a, cols, xs, epi, name, force); });
        return;
    }
    require(Epi::kReduce == 0, "reducing SpMV epilogues need 16-byte aligned CSR arrays");
    const SpmvShape shape = spmv_shape(a.rows, a.nnz, sizeof(V), sizeof(I));
    const int64_t tile_rows = static_cast<int64_t>(kThreads) * shape.rows_per_thread;
    const unsigned g = static_cast<unsigned>((a.rows + tile_rows - 1) / tile_rows);
    const size_t smem = static_cast<size_t>(shape.chunk) * (sizeof(V) + sizeof(I));
    if (shape.rows_per_thread == 2) {
        allow_smem<csr_tile_kernel<T, I, 2, XS, Epi, V>>(smem);
        launch_kernel(ctx, name, csr_tile_kernel<T, I, 2, XS, Epi, V>, g, kThreads, smem, a.rows, a.rp, a.ci, a.val,
                      shape.chunk, xs, epi);
    } else {
        allow_smem<csr_tile_kernel<T, I, 1, XS, Epi, V>>(smem);
        launch_kernel(ctx, name, csr_tile_kernel<T, I, 1, XS, Epi, V>, g, kThreads, smem, a.rows, a.rp, a.ci, a.val,
                      shape.chunk, xs, epi);
    }
}

// y = b - A x epilogue used to time candidate shapes (the residual and
// Jacobi sweeps of the cycle read a row operand besides x, as this does).
template <class T>
struct TuneStore {
    static constexpr int kReduce = 0;
    struct Pre {
        T b;
    };
    const T *__restrict__ b;
    T *__restrict__ y;
    double *partial{nullptr};
    __device__ __forceinline__ bool skip() const { return false; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &) const {
        return {b[i]};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&)[1]) const {
        y[i] = p.b - acc;
    }
};

// THERMOFEM_B200_TUNE_LOG=1 prints every timed candidate to stderr.
inline bool tune_log() {
    static const bool on = [] {
        const char *v = std::getenv("THERMOFEM_B200_TUNE_LOG");
        return v && v[0] == '1';
    }();
    return on;
}

template <class T, class I, class C, class V>
PipeConfig autotune_columns(tf_ctx *ctx, const Csr<T, I, V> &a, const T *x, T *y, float *best_ms) {
    PipeConfig best{};
    float best_t = 0;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    // Each timed launch starts as it does inside a solve.  An operator larger
    // than half the L2 cache is evicted by the rest of a cycle before its
    // next use: it is timed cold (a write of more than the L2 size before
    // every launch, then a copy x -> y, so x and y are recently touched);
    // smaller ones are timed back to back.
    const bool cold = static_cast<double>(a.nnz) * (sizeof(V) + sizeof(C)) +
                          static_cast<double>(a.rows) * (sizeof(I) + 2 * sizeof(T)) >
                      static_cast<double>(kTuneFlushBytes) / 3;
    // (the context's second scratch arena: allocated once, kept for later setups)
    unsigned char *flush = cold ? static_cast<unsigned char *>(ctx->arena(kTuneFlushBytes, 1)) : nullptr;
    auto time_cfg = [&](const PipeConfig &cfg) {
        for (int w = 0; w < 2; ++w) launch(ctx, a, PlainX<T>{x}, TuneStore<T>{x, y, nullptr}, "autotune", &cfg);
        if (!cold) {
            cuda_check(cudaEventRecord(e0, ctx->stream), "event");
            for (int r = 0; r < 5; ++r) launch(ctx, a, PlainX<T>{x}, TuneStore<T>{x, y, nullptr}, "autotune", &cfg);
            cuda_check(cudaEventRecord(e1, ctx->stream), "event");
            cuda_check(cudaEventSynchronize(e1), "event");
            float ms = 0;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event");
            return ms / 5;
        }
        float total = 0;
        for (int r = 0; r < 5; ++r) {
            cuda_check(cudaMemsetAsync(flush, r, kTuneFlushBytes, ctx->stream), "tune flush");
            cuda_check(cudaMemcpyAsync(y, x, static_cast<size_t>(a.rows) * sizeof(T), cudaMemcpyDeviceToDevice,
                                       ctx->stream),
                       "tune copy");
            cuda_check(cudaEventRecord(e0, ctx->stream), "event");
            launch(ctx, a, PlainX<T>{x}, TuneStore<T>{x, y, nullptr}, "autotune", &cfg);
            cuda_check(cudaEventRecord(e1, ctx->stream), "event");
            cuda_check(cudaEventSynchronize(e1), "event");
            float ms = 0;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event");
            total += ms;
        }
        return total / 5;
    };
    bool first = true;
    for (int rpt : {1, 2}) {
        for (int stages : {2, 3}) {
            for (int ctas : {1, 2, 3, 4, 5, 6}) {
                for (int pct : {100, 125}) {
                    const PipeConfig cfg{stages, ctas, pct, rpt};
                    const PipeShape p = pipe_shape<V, I, C>(a.rows, a.nnz, ctx->sm_count, cfg);
                    if (p.smem * ctas > 220 * 1024) continue;
                    if ((rpt == 1 && ctas < 2) || (rpt == 2 && ctas > 3)) continue;
                    int resident = 0;
                    if (rpt == 2) {
                        allow_smem<csr_pipe_kernel<T, I, C, 2, PlainX<T>, TuneStore<T>, V>>(p.smem);
                        resident = resident_ctas<csr_pipe_kernel<T, I, C, 2, PlainX<T>, TuneStore<T>, V>>(kThreads + 32,
                                                                                                       p.smem);
                    } else {
                        allow_smem<csr_pipe_kernel<T, I, C, 1, PlainX<T>, TuneStore<T>, V>>(p.smem);
                        resident = resident_ctas<csr_pipe_kernel<T, I, C, 1, PlainX<T>, TuneStore<T>, V>>(kThreads + 32,
                                                                                                       p.smem);
                    }
                    if (resident < ctas) continue;
                    const float ms = time_cfg(cfg);
                    if (tune_log())
                        std::fprintf(stderr,
                                     "tf_autotune_spmv rows=%lld nnz=%lld T=%d C=%d rpt=%d stages=%d ctas=%d cap=%d%% "
                                     "%.2f us\n",
                                     static_cast<long long>(a.rows), static_cast<long long>(a.nnz),
                                     static_cast<int>(sizeof(T)), static_cast<int>(sizeof(C)), rpt, stages, ctas, pct,
                                     ms * 1e3f);
                    if (first || ms < best_t) {
                        best_t = ms;
                        best = cfg;
                        first = false;
                    }
                }
            }
        }
    }
    if constexpr (std::is_same_v<I, int32_t>) {
        // a sliced copy (2-byte offsets: tuned under C = int16_t) or a banded one
        if (a.sp && (a.bd || std::is_same_v<C, int16_t>)) {
            // The sliced copy: next-tile prefetch on/off x resident CTAs per
            // SM, unless THERMOFEM_B200_SLICED_SHAPE="prefetch,ctas" forces one.
            int forced_pf = -1, forced_ctas = 0;
            if (const char *v = std::getenv("THERMOFEM_B200_SLICED_SHAPE"))
                if (std::sscanf(v, "%d,%d", &forced_pf, &forced_ctas) != 2) forced_pf = -1;
            PipeConfig sbest = best;
            float sbest_t = 0;
            bool sfirst = true;
            // shapes: (kind, prefetch or stages, ctas, group); kind 1 direct,
            // 2 staged (group: tiles per stage)
            std::vector<std::tuple<int, int, int, int>> shapes;
            if (forced_pf >= 0) {
                // "prefetch,ctas" forces the direct kernel, "2,stages,ctas[,group]" the staged one
                int a3 = 0, a4 = 1;
                const char *v = std::getenv("THERMOFEM_B200_SLICED_SHAPE");
                const int got = v ? std::sscanf(v, "%d,%d,%d,%d", &forced_pf, &forced_ctas, &a3, &a4) : 0;
                const int group = forced_pf == 3 ? 4 : (got == 4 && (a4 == 2 || a4 == 4) ? a4 : 1);
                if (got >= 3 && forced_pf == 3 && a.bd && sliced_stage_cap(a, 4))
                    shapes.emplace_back(3, forced_ctas < 2 ? 2 : (forced_ctas > kMaxStages ? kMaxStages : forced_ctas),
                                        a3 < 1 ? 1 : a3, 4);
                else if (got >= 3 && forced_pf == 2 && sliced_stage_cap(a, group))
                    shapes.emplace_back(2, forced_ctas < 2 ? 2 : (forced_ctas > kMaxStages ? kMaxStages : forced_ctas),
                                        a3 < 1 ? 1 : a3, group);
                else
                    shapes.emplace_back(1, forced_pf ? 1 : 0, forced_ctas < 1 ? 1 : forced_ctas, 1);
            } else {
                for (int pf : {0, 1})
                    for (int ctas : {2, 3, 4, 5, 6}) shapes.emplace_back(1, pf, ctas, 1);
                for (int group : {1, 2, 4})
                    if (sliced_stage_cap(a, group))
                        for (int stg : {2, 3, 4})
                            for (int ctas : {1, 2, 3, 4, 5}) shapes.emplace_back(2, stg, ctas, group);
                if (a.bd && sliced_stage_cap(a, 4))
                    for (int stg : {2, 3, 4})
                        for (int ctas : {1, 2, 3, 4}) shapes.emplace_back(3, stg, ctas, 4);
            }
            for (const auto &[kind, knob, ctas, group] : shapes) {
                {
                    PipeConfig cfg = best;
                    cfg.sliced = kind;
                    cfg.sliced_ctas = ctas;
                    int resident = 0;
                    if (kind >= 2) {
                        cfg.sliced_stages = knob;
                        cfg.sliced_group = group;
                        const size_t stage = sliced_stage_bytes(a, group, sliced_stage_cap(a, group));
                        if ((stage * knob > kStagedSmemMax || stage * knob * ctas > 220 * 1024) && forced_pf < 0)
                            continue;
                        // (a forced ring deeper than the shared memory runs shallower, as launch_sliced does)
                        const size_t smem = stage * std::min<int>(knob, static_cast<int>(kStagedSmemMax / stage));
                        resident = with_staged_kernel<T, I, PlainX<T>, TuneStore<T>>(
                            a, group,
                            [&](auto tag, auto) {
                                constexpr auto kernel = decltype(tag)::kernel;
                                allow_smem<kernel>(smem);
                                return resident_ctas<kernel>(kThreads + 32, smem);
                            },
                            kind == 3);
                    } else {
                        cfg.prefetch = knob;
                        // (the column source does not change the kernel's registers much; offsets bound it)
                        resident = knob ? resident_ctas<sliced_kernel<T, 8, true, PlainX<T>, TuneStore<T>, OffsetCols, V>>(
                                              kThreads, 0)
                                        : resident_ctas<sliced_kernel<T, 8, false, PlainX<T>, TuneStore<T>, OffsetCols, V>>(
                                              kThreads, 0);
                    }
                    if (resident < ctas && forced_pf < 0) continue;
                    const float ms = time_cfg(cfg);
                    if (tune_log())
                        std::fprintf(stderr,
                                     "tf_autotune_spmv rows=%lld nnz=%lld T=%d %s %s=%d ctas=%d group=%d %.2f us\n",
                                     static_cast<long long>(a.rows), static_cast<long long>(a.nnz),
                                     static_cast<int>(sizeof(T)), a.bd ? "banded" : "sliced",
                                     kind == 3 ? "quad stages" : (kind == 2 ? "staged stages" : "prefetch"), knob, ctas,
                                     group, ms * 1e3f);
                    if (sfirst || ms < sbest_t) {
                        sbest_t = ms;
                        sbest = cfg;
                        sfirst = false;
                    }
                }
            }
            if (!sfirst && (forced_pf >= 0 || sbest_t < best_t)) {
                best = sbest;
                best_t = sbest_t;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_faults(ctx);
    store_config<T, I, C, V>(a.rows, a.nnz, ctx->sm_count, best);
    if (best_ms) *best_ms = best_t;
    return best;
}

// Times the feasible rows per thread, ring depths, CTAs per SM and chunk
// capacities on this operator (two warm-up and five timed launches each,
// CUDA events on the context stream) and caches the fastest for every later
// launch over an operator of the same shape and storage.  y is overwritten.
template <class T, class I, class V>
PipeConfig autotune(tf_ctx *ctx, const Csr<T, I, V> &a, const T *x, T *y, float *best_ms) {
    if (a.rows == 0 || !aligned16(a.rp) || (a.nnz && (!aligned16(a.ci) || !aligned16(a.val)))) return PipeConfig{};
    return with_columns(a, [&](auto cols) {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(cols)>>;
        return autotune_columns<T, I, C, V>(ctx, a, x, y, best_ms);
    });
}

// True when operators of a's shape and storage already have a cached shape.
template <class T, class I, class V>
bool tuned(tf_ctx *ctx, const Csr<T, I, V> &a) {
    return with_columns(a, [&](auto cols) {
        using C = std::remove_cv_t<std::remove_pointer_t<decltype(cols)>>;
        return has_config<T, I, C, V>(a.rows, a.nnz, ctx->sm_count);
    });
}

}  // namespace tile
}  // namespace tfb
