// coarse_cycle.cu -- the small levels of an AMG cycle as one thread-block
// cluster working out of distributed shared memory.
//
// Below a few ten thousand rows every level operation of the cycle is a few
// microseconds of launch and memory latency for well under a microsecond of
// work: each launched kernel chains three or four dependent global-memory
// round trips (row offsets, columns, gathered values).  Here the host records
// the level steps of the sub-cycle that starts at the first small level (the
// same recursion as the large levels: Cycle.cuh:35-63) and one cluster of up
// to 16 CTAs runs them.  Rows of every level (fewer than 65536) are split
// into equal contiguous ranges, one per CTA; a row's owner is a multiply-high
// by the range length's reciprocal (exact below 65536 rows).  At the start
// each CTA bulk-copies (cp.async.bulk, one copy per array, issued by as many
// threads) its rows' matrix entries,
// diagonal and transfer maps into its shared memory, together with the plan
// and the steps; every vector of the sub-cycle lives there too.  A gather of
// another row's value is a distributed shared-memory load from the owning
// CTA; the hardware cluster barrier (release/acquire) separates dependent
// steps.  All CTAs of a cluster are co-scheduled by construction, so no
// barrier can wait on a CTA that is not running.  Only the root level's
// vectors are read from and written back to global memory.
//
// Every step computes exactly what the launched kernels compute, in the
// same order: row products left to right, x_out = x + w d (b - A x),
// residuals rounded to the level type before the member sums of the
// restriction (member order), x = w d b from a zero guess, prolongation
// x += e[map] (or fine[m] += x_c over the members m of c), the dense coarse
// inverse with the warp-strided FP64 sum; so the cycle's result is the same
// to the bit.
//
// When every level of the region fits in one CTA's shared memory (about
// 25,000 nonzeros in FP32), the region is that one CTA: gathers are plain
// shared-memory loads and steps are separated by __syncthreads.  Measured on
// B200, a 16-CTA cluster barrier costs about a microsecond and a distributed
// shared-memory round trip about half of one, so the cluster form only pays
// when the levels do not fit in one CTA.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

#include "coarse_cycle.cuh"
#include "tile.cuh"

namespace cg = cooperative_groups;

namespace tfb {

namespace {

enum TailOp : int {
    kTZero = 0,
    kTJacobiZero = 1,
    kTSweep = 2,
    kTProlongSweep = 3,
    kTResidualRestrict = 4,
    kTRestrict = 5,
    kTProlong = 6,
    kTDense = 7,
};

constexpr int kTailMaxCluster = 16;

}  // namespace

template <class S>
struct TailLevelDev {
    int n, R;        // rows, rows per CTA
    int nn, Rn;      // rows and rows per CTA of the next level (0 on the last level)
    unsigned mag, cmag;  // ceil(2^32 / R), ceil(2^32 / Rn) (0 when the length is 1)
    int cols16;          // columns staged as 2-byte offsets from the row
    int e0[kTailMaxCluster], m0[kTailMaxCluster];  // per CTA: first entry of its rows, first member of its aggregates
    // shared-memory byte offsets of a CTA's share (the same in every CTA)
    unsigned o_rp, o_ci, o_val, o_dinv, o_rhs, o_x0, o_x1, o_map, o_off, o_mem;
};

struct TailStepDev {
    int op, level, a, b, c;
};

// One bulk copy into a CTA's shared memory: `bytes` (a multiple of 16) from
// a 16-byte aligned source, then a ragged end of up to seven 2-byte units.
struct TailCopy {
    const void *src;
    const void *tail_src;
    unsigned dst, bytes, tail_dst, tail_halves;
};

template <class S>
struct TailHeader {
    int levels, dense_n;
    S w;
    const double *inv;
    S *root_rhs, *root_x0, *root_x1;  // the root level's global vectors
    unsigned o_poff, o_pmem;          // the root's aggregates in the level above (restriction, prolongation)
    int pm0[kTailMaxCluster];         // per CTA: first member of its root rows there
    unsigned o_steps;                 // the steps' shared-memory byte offset
    unsigned copy_begin[kTailMaxCluster + 1];
    unsigned tx_bytes[kTailMaxCluster];
    TailLevelDev<S> lv[kTailMaxLevels];
};

template <class S>
struct TailDevice {
    DeviceBuffer<TailHeader<S>> header;
    DeviceBuffer<TailStepDev> steps;
    DeviceBuffer<TailCopy> copies;
};

namespace {

template <class T>
__device__ __forceinline__ T *at(unsigned char *base, unsigned off) {
    return reinterpret_cast<T *>(base + off);
}

// Rows per CTA and the reciprocal that finds a row's owner: for row < 2^16
// and R < 2^16, floor(row * ceil(2^32 / R) / 2^32) = floor(row / R).
struct Part {
    int R;
    unsigned mag;
};

// The CTAs of a region: a cluster (values of other CTAs' rows through
// distributed shared memory, the cluster barrier) or, when every level fits
// in one CTA, that CTA alone (plain shared-memory loads, __syncthreads).
template <bool kSingle>
struct Group {
    __device__ __forceinline__ int rank() const {
        if constexpr (kSingle) return 0;
        else return static_cast<int>(cg::this_cluster().block_rank());
    }
    __device__ __forceinline__ void sync() const {
        if constexpr (kSingle) __syncthreads();
        else cg::this_cluster().sync();
    }
    // Value of row `row` of the vector that sits at `local` in every CTA.
    template <class S>
    __device__ __forceinline__ S load(S *local, int row, Part p) const {
        if constexpr (kSingle) {
            return local[row];
        } else {
            const unsigned owner = p.mag ? __umulhi(static_cast<unsigned>(row), p.mag) : static_cast<unsigned>(row);
            return *cg::this_cluster().map_shared_rank(local + (row - static_cast<int>(owner) * p.R), owner);
        }
    }
};

// This CTA's share of a level.  The constant arrays were bulk-copied from
// 16-byte aligned starts, so each begins `lo % (16 / element size)` elements
// into its buffer; offsets (rp, off) are still global and rebased on use.
template <class S>
struct LevelView {
    int r0, nr, c0, nc, e0, m0;
    const int32_t *rp, *ci;
    const int16_t *cd;  // set instead of ci when the columns are row offsets
    const S *val, *dinv;
    const int32_t *map, *off, *mem;
};

template <class S>
__device__ __forceinline__ LevelView<S> view(unsigned char *sm, const TailLevelDev<S> &L, int rank) {
    constexpr int VI = 4, VS = 16 / static_cast<int>(sizeof(S));
    LevelView<S> v;
    v.r0 = rank * L.R;
    v.nr = max(0, min(L.R, L.n - v.r0));
    v.c0 = rank * L.Rn;
    v.nc = L.Rn > 0 ? max(0, min(L.Rn, L.nn - v.c0)) : 0;
    v.e0 = L.e0[rank];
    v.m0 = L.m0[rank];
    v.rp = at<int32_t>(sm, L.o_rp) + v.r0 % VI;
    v.ci = at<int32_t>(sm, L.o_ci) + v.e0 % VI;
    v.cd = L.cols16 ? at<int16_t>(sm, L.o_ci) + v.e0 % 8 : nullptr;
    v.val = at<S>(sm, L.o_val) + v.e0 % VS;
    v.dinv = at<S>(sm, L.o_dinv) + v.r0 % VS;
    v.map = at<int32_t>(sm, L.o_map) + v.r0 % VI;
    v.off = at<int32_t>(sm, L.o_off) + v.c0 % VI;
    v.mem = at<int32_t>(sm, L.o_mem) + v.m0 % VI;
    return v;
}

// Own row i times x, left to right, eight gathers in flight.
template <class G, class S>
__device__ __forceinline__ S row_product(const G &cl, const LevelView<S> &v, S *x, Part p, int i) {
    const int s = v.rp[i] - v.e0, e = v.rp[i + 1] - v.e0, row = v.r0 + i;
    S acc = S(0);
    for (int j0 = s; j0 < e; j0 += 8) {
        S y[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = j0 + u;
            const int col = j < e ? (v.cd ? row + v.cd[j] : v.ci[j]) : 0;
            y[u] = j < e ? cl.load(x, col, p) : S(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc += (j0 + u < e ? v.val[j0 + u] : S(0)) * y[u];
    }
    return acc;
}

template <class S>
__device__ __forceinline__ S *xbuf(unsigned char *sm, const TailLevelDev<S> &L, int sel) {
    return at<S>(sm, sel ? L.o_x1 : L.o_x0);
}

// Own aggregates of the next level: b = sum of src over their members; with
// jz >= 0 also x_jz = w d b there.
template <class G, class S>
__device__ __forceinline__ void restrict_own(const G &cl, unsigned char *sm, const TailLevelDev<S> &L,
                                             const TailLevelDev<S> &C, S *src, int jz, S w, int rank) {
    const LevelView<S> v = view(sm, L, rank), cv = view(sm, C, rank);
    S *crhs = at<S>(sm, C.o_rhs);
    S *cx = jz >= 0 ? xbuf(sm, C, jz) : nullptr;
    for (int k = threadIdx.x; k < v.nc; k += blockDim.x) {
        const int j0 = v.off[k] - v.m0, j1 = v.off[k + 1] - v.m0;
        S sum = S(0);
        for (int j = j0; j < j1; ++j) sum += cl.load(src, v.mem[j], Part{L.R, L.mag});
        crhs[k] = sum;
        if (cx) cx[k] = w * cv.dinv[k] * sum;
    }
}

template <class S, bool kSingle>
__global__ void __launch_bounds__(kTailThreads, 1)
    tail_kernel(const TailHeader<S> *ghdr, const TailStepDev *gsteps, const TailCopy *copies, int first, int count,
                ProgramIO<S> io, int root_cur, int early, int *fault) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ uint64_t load_bar;
    const Group<kSingle> cl;
    const int rank = cl.rank();
    const int tid = threadIdx.x, nt = blockDim.x;
    if (!early) pdl_wait();
    // the plan first (every step reads it), then this CTA's constant arrays
    // (read-only while a cycle runs) by bulk copies, one per thread
    {
        const int words = static_cast<int>(sizeof(TailHeader<S>) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(ghdr);
        int *dst = reinterpret_cast<int *>(sm);
        for (int k = tid; k < words; k += nt) dst[k] = __ldg(src + k);
    }
    if (tid == 0) {
        tile::mbar_init(&load_bar, 1);
        tile::mbar_fence_init();
    }
    __syncthreads();
    const TailHeader<S> &H = *reinterpret_cast<const TailHeader<S> *>(sm);
    {
        TailStepDev *st = at<TailStepDev>(sm, H.o_steps);
        const int words = count * static_cast<int>(sizeof(TailStepDev) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(gsteps + first);
        for (int k = tid; k < words; k += nt) reinterpret_cast<int *>(st)[k] = __ldg(src + k);
    }
    if (tid == 0) tile::mbar_arrive_expect_tx(&load_bar, H.tx_bytes[rank]);
    __syncthreads();
    for (unsigned k = H.copy_begin[rank] + tid; k < H.copy_begin[rank + 1]; k += nt) {
        const TailCopy c = copies[k];
        if (c.bytes) tile::bulk_load(sm + c.dst, c.src, c.bytes, &load_bar);
        for (unsigned q = 0; q < c.tail_halves; ++q)
            at<unsigned short>(sm, c.tail_dst)[q] = __ldg(reinterpret_cast<const unsigned short *>(c.tail_src) + q);
    }
    const bool loaded = tile::mbar_wait(&load_bar, 0);
    if (!loaded && tid == 0) atomicExch(fault, 1);
    if (early) pdl_wait();
    pdl_trigger();
    const S w = H.w;
    const TailStepDev *steps = at<TailStepDev>(sm, H.o_steps);
    const TailLevelDev<S> &R = H.lv[0];
    const LevelView<S> rv = view(sm, R, rank);
    // the root's aggregates in the level above: [poff[i], poff[i+1]) of pmem
    const int32_t *poff = at<int32_t>(sm, H.o_poff) + rv.r0 % 4;
    const int32_t *pmem = at<int32_t>(sm, H.o_pmem) + H.pm0[rank] % 4;
    __syncthreads();  // ragged ends written by other threads
    {
        // the root's right-hand side (restricted here, or as stored) and iterates
        S *rhs = at<S>(sm, R.o_rhs), *x0 = at<S>(sm, R.o_x0), *x1 = at<S>(sm, R.o_x1);
        for (int i = tid; i < rv.nr; i += nt) {
            const int row = rv.r0 + i;
            S b;
            if (io.rsrc) {
                const int j0 = poff[i] - H.pm0[rank], j1 = poff[i + 1] - H.pm0[rank];
                S t[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) t[u] = j0 + u < j1 ? io.rsrc[pmem[j0 + u]] : S(0);
                b = S(0);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (j0 + u < j1) b += t[u];
                for (int j = j0 + 4; j < j1; ++j) b += io.rsrc[pmem[j]];
            } else {
                b = H.root_rhs[row];
            }
            rhs[i] = b;
            x0[i] = H.root_x0[row];
            x1[i] = H.root_x1[row];
        }
    }
    cl.sync();
    for (int k = 0; k < count; ++k) {
        const TailStepDev st = steps[k];
        const TailLevelDev<S> &L = H.lv[st.level];
        const LevelView<S> v = view(sm, L, rank);
        const int nr = v.nr;
        const Part p{L.R, L.mag};
        S *rhs = at<S>(sm, L.o_rhs);
        S *xa = st.a >= 0 ? xbuf(sm, L, st.a) : nullptr;
        S *xb = st.b >= 0 ? xbuf(sm, L, st.b) : nullptr;
        switch (st.op) {
            case kTZero:
                for (int i = tid; i < nr; i += nt) xa[i] = S(0);
                break;
            case kTJacobiZero:
                for (int i = tid; i < nr; i += nt) xa[i] = w * v.dinv[i] * rhs[i];
                break;
            case kTProlong:
            case kTProlongSweep: {
                S *xc = xbuf(sm, H.lv[st.level + 1], st.c);
                for (int i = tid; i < nr; i += nt) xa[i] = xa[i] + cl.load(xc, v.map[i], Part{L.Rn, L.cmag});
                if (st.op == kTProlong) break;
                cl.sync();
                for (int i = tid; i < nr; i += nt)
                    xb[i] = xa[i] + w * v.dinv[i] * (rhs[i] - row_product(cl, v, xa, p, i));
                break;
            }
            case kTSweep:
                for (int i = tid; i < nr; i += nt)
                    xb[i] = xa[i] + w * v.dinv[i] * (rhs[i] - row_product(cl, v, xa, p, i));
                break;
            case kTResidualRestrict: {
                S *r = xbuf(sm, L, 1 - st.a);  // the ping-pong scratch buffer
                for (int i = tid; i < nr; i += nt) r[i] = rhs[i] - row_product(cl, v, xa, p, i);
                cl.sync();
                restrict_own(cl, sm, L, H.lv[st.level + 1], r, st.c, w, rank);
                break;
            }
            case kTRestrict:
                restrict_own(cl, sm, L, H.lv[st.level + 1], rhs, st.c, w, rank);
                break;
            case kTDense: {
                // one warp per own row of the dense inverse (dense_apply_kernel's sum)
                const int n = H.dense_n, warp = tid >> 5, lane = tid & 31;
                for (int i = warp; i < nr; i += nt >> 5) {
                    const int row = v.r0 + i;
                    double s = 0;
                    for (int j = lane; j < n; j += 32)
                        s += __ldg(H.inv + static_cast<int64_t>(row) * n + j) *
                             static_cast<double>(cl.load(rhs, j, p));
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                    if (lane == 0) xa[i] = static_cast<S>(s);
                }
                break;
            }
            default:
                break;
        }
        cl.sync();
    }
    {
        // the root back to global memory, and its prolongation when asked
        const S *rhs = at<S>(sm, R.o_rhs), *x0 = at<S>(sm, R.o_x0), *x1 = at<S>(sm, R.o_x1);
        for (int i = tid; i < rv.nr; i += nt) {
            const int row = rv.r0 + i;
            H.root_x0[row] = x0[i];
            H.root_x1[row] = x1[i];
            H.root_rhs[row] = rhs[i];
            if (io.sfine) {
                // members are distinct rows: all loads first, then the stores
                const S val = root_cur ? x1[i] : x0[i];
                const int j0 = poff[i] - H.pm0[rank], j1 = poff[i + 1] - H.pm0[rank];
                for (int jb = j0; jb < j1; jb += 4) {
                    int m[4];
                    S f[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        m[u] = jb + u < j1 ? pmem[jb + u] : -1;
                        f[u] = m[u] >= 0 ? io.sfine[m[u]] : S(0);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (m[u] >= 0) io.sfine[m[u]] = f[u] + val;
                }
            }
        }
    }
    if (!loaded && tid == 0) tile::mbar_wait(&load_bar, 0);  // no copy left in flight
}

unsigned align16(size_t v) { return static_cast<unsigned>((v + 15) & ~size_t(15)); }

// The dynamic shared memory a kernel may use is one attribute per function
// and device: raise it to what a region needs, never lower it (other
// regions of the process may need more).
template <auto Kernel>
void allow_region_smem(size_t bytes) {
    static std::mutex m;
    static std::map<int, size_t> granted;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(m);
    auto it = granted.find(dev);
    if (bytes <= 48 * 1024 || (it != granted.end() && bytes <= it->second)) return;
    cuda_check(cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
               "region shared memory");
    granted[dev] = bytes;
}

unsigned reciprocal(int64_t R) { return R > 1 ? static_cast<unsigned>(((uint64_t(1) << 32) + R - 1) / R) : 0u; }

}  // namespace

template <class S>
TailRegion<S>::TailRegion() = default;
template <class S>
TailRegion<S>::~TailRegion() = default;

namespace {

// A copy on the context's stream, waited for on that stream only.  Never the
// legacy default stream, which another thread's work or a capture in
// progress may be using.
void copy_and_wait(tf_ctx *ctx, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, const char *what) {
    if (!bytes) return;
    cuda_check(cudaMemcpyAsync(dst, src, bytes, kind, ctx->stream), what);
    cuda_check(cudaStreamSynchronize(ctx->stream), what);
}

}  // namespace

template <class S>
bool TailRegion<S>::plan(tf_ctx *ctx, const std::vector<TailLevel<S>> &levels, const TailParent &parent,
                         const double *inv, int dense_n, S w, int max_steps) {
    dev_.reset();
    cluster_ = 0;
    if (levels.empty() || levels.size() > static_cast<size_t>(kTailMaxLevels)) return false;
    // row offsets and aggregate offsets, to size every CTA's share
    std::vector<std::vector<int32_t>> rps(levels.size()), offs(levels.size());
    for (size_t d = 0; d < levels.size(); ++d) {
        const auto &L = levels[d];
        if (L.n <= 0 || L.n >= (1 << 16)) return false;
        rps[d].resize(static_cast<size_t>(L.n) + 1);
        copy_and_wait(ctx, rps[d].data(), L.rp, rps[d].size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                      "region plan");
        if (d + 1 < levels.size()) {
            if (!L.map || !L.off || !L.mem) return false;
            offs[d].resize(static_cast<size_t>(levels[d + 1].n) + 1);
            copy_and_wait(ctx, offs[d].data(), L.off, offs[d].size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          "region plan");
        }
    }
    if (!parent.off || !parent.mem || parent.n <= 0) return false;
    std::vector<int32_t> poffs(static_cast<size_t>(levels[0].n) + 1);
    copy_and_wait(ctx, poffs.data(), parent.off, poffs.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                  "region plan");
    int max_optin = 0;
    cuda_check(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device),
               "shared memory limit");
    cuda_check(cudaFuncSetAttribute(tail_kernel<S, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
               "cluster attribute");
    auto h = std::make_unique<TailHeader<S>>();
    // one CTA when everything fits there (no cluster barrier, no remote
    // loads), else the largest cluster that holds the levels
    for (int C : {1, kTailMaxCluster, 8, 4, 2}) {
        std::memset(h.get(), 0, sizeof(TailHeader<S>));
        h->levels = static_cast<int>(levels.size());
        h->dense_n = dense_n;
        h->w = w;
        h->inv = inv;
        h->root_rhs = levels[0].rhs;
        h->root_x0 = levels[0].x0;
        h->root_x1 = levels[0].x1;
        std::vector<std::vector<TailCopy>> cps(static_cast<size_t>(C));
        std::vector<size_t> tx(static_cast<size_t>(C), 0);
        size_t bytes = 0;
        auto take = [&](size_t b) {
            const unsigned o = align16(bytes);
            bytes = o + b;
            return o;
        };
        take(sizeof(TailHeader<S>));
        h->o_steps = take(static_cast<size_t>(max_steps) * sizeof(TailStepDev));
        // one array range [lo, hi) of an array of len elements of esize
        // bytes, staged 16-byte aligned at smem offset o (Range's split)
        auto stage = [&](int k, const void *src, int64_t lo, int64_t hi, int64_t len, size_t esize, unsigned o) {
            if (hi <= lo) return;
            const int64_t V = 16 / static_cast<int64_t>(esize);
            const int64_t a0 = lo - lo % V, a1 = (hi + V - 1) / V * V;
            int64_t be = a1 <= len ? a1 : hi - hi % V;
            if (be < a0) be = a0;
            TailCopy c{};
            c.src = static_cast<const char *>(src) + a0 * static_cast<int64_t>(esize);
            c.dst = o;
            c.bytes = static_cast<unsigned>((be - a0) * static_cast<int64_t>(esize));
            if (be < hi) {
                c.tail_src = static_cast<const char *>(src) + be * static_cast<int64_t>(esize);
                c.tail_dst = o + static_cast<unsigned>((be - a0) * static_cast<int64_t>(esize));
                c.tail_halves = static_cast<unsigned>((hi - be) * static_cast<int64_t>(esize) / 2);
            }
            tx[static_cast<size_t>(k)] += c.bytes;
            cps[static_cast<size_t>(k)].push_back(c);
        };
        for (size_t d = 0; d < levels.size(); ++d) {
            const auto &L = levels[d];
            auto &D = h->lv[d];
            const bool last = d + 1 == levels.size();
            D.n = static_cast<int>(L.n);
            D.R = static_cast<int>((L.n + C - 1) / C);
            D.nn = last ? 0 : static_cast<int>(levels[d + 1].n);
            D.Rn = last ? 0 : (D.nn + C - 1) / C;
            D.mag = reciprocal(D.R);
            D.cmag = last ? 0u : reciprocal(D.Rn);
            const int64_t R = D.R, Rn = D.Rn;
            size_t ecap = 0, mcap = 0;
            for (int k = 0; k < C; ++k) {
                const int64_t a = std::min<int64_t>(k * R, L.n), b = std::min<int64_t>((k + 1) * R, L.n);
                D.e0[k] = rps[d][a];
                ecap = std::max<size_t>(ecap, static_cast<size_t>(rps[d][b] - rps[d][a]));
                if (!last) {
                    const int64_t ca = std::min<int64_t>(k * Rn, D.nn), cb = std::min<int64_t>((k + 1) * Rn, D.nn);
                    D.m0[k] = offs[d][ca];
                    mcap = std::max<size_t>(mcap, static_cast<size_t>(offs[d][cb] - offs[d][ca]));
                }
            }
            // constant arrays: room for a 16-byte aligned start and end
            const size_t VS = 16 / sizeof(S);
            D.o_rp = take((static_cast<size_t>(R) + 1 + 8) * sizeof(int32_t));
            D.cols16 = L.cd ? 1 : 0;
            D.o_ci = take((ecap + 8) * (L.cd ? sizeof(int16_t) : sizeof(int32_t)));
            D.o_val = take((ecap + 2 * VS) * sizeof(S));
            D.o_dinv = take((static_cast<size_t>(R) + 2 * VS) * sizeof(S));
            D.o_rhs = take(static_cast<size_t>(R) * sizeof(S));
            D.o_x0 = take(static_cast<size_t>(R) * sizeof(S));
            D.o_x1 = take(static_cast<size_t>(R) * sizeof(S));
            D.o_map = take(last ? 0 : (static_cast<size_t>(R) + 8) * sizeof(int32_t));
            D.o_off = take(last ? 0 : (static_cast<size_t>(Rn) + 1 + 8) * sizeof(int32_t));
            D.o_mem = take(last ? 0 : (mcap + 8) * sizeof(int32_t));
            const int64_t nnz = rps[d].back();
            for (int k = 0; k < C; ++k) {
                const int64_t r0 = std::min<int64_t>(k * R, L.n), r1 = std::min<int64_t>((k + 1) * R, L.n);
                if (r1 > r0) {
                    stage(k, L.rp, r0, r1 + 1, L.n + 1, 4, D.o_rp);
                    if (L.cd)
                        stage(k, L.cd, rps[d][r0], rps[d][r1], nnz, 2, D.o_ci);
                    else
                        stage(k, L.ci, rps[d][r0], rps[d][r1], nnz, 4, D.o_ci);
                    stage(k, L.val, rps[d][r0], rps[d][r1], nnz, sizeof(S), D.o_val);
                    stage(k, L.dinv, r0, r1, L.n, sizeof(S), D.o_dinv);
                    if (!last) stage(k, L.map, r0, r1, L.n, 4, D.o_map);
                }
                if (!last) {
                    const int64_t c0 = std::min<int64_t>(k * Rn, D.nn), c1 = std::min<int64_t>((k + 1) * Rn, D.nn);
                    if (c1 > c0) {
                        stage(k, L.off, c0, c1 + 1, D.nn + 1, 4, D.o_off);
                        stage(k, L.mem, offs[d][c0], offs[d][c1], L.n, 4, D.o_mem);
                    }
                }
            }
        }
        {
            // the root's aggregates in the level above
            const int64_t R = h->lv[0].R, n0 = levels[0].n;
            size_t pcap = 0;
            for (int k = 0; k < C; ++k) {
                const int64_t a = std::min<int64_t>(k * R, n0), b = std::min<int64_t>((k + 1) * R, n0);
                h->pm0[k] = poffs[a];
                pcap = std::max<size_t>(pcap, static_cast<size_t>(poffs[b] - poffs[a]));
            }
            h->o_poff = take((static_cast<size_t>(R) + 1 + 8) * sizeof(int32_t));
            h->o_pmem = take((pcap + 8) * sizeof(int32_t));
            for (int k = 0; k < C; ++k) {
                const int64_t r0 = std::min<int64_t>(k * R, n0), r1 = std::min<int64_t>((k + 1) * R, n0);
                if (r1 > r0) {
                    stage(k, parent.off, r0, r1 + 1, n0 + 1, 4, h->o_poff);
                    stage(k, parent.mem, poffs[r0], poffs[r1], parent.n, 4, h->o_pmem);
                }
            }
        }
        bytes = align16(bytes);
        if (bytes > static_cast<size_t>(max_optin) - 1024) continue;
        bool tx_ok = true;
        for (int k = 0; k < C; ++k) tx_ok = tx_ok && tx[static_cast<size_t>(k)] < (1u << 20);
        if (!tx_ok) continue;
        if (C == 1) {
            allow_region_smem<tail_kernel<S, true>>(bytes);
        } else {
            allow_region_smem<tail_kernel<S, false>>(bytes);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(static_cast<unsigned>(C));
            cfg.blockDim = dim3(kTailThreads);
            cfg.dynamicSmemBytes = bytes;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = static_cast<unsigned>(C);
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, tail_kernel<S, false>, &cfg) != cudaSuccess || clusters < 1) {
                cudaGetLastError();
                continue;
            }
        }
        std::vector<TailCopy> flat;
        for (int k = 0; k < C; ++k) {
            h->copy_begin[k] = static_cast<unsigned>(flat.size());
            h->tx_bytes[k] = static_cast<unsigned>(tx[static_cast<size_t>(k)]);
            flat.insert(flat.end(), cps[static_cast<size_t>(k)].begin(), cps[static_cast<size_t>(k)].end());
        }
        h->copy_begin[C] = static_cast<unsigned>(flat.size());
        cluster_ = C;
        smem_ = bytes;
        max_steps_ = max_steps;
        levels_ = levels;
        dev_ = std::make_unique<TailDevice<S>>();
        dev_->header.allocate(1);
        copy_and_wait(ctx, dev_->header.data(), h.get(), sizeof(TailHeader<S>), cudaMemcpyHostToDevice,
                      "region plan upload");
        dev_->copies.allocate(std::max<size_t>(flat.size(), 1));
        if (!flat.empty())
            copy_and_wait(ctx, dev_->copies.data(), flat.data(), flat.size() * sizeof(TailCopy),
                          cudaMemcpyHostToDevice, "region copies upload");
        steps_.clear();
        entries_.clear();
        return true;
    }
    return false;
}

template <class S>
bool TailRegion<S>::add_entry(const std::vector<CoarseStep<S>> &rec, size_t first, size_t count) {
    if (static_cast<int>(count) > max_steps_) return false;
    const int nl = static_cast<int>(levels_.size());
    auto level_of = [&](const S *p) {
        for (int d = 0; d < nl; ++d)
            if (p && (p == levels_[d].x0 || p == levels_[d].x1 || p == levels_[d].rhs)) return d;
        return -1;
    };
    auto sel = [&](const S *p, int d) {
        if (d < 0 || d >= nl || !p) return -1;
        return p == levels_[d].x0 ? 0 : (p == levels_[d].x1 ? 1 : -1);
    };
    std::vector<Step> out;
    for (size_t k = first; k < first + count; ++k) {
        const CoarseStep<S> &s = rec[k];
        Step t{0, -1, -1, -1, -1};
        switch (s.op) {
            case kStepZero:
            case kStepJacobiZero:
                t.op = s.op == kStepZero ? kTZero : kTJacobiZero;
                t.level = level_of(s.xout);
                t.a = sel(s.xout, t.level);
                if (t.a < 0) return false;
                break;
            case kStepSweep:
                t.level = level_of(s.xout);
                t.a = sel(s.xin, t.level);
                t.b = sel(s.xout, t.level);
                if (t.a < 0 || t.b < 0 || t.a == t.b) return false;
                t.op = kTSweep;
                if (s.map) {
                    t.op = kTProlongSweep;
                    t.c = sel(s.e, t.level + 1);
                    if (t.c < 0) return false;
                }
                break;
            case kStepResidualRestrict:
            case kStepRestrict:
                t.op = s.op == kStepResidualRestrict ? kTResidualRestrict : kTRestrict;
                t.level = level_of(s.rhs);
                if (t.level < 0 || t.level + 1 >= nl || s.rhs != levels_[t.level].rhs ||
                    s.coarse_rhs != levels_[t.level + 1].rhs)
                    return false;
                if (t.op == kTResidualRestrict) {
                    t.a = sel(s.xin, t.level);
                    if (t.a < 0) return false;
                }
                if (s.cx) {
                    t.c = sel(s.cx, t.level + 1);
                    if (t.c < 0) return false;
                }
                break;
            case kStepProlong:
                t.op = kTProlong;
                t.level = level_of(s.xout);
                t.a = sel(s.xout, t.level);
                t.c = sel(s.e, t.level + 1);
                if (t.a < 0 || t.c < 0 || s.xin != s.xout) return false;
                break;
            case kStepDense:
                t.op = kTDense;
                t.level = level_of(s.xout);
                t.a = sel(s.xout, t.level);
                if (t.a < 0 || t.level != nl - 1) return false;
                break;
            default:
                return false;
        }
        out.push_back(t);
    }
    entries_.emplace_back(static_cast<int>(steps_.size()), static_cast<int>(out.size()));
    steps_.insert(steps_.end(), out.begin(), out.end());
    return true;
}

template <class S>
void TailRegion<S>::upload(tf_ctx *ctx) {
    std::vector<TailStepDev> d(steps_.size());
    for (size_t k = 0; k < steps_.size(); ++k)
        d[k] = TailStepDev{steps_[k].op, steps_[k].level, steps_[k].a, steps_[k].b, steps_[k].c};
    dev_->steps.allocate(std::max<size_t>(d.size(), 1));
    if (!d.empty())
        copy_and_wait(ctx, dev_->steps.data(), d.data(), d.size() * sizeof(TailStepDev), cudaMemcpyHostToDevice,
                      "region steps upload");
}

template <class S>
void TailRegion<S>::launch(tf_ctx *ctx, int entry, const ProgramIO<S> &io, int root_cur) const {
    const auto [first, count] = entries_.at(static_cast<size_t>(entry));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(cluster_));
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = smem_;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[2];
    int na = 0;
    if (cluster_ > 1) {
        attr[na].id = cudaLaunchAttributeClusterDimension;
        attr[na].val.clusterDim.x = static_cast<unsigned>(cluster_);
        attr[na].val.clusterDim.y = 1;
        attr[na].val.clusterDim.z = 1;
        ++na;
    }
    if (ctx->pdl) {
        attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    cfg.attrs = attr;
    cfg.numAttrs = na;
    if (cluster_ > 1) allow_region_smem<tail_kernel<S, false>>(smem_);
    else allow_region_smem<tail_kernel<S, true>>(smem_);
    auto kernel = cluster_ > 1 ? tail_kernel<S, false> : tail_kernel<S, true>;
    cuda_check(cudaLaunchKernelEx(&cfg, kernel, static_cast<const TailHeader<S> *>(dev_->header.data()),
                                  static_cast<const TailStepDev *>(dev_->steps.data()),
                                  static_cast<const TailCopy *>(dev_->copies.data()), first, count, io, root_cur,
                                  ctx->stable ? 1 : 0, ctx->fault),
               "small-level region launch");
    launched(ctx, "small_levels");
}

template class TailRegion<float>;
template class TailRegion<double>;

}  // namespace tfb
