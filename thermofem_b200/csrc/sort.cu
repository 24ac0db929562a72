// sort.cu -- the project's own scan, stable LSD radix sort of (u64, f64)
// pairs, left-to-right reduce-by-key and coordinate compression.  They
// replace the CUB DeviceScan / DeviceRadixSort / DeviceReduce::ReduceByKey
// calls of the reference setup (src/Multigrid/GpuAggregation.cu:116-234).
//
// Determinism: the sort is stable and every run of equal keys is reduced by
// one thread from left to right, so Galerkin and canonical sums come out in
// the order the reference's host oracle uses (stable sort, then sequential
// sum), independent of the GPU.
#include "ops.cuh"

namespace tfb {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kDigits = 256;

// Stream-ordered temporary allocation (cudaMallocAsync / cudaFreeAsync).
template <class T>
class TempBuffer {
  public:
    TempBuffer(tf_ctx *ctx, size_t n) : ctx_(ctx) {
        if (n) cuda_check(cudaMallocAsync(&p_, n * sizeof(T), ctx->stream), "cudaMallocAsync");
    }
    ~TempBuffer() {
        if (p_) cudaFreeAsync(p_, ctx_->stream);
    }
    TempBuffer(const TempBuffer &) = delete;
    TempBuffer &operator=(const TempBuffer &) = delete;
    T *data() const { return static_cast<T *>(p_); }

  private:
    tf_ctx *ctx_;
    void *p_{nullptr};
};

// Block-wide exclusive scan of kScanItems consecutive items per thread.
// Returns the block total; out[k] = exclusive prefix of item k of this thread.
__device__ __forceinline__ int block_scan(int (&v)[kScanItems], int *warp_tot) {
    int local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int t = v[k];
        v[k] = local;
        local += t;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    int warp_prefix = 0, total = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) {
        if (w < warp) warp_prefix += warp_tot[w];
        total += warp_tot[w];
    }
    const int prefix = warp_prefix + inc - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] += prefix;
    return total;
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(int64_t n, const int32_t *__restrict__ in,
                                                                int32_t *__restrict__ sums) {
    __shared__ int warp_tot[kScanThreads / 32];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) t += warp_tot[w];
        sums[blockIdx.x] = t;
    }
}

// Scans each tile and adds the tile's offset (offsets == nullptr: single tile).
__global__ void __launch_bounds__(kScanThreads) scan_tiles(int64_t n, const int32_t *in, int32_t *out,
                                                            const int32_t *__restrict__ offsets) {
    __shared__ int warp_tot[kScanThreads / 32];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanItems;
    int v[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0;
    block_scan(v, warp_tot);
    const int add = offsets ? offsets[blockIdx.x] : 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) out[base + k] = v[k] + add;
}

__global__ void __launch_bounds__(kSortThreads) radix_hist(int64_t n, int shift, const uint64_t *__restrict__ keys,
                                                           int32_t *__restrict__ counts, int tiles) {
    __shared__ int hist[kDigits];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile;
#pragma unroll 4
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t i = base + r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    counts[static_cast<int64_t>(threadIdx.x) * tiles + blockIdx.x] = hist[threadIdx.x];
}

// Stable scatter: items of a tile are ranked round by round (256 items per
// round, in index order); within a round, per-warp match masks give the rank
// among equal digits and per-warp digit counts order the warps.
__global__ void __launch_bounds__(kSortThreads) radix_scatter(int64_t n, int shift, const uint64_t *__restrict__ kin,
                                                              const double *__restrict__ vin,
                                                              uint64_t *__restrict__ kout,
                                                              double *__restrict__ vout,
                                                              const int32_t *__restrict__ offsets, int tiles) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ int base[kDigits];
    __shared__ int wcount[kWarps][kDigits];
    base[threadIdx.x] = offsets[static_cast<int64_t>(threadIdx.x) * tiles + blockIdx.x];
#pragma unroll
    for (int w = 0; w < kWarps; ++w) wcount[w][threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t tile0 = static_cast<int64_t>(blockIdx.x) * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t i = tile0 + r * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const uint64_t key = valid ? kin[i] : 0;
        const double val = valid ? vin[i] : 0.0;
        const int d = valid ? static_cast<int>((key >> shift) & 255u) : kDigits;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        if (valid && lane == __ffs(peers) - 1) wcount[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int pos = base[d] + rank;
            for (int w = 0; w < warp; ++w) pos += wcount[w][d];
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        int s = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            s += wcount[w][threadIdx.x];
            wcount[w][threadIdx.x] = 0;
        }
        base[threadIdx.x] += s;
        __syncthreads();
    }
}

__global__ void run_heads(int64_t n, const uint64_t *__restrict__ keys, int32_t *__restrict__ flags) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
    else if (i == n) flags[n] = 0;
}

__global__ void run_reduce(int64_t n, const uint64_t *__restrict__ keys, const double *__restrict__ vals, int op,
                           const int32_t *__restrict__ flags, const int32_t *__restrict__ seg,
                           uint64_t *__restrict__ kout, double *__restrict__ vout) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n || !flags[i]) return;
    const uint64_t k = keys[i];
    double s = vals[i];
    for (int64_t j = i + 1; j < n && keys[j] == k; ++j) s = op ? (s > vals[j] ? s : vals[j]) : s + vals[j];
    kout[seg[i]] = k;
    vout[seg[i]] = s;
}

__global__ void unpack_kernel(int64_t u, const uint64_t *__restrict__ keys, const double *__restrict__ vals,
                              int col_bits, int32_t *__restrict__ counts, int32_t *__restrict__ cols,
                              double *__restrict__ out) {
    const int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (j >= u) return;
    const uint64_t k = keys[j];
    atomicAdd(counts + static_cast<int64_t>(k >> col_bits), 1);
    cols[j] = static_cast<int32_t>(k & ((uint64_t(1) << col_bits) - 1));
    out[j] = vals[j];
}

}  // namespace

void scan_exclusive(tf_ctx *ctx, int64_t n, const int32_t *in, int32_t *out) {
    if (n <= 0) return;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        scan_tiles<<<1, kScanThreads, 0, ctx->stream>>>(n, in, out, nullptr);
        launched(ctx, "scan");
        return;
    }
    TempBuffer<int32_t> sums(ctx, static_cast<size_t>(tiles));
    scan_tile_sums<<<static_cast<unsigned>(tiles), kScanThreads, 0, ctx->stream>>>(n, in, sums.data());
    launched(ctx, "scan_sums");
    scan_exclusive(ctx, tiles, sums.data(), sums.data());
    scan_tiles<<<static_cast<unsigned>(tiles), kScanThreads, 0, ctx->stream>>>(n, in, out, sums.data());
    launched(ctx, "scan_tiles");
}

void radix_sort_pairs(tf_ctx *ctx, int64_t n, const uint64_t *kin, const double *vin, uint64_t *kout, double *vout,
                      int end_bit) {
    require(end_bit >= 1 && end_bit <= 64, "radix sort end bit must be 1..64");
    require(n < INT32_MAX, "radix sort supports fewer than 2^31 items", TF_ERR_LENGTH);
    if (n <= 0) return;
    const int passes = (end_bit + 7) / 8;
    const int tiles = static_cast<int>((n + kSortTile - 1) / kSortTile);
    TempBuffer<uint64_t> tk(ctx, passes > 1 ? static_cast<size_t>(n) : 0);
    TempBuffer<double> tv(ctx, passes > 1 ? static_cast<size_t>(n) : 0);
    TempBuffer<int32_t> counts(ctx, static_cast<size_t>(kDigits) * tiles);
    const uint64_t *sk = kin;
    const double *sv = vin;
    for (int p = 0; p < passes; ++p) {
        // The last pass lands in the output buffers.
        const bool to_out = ((passes - 1 - p) % 2) == 0;
        uint64_t *dk = to_out ? kout : tk.data();
        double *dv = to_out ? vout : tv.data();
        radix_hist<<<tiles, kSortThreads, 0, ctx->stream>>>(n, 8 * p, sk, counts.data(), tiles);
        launched(ctx, "radix_hist");
        scan_exclusive(ctx, static_cast<int64_t>(kDigits) * tiles, counts.data(), counts.data());
        radix_scatter<<<tiles, kSortThreads, 0, ctx->stream>>>(n, 8 * p, sk, sv, dk, dv, counts.data(), tiles);
        launched(ctx, "radix_scatter");
        sk = dk;
        sv = dv;
    }
}

int64_t reduce_by_key(tf_ctx *ctx, int64_t n, const uint64_t *keys, const double *vals, int op, uint64_t *kout,
                      double *vout) {
    if (n <= 0) return 0;
    TempBuffer<int32_t> flags(ctx, static_cast<size_t>(n) + 1), seg(ctx, static_cast<size_t>(n) + 1);
    run_heads<<<grid_for(n + 1), kBlock, 0, ctx->stream>>>(n, keys, flags.data());
    launched(ctx, "run_heads");
    scan_exclusive(ctx, n + 1, flags.data(), seg.data());
    run_reduce<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, keys, vals, op, flags.data(), seg.data(), kout, vout);
    launched(ctx, "run_reduce");
    return read_scalar(ctx, seg.data() + n);
}

int column_bits(int rows) {
    int bits = 1;
    for (unsigned r = static_cast<unsigned>(rows - 1); r >>= 1;) ++bits;
    return bits;
}

std::unique_ptr<tf_dcsr> compress(tf_ctx *ctx, int rows, int64_t n, const uint64_t *keys, const double *vals, int col_bits, int op) {
    auto out = std::make_unique<tf_dcsr>();
    out->rows = out->cols = rows;
    out->offsets.allocate(static_cast<size_t>(rows + 1) * sizeof(int32_t));
    int32_t *rp = reinterpret_cast<int32_t *>(out->offsets.data());
    if (n == 0) {
        memset_async(ctx, rp, 0, static_cast<size_t>(rows + 1) * sizeof(int32_t));
        return out;
    }
    TempBuffer<uint64_t> sk(ctx, static_cast<size_t>(n)), uk(ctx, static_cast<size_t>(n));
    TempBuffer<double> sv(ctx, static_cast<size_t>(n)), uv(ctx, static_cast<size_t>(n));
    radix_sort_pairs(ctx, n, keys, vals, sk.data(), sv.data(), col_bits + column_bits(rows));
    const int64_t u = reduce_by_key(ctx, n, sk.data(), sv.data(), op, uk.data(), uv.data());
    out->nnz = u;
    out->indices.allocate(static_cast<size_t>(u) * sizeof(int32_t));
    out->values.allocate(static_cast<size_t>(u) * sizeof(double));
    memset_async(ctx, rp, 0, static_cast<size_t>(rows + 1) * sizeof(int32_t));
    unpack_kernel<<<grid_for(u), kBlock, 0, ctx->stream>>>(u, uk.data(), uv.data(), col_bits, rp,
                                                           reinterpret_cast<int32_t *>(out->indices.data()),
                                                           reinterpret_cast<double *>(out->values.data()));
    launched(ctx, "unpack");
    scan_exclusive(ctx, rows + 1, rp, rp);
    return out;
}

}  // namespace tfb
