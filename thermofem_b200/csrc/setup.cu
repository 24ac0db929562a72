// setup.cu -- device stages of the aggregation AMG setup: canonical form,
// strength graph, synchronous handshake matching, graph contraction,
// singleton absorption, member tables and the Galerkin product.
//
// The algorithm is the reference's (src/Multigrid/GpuAggregation.cu, whose
// host statement is test/support/NativeAggregationOracle.cu); the results
// (aggregates, member order, histograms, coarse sparsity) are meant to be
// bit-identical to it, which is why every stage keeps the reference's
// snapshot semantics: proposals of a matching round are all written before
// any are accepted, absorption reads the pre-round map and sizes, member
// slots are re-sorted after the atomic fill.  Sorting, reduction and scans
// are the project's own (sort.cu).
#include "ops.cuh"

namespace tfb {
namespace {

// Stream-ordered temporary allocation (cudaMallocAsync / cudaFreeAsync).
template <class T>
class Temp {
  public:
    Temp(tf_ctx *ctx, size_t n) : ctx_(ctx), n_(n) {
        if (n) cuda_check(cudaMallocAsync(&p_, n * sizeof(T), ctx->stream), "cudaMallocAsync");
    }
    ~Temp() {
        if (p_) cudaFreeAsync(p_, ctx_->stream);
    }
    Temp(const Temp &) = delete;
    Temp &operator=(const Temp &) = delete;
    T *data() const { return static_cast<T *>(p_); }
    size_t size() const { return n_; }

  private:
    tf_ctx *ctx_;
    size_t n_;
    void *p_{nullptr};
};

__device__ __forceinline__ uint64_t sort_key(int r, int c, int bits) {
    return (static_cast<uint64_t>(static_cast<unsigned>(r)) << bits) | static_cast<unsigned>(c);
}

// Symmetric edge priority (GpuAggregation.cu:49-54): splitmix64 finaliser of
// (min(i,j) << 32 | max(i,j)); breaks equal-weight proposals identically on
// both endpoints.
__device__ __forceinline__ uint64_t edge_priority(int i, int j) {
    uint64_t h = (static_cast<uint64_t>(static_cast<unsigned>(min(i, j))) << 32) | static_cast<unsigned>(max(i, j));
    h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ULL;
    h = (h ^ (h >> 27)) * 0x94d049bb133111ebULL;
    return h ^ (h >> 31);
}

// Coordinate keys of every entry, optionally mapped (canonical: map null;
// Galerkin: map = aggregates).  GpuAggregation.cu:136-146.
__global__ void map_entries(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                            const double *__restrict__ a, const int32_t *__restrict__ map, uint64_t *__restrict__ keys,
                            double *__restrict__ vals, int bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = map ? map[i] : i;
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
        const int c = map ? map[ci[j]] : ci[j];
        keys[j] = sort_key(r, c, bits);
        vals[j] = a[j];
    }
}

// Strong edges in both directions (GpuAggregation.cu:339-364); count pass
// when keys is null, fill pass at the scanned offsets otherwise.
__global__ void strength_edges(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                               const double *__restrict__ a, const double *__restrict__ mx, double theta,
                               uint64_t *__restrict__ keys, double *__restrict__ w, int32_t *__restrict__ count,
                               int bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int pos = keys ? count[i] : 0;
    const double m = mx[i];
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
        const int c = ci[j];
        const double weight = (i != c && m > 0 && fabs(a[j]) / m >= theta) ? fabs(a[j]) / m : 0.0;
        if (weight > 0) {
            if (keys) {
                keys[pos] = sort_key(i, c, bits);
                keys[pos + 1] = sort_key(c, i, bits);
                w[pos] = w[pos + 1] = weight;
            }
            pos += 2;
        }
    }
    if (!keys) count[i] = pos;
}

// Each unmatched vertex proposes its best unmatched neighbour from one
// snapshot of mate[] (GpuAggregation.cu:402-431).
__global__ void propose(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                        const double *__restrict__ w, const int32_t *__restrict__ mate, int32_t *__restrict__ proposal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int best = -1;
    double score = 0;
    uint64_t priority = 0;
    if (mate[i] < 0) {
        for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
            const int c = ci[j];
            const double s = w[j];
            if (c == i || mate[c] >= 0 || s <= 0 || s < score) continue;
            const uint64_t cand = edge_priority(i, c);
            if (s > score || (s == score && (best < 0 || cand > priority || (cand == priority && c < best)))) {
                best = c;
                score = s;
                priority = cand;
            }
        }
    }
    proposal[i] = best;
}

// Mutual proposals become pairs (GpuAggregation.cu:440-449).
__global__ void accept(int n, const int32_t *__restrict__ proposal, int32_t *__restrict__ mate) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = proposal[i];
    if (p >= 0 && proposal[p] == i) mate[i] = p;
}

// Root flags with a zero sentinel at n (GpuAggregation.cu:458-463).
__global__ void roots(int n, const int32_t *__restrict__ mate, int32_t *__restrict__ flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) flags[i] = (i < n && (mate[i] < 0 || i < mate[i])) ? 1 : 0;
}

__global__ void assign(int n, const int32_t *__restrict__ mate, const int32_t *__restrict__ prefix,
                       int32_t *__restrict__ map) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) map[i] = prefix[mate[i] < 0 ? i : min(i, mate[i])];
}

__global__ void compose(int n, int32_t *__restrict__ map, const int32_t *__restrict__ second) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) map[i] = second[map[i]];
}

// Cross-aggregate edges of the graph under map (GpuAggregation.cu:534-553).
__global__ void map_graph(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                          const double *__restrict__ w, const int32_t *__restrict__ map, int32_t *__restrict__ offsets,
                          uint64_t *__restrict__ keys, double *__restrict__ vals, int bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int pos = keys ? offsets[i] : 0;
    const int mi = map[i];
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
        const int mc = map[ci[j]];
        if (mi != mc && w[j] > 0) {
            if (keys) {
                keys[pos] = sort_key(mi, mc, bits);
                vals[pos] = w[j];
            }
            ++pos;
        }
    }
    if (!keys) offsets[i] = pos;
}

// Four-slot member table filled by integer atomics (GpuAggregation.cu:586-593);
// the slot order is then fixed by sort_members.
__global__ void slot_members(int n, const int32_t *__restrict__ map, int32_t *__restrict__ sizes,
                             int32_t *__restrict__ slots, int *overflow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = map[i];
    const int slot = atomicAdd(sizes + c, 1);
    if (slot < 4) slots[static_cast<int64_t>(c) * 4 + slot] = i;
    else atomicExch(overflow, 1);
}

__global__ void sort_members(int n, const int32_t *__restrict__ sizes, int32_t *__restrict__ slots) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    int32_t *m = slots + static_cast<int64_t>(c) * 4;
    const int s = min(sizes[c], 4);
    for (int i = 1; i < s; ++i) {
        const int v = m[i];
        int j = i;
        while (j > 0 && m[j - 1] > v) {
            m[j] = m[j - 1];
            --j;
        }
        m[j] = v;
    }
}

// A singleton proposes to the neighbouring aggregate of size 2..3 with the
// largest weight, ties to the smaller aggregate id (GpuAggregation.cu:646-669).
__global__ void propose_absorption(int n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                   const double *__restrict__ w, const int32_t *__restrict__ map,
                                   const int32_t *__restrict__ sizes, int32_t *__restrict__ proposal,
                                   double *__restrict__ scores) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int best = -1;
    double score = 0;
    if (sizes[map[i]] == 1) {
        for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
            const int c = map[ci[j]];
            const double s = w[j];
            if (sizes[c] < 2 || sizes[c] >= 4 || s <= 0) continue;
            if (s > score || (s == score && (best < 0 || c < best))) {
                best = c;
                score = s;
            }
        }
    }
    proposal[i] = best;
    scores[i] = score;
}

// Each target keeps its best distinct proposers, weight descending then
// fine id ascending, up to its remaining capacity (GpuAggregation.cu:685-720).
__global__ void accept_absorption(int coarse, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                  const int32_t *__restrict__ sizes, const int32_t *__restrict__ slots,
                                  const int32_t *__restrict__ proposal, const double *__restrict__ scores,
                                  int32_t *__restrict__ next) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= coarse || sizes[c] < 2 || sizes[c] >= 4) return;
    int sel[2] = {-1, -1};
    double sw[2] = {-1, -1};
    const int cap = 4 - sizes[c];
    for (int k = 0; k < sizes[c]; ++k) {
        const int row = slots[static_cast<int64_t>(c) * 4 + k];
        for (int32_t j = rp[row]; j < rp[row + 1]; ++j) {
            const int i = ci[j];
            if (proposal[i] != c || i == sel[0] || i == sel[1]) continue;
            const double s = scores[i];
            for (int q = 0; q < cap; ++q) {
                if (s > sw[q] || (s == sw[q] && i < sel[q])) {
                    for (int r = cap - 1; r > q; --r) {
                        sel[r] = sel[r - 1];
                        sw[r] = sw[r - 1];
                    }
                    sel[q] = i;
                    sw[q] = s;
                    break;
                }
            }
        }
    }
    for (int q = 0; q < cap; ++q)
        if (sel[q] >= 0) next[sel[q]] = c;
}

__global__ void occupied(int n, const int32_t *__restrict__ sizes, int32_t *__restrict__ flags) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= n) flags[c] = (c < n && sizes[c] > 0) ? 1 : 0;
}

// Member CSR in ascending fine order and the size histogram
// (GpuAggregation.cu:745-757).
__global__ void pack_members(int coarse, const int32_t *__restrict__ sizes, const int32_t *__restrict__ slots,
                             const int32_t *__restrict__ offsets, int32_t *__restrict__ out, int32_t *histogram) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= coarse) return;
    for (int k = 0; k < sizes[c]; ++k) out[offsets[c] + k] = slots[static_cast<int64_t>(c) * 4 + k];
    if (sizes[c]) atomicAdd(histogram + sizes[c] - 1, 1);
}

// sizes[coarse + 1] (zeroed sentinel) and sorted four-slot members.
void build_members(tf_ctx *ctx, int n, int coarse, const int32_t *map, int32_t *sizes, int32_t *slots, int *overflow) {
    memset_async(ctx, sizes, 0, (static_cast<size_t>(coarse) + 1) * sizeof(int32_t));
    slot_members<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, map, sizes, slots, overflow);
    launched(ctx, "slot_members");
    sort_members<<<grid_for(coarse), kBlock, 0, ctx->stream>>>(coarse, sizes, slots);
    launched(ctx, "sort_members");
}

}  // namespace

std::unique_ptr<tf_dcsr> canonicalize(tf_ctx *ctx, const Csr<double, int32_t> &a) {
    const int n = static_cast<int>(a.rows);
    Temp<uint64_t> keys(ctx, static_cast<size_t>(a.nnz));
    Temp<double> vals(ctx, static_cast<size_t>(a.nnz));
    const int bits = column_bits(n);
    map_entries<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, a.rp, a.ci, a.val, nullptr, keys.data(), vals.data(), bits);
    launched(ctx, "map_entries");
    return compress(ctx, n, a.nnz, keys.data(), vals.data(), bits, 0);
}

std::unique_ptr<tf_dcsr> strength_graph(tf_ctx *ctx, const Csr<double, int32_t> &a, const double *row_max,
                                        double theta) {
    require(std::isfinite(theta) && theta >= 0 && theta <= 1, "Invalid strength threshold");
    require(a.nnz <= INT32_MAX / 2, "Native AMG: strength graph exceeds 32-bit capacity", TF_ERR_LENGTH);
    const int n = static_cast<int>(a.rows);
    const int bits = column_bits(n);
    Temp<int32_t> count(ctx, static_cast<size_t>(n) + 1), offsets(ctx, static_cast<size_t>(n) + 1);
    memset_async(ctx, count.data() + n, 0, sizeof(int32_t));
    strength_edges<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, a.rp, a.ci, a.val, row_max, theta, nullptr, nullptr,
                                                            count.data(), bits);
    launched(ctx, "strength_count");
    scan_exclusive(ctx, n + 1, count.data(), offsets.data());
    const int32_t m = read_scalar(ctx, offsets.data() + n);
    Temp<uint64_t> keys(ctx, static_cast<size_t>(m));
    Temp<double> w(ctx, static_cast<size_t>(m));
    if (m) {
        strength_edges<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, a.rp, a.ci, a.val, row_max, theta, keys.data(),
                                                                w.data(), offsets.data(), bits);
        launched(ctx, "strength_fill");
    }
    return compress(ctx, n, m, keys.data(), w.data(), bits, 1);
}

int match_pairs(tf_ctx *ctx, const Csr<double, int32_t> &g, int rounds, int32_t *map) {
    require(rounds >= 1 && rounds <= 8, "Invalid matching configuration");
    const int n = static_cast<int>(g.rows);
    Temp<int32_t> mate(ctx, static_cast<size_t>(n)), proposal(ctx, static_cast<size_t>(n));
    Temp<int32_t> flags(ctx, static_cast<size_t>(n) + 1), prefix(ctx, static_cast<size_t>(n) + 1);
    memset_async(ctx, mate.data(), 0xff, static_cast<size_t>(n) * sizeof(int32_t));
    for (int r = 0; r < rounds; ++r) {
        propose<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, g.rp, g.ci, g.val, mate.data(), proposal.data());
        launched(ctx, "propose");
        accept<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, proposal.data(), mate.data());
        launched(ctx, "accept");
    }
    roots<<<grid_for(n + 1), kBlock, 0, ctx->stream>>>(n, mate.data(), flags.data());
    launched(ctx, "roots");
    scan_exclusive(ctx, n + 1, flags.data(), prefix.data());
    assign<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, mate.data(), prefix.data(), map);
    launched(ctx, "assign");
    return read_scalar(ctx, prefix.data() + n);
}

std::unique_ptr<tf_dcsr> contract_graph(tf_ctx *ctx, const Csr<double, int32_t> &g, const int32_t *map, int count) {
    const int n = static_cast<int>(g.rows);
    const int bits = column_bits(count);
    Temp<int32_t> cnt(ctx, static_cast<size_t>(n) + 1), offsets(ctx, static_cast<size_t>(n) + 1);
    memset_async(ctx, cnt.data() + n, 0, sizeof(int32_t));
    map_graph<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, g.rp, g.ci, g.val, map, cnt.data(), nullptr, nullptr, bits);
    launched(ctx, "map_graph_count");
    scan_exclusive(ctx, n + 1, cnt.data(), offsets.data());
    const int32_t m = read_scalar(ctx, offsets.data() + n);
    Temp<uint64_t> keys(ctx, static_cast<size_t>(m));
    Temp<double> vals(ctx, static_cast<size_t>(m));
    if (m) {
        map_graph<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, g.rp, g.ci, g.val, map, offsets.data(), keys.data(),
                                                           vals.data(), bits);
        launched(ctx, "map_graph_fill");
    }
    return compress(ctx, count, m, keys.data(), vals.data(), bits, 1);
}

std::unique_ptr<tf_transfer> aggregate(tf_ctx *ctx, const Csr<double, int32_t> &g, int rounds, bool absorb) {
    require(rounds >= 1 && rounds <= 8 && g.rows > 0, "Invalid matching configuration");
    const int n = static_cast<int>(g.rows);
    auto t = std::make_unique<tf_transfer>();
    t->fine_rows = n;
    t->map.allocate(static_cast<size_t>(n));
    int32_t *map = t->map.data();
    const int first = match_pairs(ctx, g, rounds, map);
    int coarse = 0;
    {
        auto contracted = contract_graph(ctx, g, map, first);
        Temp<int32_t> second(ctx, static_cast<size_t>(first));
        coarse = match_pairs(ctx, csr_of(*contracted), rounds, second.data());
        compose<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, map, second.data());
        launched(ctx, "compose");
    }
    Temp<int32_t> sizes(ctx, static_cast<size_t>(coarse) + 1), slots(ctx, static_cast<size_t>(coarse) * 4);
    int *overflow = static_cast<int *>(ctx->arena(sizeof(int), 1));
    memset_async(ctx, overflow, 0, sizeof(int));
    build_members(ctx, n, coarse, map, sizes.data(), slots.data(), overflow);
    if (absorb) {
        Temp<int32_t> proposal(ctx, static_cast<size_t>(n)), next(ctx, static_cast<size_t>(n));
        Temp<double> scores(ctx, static_cast<size_t>(n));
        for (int round = 0; round < 2; ++round) {
            propose_absorption<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, g.rp, g.ci, g.val, map, sizes.data(),
                                                                        proposal.data(), scores.data());
            launched(ctx, "propose_absorption");
            copy_async(ctx, next.data(), map, static_cast<size_t>(n) * sizeof(int32_t));
            accept_absorption<<<grid_for(coarse), kBlock, 0, ctx->stream>>>(
                coarse, g.rp, g.ci, sizes.data(), slots.data(), proposal.data(), scores.data(), next.data());
            launched(ctx, "accept_absorption");
            copy_async(ctx, map, next.data(), static_cast<size_t>(n) * sizeof(int32_t));
            build_members(ctx, n, coarse, map, sizes.data(), slots.data(), overflow);
        }
        // Compact the ids of emptied aggregates.
        Temp<int32_t> flags(ctx, static_cast<size_t>(coarse) + 1), prefix(ctx, static_cast<size_t>(coarse) + 1);
        occupied<<<grid_for(coarse + 1), kBlock, 0, ctx->stream>>>(coarse, sizes.data(), flags.data());
        launched(ctx, "occupied");
        scan_exclusive(ctx, coarse + 1, flags.data(), prefix.data());
        compose<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, map, prefix.data());
        launched(ctx, "compose");
        const int compacted = read_scalar(ctx, prefix.data() + coarse);
        // The compacted table fits in the old allocation (compacted <= coarse).
        coarse = compacted;
        build_members(ctx, n, coarse, map, sizes.data(), slots.data(), overflow);
    }
    if (read_scalar(ctx, overflow)) fail(TF_ERR_RUNTIME, "Aggregate capacity exceeded");
    t->coarse_rows = coarse;
    t->members.allocate(static_cast<size_t>(n));
    t->offsets.allocate(static_cast<size_t>(coarse) + 1);
    scan_exclusive(ctx, coarse + 1, sizes.data(), t->offsets.data());
    int32_t *hist = static_cast<int32_t *>(ctx->arena(4 * sizeof(int32_t), 1));
    memset_async(ctx, hist, 0, 4 * sizeof(int32_t));
    pack_members<<<grid_for(coarse), kBlock, 0, ctx->stream>>>(coarse, sizes.data(), slots.data(), t->offsets.data(),
                                                               t->members.data(), hist);
    launched(ctx, "pack_members");
    cuda_check(cudaMemcpyAsync(t->histogram, hist, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream),
               "histogram readback");
    cuda_check(cudaStreamSynchronize(ctx->stream), "aggregate");
    return t;
}

std::unique_ptr<tf_dcsr> galerkin(tf_ctx *ctx, const Csr<double, int32_t> &a, const int32_t *map, int coarse) {
    const int n = static_cast<int>(a.rows);
    require(coarse >= 1, "AMG transfer dimension mismatch");
    const int bits = column_bits(coarse);
    Temp<uint64_t> keys(ctx, static_cast<size_t>(a.nnz));
    Temp<double> vals(ctx, static_cast<size_t>(a.nnz));
    map_entries<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, a.rp, a.ci, a.val, map, keys.data(), vals.data(), bits);
    launched(ctx, "map_entries");
    return compress(ctx, coarse, a.nnz, keys.data(), vals.data(), bits, 0);
}

}  // namespace tfb
