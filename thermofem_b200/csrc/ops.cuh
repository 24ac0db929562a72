// ops.cuh -- typed internal entry points of the kernels (the C ABI and the
// C++ components both call these).
#pragma once
#include "common.cuh"

#include <memory>

namespace tfb {

// Device CSR view with typed arrays.  T is the type of the vectors an SpMV
// over it reads and writes, and of its accumulators; V the type its values
// are stored in (V = T, or FP32 values under FP64 vectors: each value is
// widened before its product, so a row sums exactly as with FP64 values
// equal to the FP32 ones).
template <class T, class I, class V = T>
struct Csr {
    int64_t rows{0}, cols{0}, nnz{0};
    const I *rp{nullptr};
    const I *ci{nullptr};
    const V *val{nullptr};
    // Optional second copy of the columns as offsets from the row
    // (ci[j] - row, int16): the pipelined row-tile kernels stream it instead
    // of ci when set (see delta_columns).
    const int16_t *cd{nullptr};
    // Optional sliced copy (SlicedCopy below): slices of 32 consecutive
    // rows, entry j of row 32 s + l at sp[s] + 32 j + l (values sv, column
    // offsets from the row sc, padding kSlicePad with value 0).  The SpMV
    // family may stream it instead of the CSR arrays; results are the same
    // bits either way.
    const int32_t *sp{nullptr};
    const V *sv{nullptr};
    const int16_t *sc{nullptr};
    // Banded slices instead of per-entry offsets (SlicedCopy::band): entry
    // slot j of slice s holds one column offset shared by the slice's 32
    // rows and the mask of its padding lanes, bd[sp[s] / 32 + j] = {offset,
    // mask}; sc is then null.  Stencil operators have a handful of slots per
    // slice, so the copy streams values and almost nothing else.
    const int2 *bd{nullptr};
    // With sorted slices: the row at position t of the sliced order (rows
    // permuted within their 256-row tile, longest first).  Only epilogues
    // without partial sums stream a sorted copy.
    const int32_t *perm{nullptr};
    // Most entries of any 256-row tile (8 slices) of the sliced copy.
    int64_t sl_tile_max{0};
};

// Column offset of a padding entry of the sliced layout.
constexpr int16_t kSlicePad = -32768;

// Owner of an operator's sliced copy.
template <class T>
struct SlicedCopy {
    DeviceBuffer<int32_t> sp;
    DeviceBuffer<T> val;
    DeviceBuffer<int16_t> col;   // per-entry column offsets (sliced), or
    DeviceBuffer<int2> band;     // per-slot shared offsets and padding masks (banded)
    DeviceBuffer<int32_t> perm;  // sorted slices only
    int64_t entries{0};
    int64_t tile_max{0};  // most entries of any 256-row tile
    void release() {
        sp.release();
        val.release();
        col.release();
        band.release();
        perm.release();
        entries = 0;
        tile_max = 0;
    }
    bool banded() const { return band.data() != nullptr; }
    template <class U, class I>
    void attach(Csr<U, I, T> &c) const {
        if (sp.data()) {
            c.sp = sp.data();
            c.sv = val.data();
            c.sc = col.data();
            c.bd = band.data();
            c.perm = perm.data();
            c.sl_tile_max = tile_max;
        }
    }
};

// Launch shape of the row-tile SpMV family: rows_per_tile consecutive rows
// per CTA; their nonzeros are staged through shared memory in chunks of
// chunk entries.
struct SpmvShape {
    int rows_per_thread{2};  // 1 or 2 (rows per tile = 256 * rows_per_thread)
    int chunk{4096};         // staged entries per chunk
};
SpmvShape spmv_shape(int64_t rows, int64_t nnz, size_t value_size, size_t index_size);

// y = A x
template <class T, class I, class V = T>
void spmv(tf_ctx *ctx, const Csr<T, I, V> &a, const T *x, T *y);
// Picks and caches the fastest pipelined launch shape for operators of this
// shape (y is overwritten).  Writes the chosen ring depth, CTAs per SM, chunk
// capacity percentage, rows per thread and the best time per launch (ms)
// when non-null.
template <class T, class I>
void autotune_spmv(tf_ctx *ctx, const Csr<T, I> &a, const T *x, T *y, int *stages, int *ctas_per_sm, int *cap_pct,
                   int *rows_per_thread, float *ms);
// autotune_spmv the first time an operator of a's shape and storage is set
// up in the process; later setups reuse the cached shape
// (THERMOFEM_B200_SLICED_SHAPE forces the timing, and with it that shape).
template <class T, class I, class V = T>
void tune_spmv(tf_ctx *ctx, const Csr<T, I, V> &a, const T *x, T *y);
// The storage the SpMV family streams for a under its cached shape: true
// (sliced copy, *entries its padded entry count) or false (CSR, *entries = nnz).
template <class T, class I, class V = T>
bool streams_sliced(tf_ctx *ctx, const Csr<T, I, V> &a, int64_t entries_if_sliced, int64_t *entries);
// Stores a launch shape for operators of a's shape (validated, not timed).
template <class T, class I>
void set_spmv_config(tf_ctx *ctx, const Csr<T, I> &a, int stages, int ctas_per_sm, int cap_pct, int rows_per_thread);
// r = b - A x
template <class T, class I, class V = T>
void residual(tf_ctx *ctx, const Csr<T, I, V> &a, const T *b, const T *x, T *r);
// xo = x~ + w Dinv (b - A x~), x~ = x (+ e[map] when map != nullptr)
template <class T, class I, class V = T>
void jacobi_sweep(tf_ctx *ctx, const Csr<T, I, V> &a, const T *dinv, const T *b, const T *x, T *xo, T w,
                  const float *row_w, const int32_t *map, const T *e);
// xo = x + w Dinv (b - A x), and fine[mem[k]] += xo[c] for k in
// [off[c], off[c+1]) (the prolongation of the result fused in).
template <class T, class I, class V = T>
void jacobi_sweep_scatter(tf_ctx *ctx, const Csr<T, I, V> &a, const T *dinv, const T *b, const T *x, T *xo, T w,
                          const int32_t *off, const int32_t *mem, T *fine);
// b[c] = sum_k fine[mem[k]] (k in [off[c], off[c+1])), x = w Dinv b.
template <class T>
void restrict_jacobi_zero(tf_ctx *ctx, int64_t nc, const int32_t *off, const int32_t *mem, const T *fine, T *b,
                          const T *dinv, T *x, T w);
// x = w Dinv b
template <class T>
void jacobi_zero(tf_ctx *ctx, int64_t n, const T *dinv, const T *b, T *x, T w, const float *row_w);
template <class T>
void jacobi_update(tf_ctx *ctx, int64_t n, T w, const T *dinv, const T *b, const T *ax, T *x);
// True when some of the n indices lies outside [0, limit) (synchronises).
bool indices_out_of_range(tf_ctx *ctx, int64_t n, const int32_t *idx, int32_t limit);
// b = S(in), x = w Dinv b (a cycle's input conversion fused with its first sweep)
template <class S, class T>
void jacobi_zero_convert(tf_ctx *ctx, int64_t n, const S *dinv, const T *in, S *b, S *x, S w);
// Dinv from summed diagonal entries; throws TF_ERR_INVALID on a bad diagonal.
template <class T, class I, class V = T>
void inverse_diagonal(tf_ctx *ctx, const Csr<T, I, V> &a, T *dinv);
// cd[j] = ci[j] - row(j) as int16_t (the pipelined kernels' 2-byte column
// stream).  False, with cd unusable, when a coupling lies more than 32767
// rows from the diagonal.  THERMOFEM_B200_DELTA16=0 turns the stream off
// (delta_columns_enabled() false).
template <class I>
bool delta_columns(tf_ctx *ctx, int64_t rows, const I *rp, const I *ci, int16_t *cd);
bool delta_columns_enabled();
// Builds the sliced copy of a (which must carry its 2-byte column offsets
// cd): slice width = its longest row.  When the rows in their own order
// would pad by more than THERMOFEM_B200_SLICED_PAD percent of nnz (default
// 50 for FP64 values, 25 for FP32), allow_sort is set and
// THERMOFEM_B200_SLICED=sorted, the rows of every 256-row tile are ordered
// longest first (ties by row) and the copy carries that permutation (off by
// default: on the aggregated levels the permuted row loads and stores cost
// more in a cycle than the even slices save).  False, with out released,
// when the padding still exceeds that bound or the entries do not fit
// int32.  THERMOFEM_B200_SLICED=0 turns the copy off (sliced_enabled() false).
template <class T>
bool build_sliced(tf_ctx *ctx, const Csr<T, int32_t> &a, SlicedCopy<T> &out, bool allow_sort);
bool sliced_enabled();
// A banded copy of a (slices of 32 rows whose entries share their column
// offsets slot by slot, SlicedCopy::band) when every row is sorted without
// repeated columns, no slice needs more than 32 slots and the padding stays
// within THERMOFEM_B200_BANDED_PAD percent of nnz (default 10); false (and
// out released) otherwise.  THERMOFEM_B200_BANDED=0 turns it off.
template <class T>
bool build_banded(tf_ctx *ctx, const Csr<T, int32_t> &a, SlicedCopy<T> &out);
bool banded_enabled();
// Self-check of the bounded device waits: a kernel whose wait nothing ends
// gives up after `polls` polls and raises the context's fault word; throws
// TF_ERR_TIMEOUT from check_faults (the word is cleared).
void bounded_wait_check(tf_ctx *ctx, int64_t polls);
template <class T>
void restrict_sum(tf_ctx *ctx, int64_t nc, const int32_t *off, const int32_t *mem, const T *fine, T *coarse);
template <class T>
void prolong_add(tf_ctx *ctx, int64_t nf, const int32_t *map, const T *coarse, T *fine);
// out[k] = x_k . y_k (k < count <= 4), deterministic two-stage FP64 reduction.
template <class T>
void dot_multi(tf_ctx *ctx, int64_t n, int count, const T *const *xs, const T *const *ys, double *out);
template <class T>
void axpby(tf_ctx *ctx, int64_t n, double a, const T *x, double b, T *y);
// The Krylov solvers' fused vector steps (rr, ss: device doubles, FP64
// squared norms over the fixed dot_multi partition).
template <class T>
void krylov_cg_update(tf_ctx *ctx, int64_t n, double alpha, const T *p, const T *ap, T *x, T *r, double *rr);
template <class T>
void krylov_cg_direction(tf_ctx *ctx, int64_t n, double beta, int restart, const T *z, T *p);
template <class T>
void krylov_bicgstab_direction(tf_ctx *ctx, int64_t n, double beta, double omega, int restart, const T *r,
                               const T *v, T *p);
template <class T>
void krylov_bicgstab_s(tf_ctx *ctx, int64_t n, double alpha, const T *r, const T *v, const T *phat, T *x, T *s,
                       double *ss);
template <class T>
void krylov_bicgstab_update(tf_ctx *ctx, int64_t n, double omega, const T *shat, const T *s, const T *t, T *x, T *r,
                            double *rr);
template <class S, class D>
void convert(tf_ctx *ctx, int64_t n, const S *src, D *dst);
template <class T>
void fill_zero(tf_ctx *ctx, int64_t n, T *x);

// Structural validation (offsets monotone/bounded, indices in range).
template <class I>
bool csr_structure_ok(tf_ctx *ctx, int64_t rows, int64_t cols, int64_t nnz, const I *rp, const I *ci);
// bit 1 unsorted/duplicate, bit 2 invalid/nonfinite.
template <class T, class I>
int csr_canonical_flags(tf_ctx *ctx, const Csr<T, I> &a);
// Finite values, nonfinite entry or bad diagonal -> false; row max |offdiag|.
bool row_stats(tf_ctx *ctx, const Csr<double, int32_t> &a, double *row_max);

// Sorting primitives (sort.cu).
void radix_sort_pairs(tf_ctx *ctx, int64_t n, const uint64_t *kin, const double *vin, uint64_t *kout,
                      double *vout, int end_bit);
int64_t reduce_by_key(tf_ctx *ctx, int64_t n, const uint64_t *keys, const double *vals, int op, uint64_t *kout,
                      double *vout);
void scan_exclusive(tf_ctx *ctx, int64_t n, const int32_t *in, int32_t *out);

// Coordinate compression (sort + reduce + unpack) into an owned CSR.
std::unique_ptr<tf_dcsr> compress(tf_ctx *ctx, int rows, int64_t n, const uint64_t *keys, const double *vals, int col_bits, int op);
int column_bits(int rows);

// Setup stages (setup.cu), on canonical FP64/int32 operands.
std::unique_ptr<tf_dcsr> canonicalize(tf_ctx *ctx, const Csr<double, int32_t> &a);
std::unique_ptr<tf_dcsr> strength_graph(tf_ctx *ctx, const Csr<double, int32_t> &a, const double *row_max, double theta);
int match_pairs(tf_ctx *ctx, const Csr<double, int32_t> &g, int rounds, int32_t *map);
std::unique_ptr<tf_dcsr> contract_graph(tf_ctx *ctx, const Csr<double, int32_t> &g, const int32_t *map, int count);
std::unique_ptr<tf_transfer> aggregate(tf_ctx *ctx, const Csr<double, int32_t> &g, int rounds, bool absorb);
std::unique_ptr<tf_dcsr> galerkin(tf_ctx *ctx, const Csr<double, int32_t> &a, const int32_t *map, int coarse);

// Coarse LU (coarse.cu).
bool coarse_lu_factor(tf_ctx *ctx, const Csr<double, int32_t> &a, double *lu, int32_t *pivots);
template <class T>
void coarse_lu_solve(tf_ctx *ctx, int n, const double *lu, const int32_t *pivots, const T *b, T *x);
// Explicit inverse (row major) from the factor, for the per-cycle dense apply.
void coarse_inverse(tf_ctx *ctx, int n, const double *lu, const int32_t *pivots, double *inv);
template <class T>
void coarse_dense_apply(tf_ctx *ctx, int n, const double *inv, const T *b, T *x);
// coarse_dense_apply with the transfers around it fused in: when rfine is
// set, b is first restricted from it (b[c] = sum of rfine over roff/rmem
// members, stored); when fine is set, x is then prolonged into it
// (fine[smem[k]] += x[c] over soff/smem members).
template <class T>
void coarse_dense_apply_fused(tf_ctx *ctx, int n, const double *inv, T *b, T *x, const T *rfine, const int32_t *roff,
                              const int32_t *rmem, const int32_t *soff, const int32_t *smem, T *fine);

inline Csr<double, int32_t> csr_of(const tf_dcsr &m) {
    Csr<double, int32_t> c;
    c.rows = m.rows;
    c.cols = m.cols;
    c.nnz = m.nnz;
    c.rp = reinterpret_cast<const int32_t *>(m.offsets.data());
    c.ci = reinterpret_cast<const int32_t *>(m.indices.data());
    c.val = reinterpret_cast<const double *>(m.values.data());
    return c;
}

template <class T, class I>
Csr<T, I> csr_of(const tf_csr &m) {
    Csr<T, I> c;
    c.rows = m.rows;
    c.cols = m.cols;
    c.nnz = m.nnz;
    c.rp = static_cast<const I *>(m.offsets);
    c.ci = static_cast<const I *>(m.indices);
    c.val = static_cast<const T *>(m.values);
    return c;
}

}  // namespace tfb
