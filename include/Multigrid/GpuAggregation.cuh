// GpuAggregation.cuh -- the aggregation AMG setup stages and transfer
// operations (drop-in for include/Multigrid/GpuAggregation.cuh:13-101 of
// Mgepahmge/ThermoFEM: AggregateTransfer and CoarseFactor with the same
// fields, GpuAggregation's five stages, the free transfer, coarse-factor and
// conversion functions, the same checks and messages).
//
// Every stage runs on the library's kernels (tf_canonicalize, tf_row_stats,
// tf_strength, tf_aggregate, tf_galerkin_map, tf_restrict, tf_prolong,
// tf_coarse_lu_factor / _solve, tf_convert) and gives the reference's results
// bit for bit: aggregates, member tables, histograms and coarse patterns,
// and coarse values too (every merged entry is summed in the stable order).
// A GpuAggregation works on the device that was current when it was made;
// its results live there.  The dense coarse LU takes up to 256 rows (the
// reference: 64).
#pragma once

#include <LinearAlgebra/Operations.cuh>

#include <array>
#include <climits>
#include <cmath>
#include <memory>

namespace thermofem::multigrid {

struct AggregateTransfer {
    CudaBuffer<int> aggregate_, offsets_, members_;  ///< fine -> aggregate map, member offsets, members (ascending)
    int fineRows_{}, coarseRows_{};
    std::array<int, 4> histogram_{};                 ///< aggregates of 1, 2, 3 and 4 members
};

struct CoarseFactor {
    CudaBuffer<double> lu_;   ///< rows x rows, row-major, unit lower part below the diagonal
    CudaBuffer<int> pivots_;  ///< the row swapped in at each step
    bool factored_{false}, singular_{false};
    int rows_{};
};

namespace detail {

/// Takes a library-owned device CSR (f64 values, int32 indices) into a
/// CsrMatrix<double> of its own buffers.
inline CsrMatrix<double> adopt(tf_dcsr *owned, b200::Context &ctx) {
    struct Free {
        void operator()(tf_dcsr *m) const noexcept { tf_dcsr_free(m); }
    };
    std::unique_ptr<tf_dcsr, Free> hold(owned);
    tf_csr v{};
    b200::check(tf_dcsr_view(owned, &v));
    CudaBuffer<int> rp(static_cast<std::size_t>(v.rows) + 1), ci(static_cast<std::size_t>(v.nnz));
    CudaBuffer<double> val(static_cast<std::size_t>(v.nnz));
    auto copy = [&](void *dst, const void *src, std::size_t bytes) {
        if (bytes)
            thermofem::detail::cudaCall(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx.stream()),
                                        "cudaMemcpyAsync");
    };
    copy(rp.data(), v.offsets, rp.sizeBytes());
    copy(ci.data(), v.indices, ci.sizeBytes());
    copy(val.data(), v.values, val.sizeBytes());
    ctx.synchronize();
    CsrMatrix<double> m;
    // the library's stages produce valid CSR: take the buffers without a second check
    m = CsrMatrix<double>::fromBuffers(static_cast<std::size_t>(v.rows), static_cast<std::size_t>(v.cols),
                                       std::move(rp), std::move(ci), std::move(val));
    return m;
}

template <class T>
const T *onDevice(const CudaBuffer<T> &b) {
    return b.empty() ? nullptr : b.deviceData();
}

}  // namespace detail

class GpuAggregation {
  public:
    /// compactKeys: the reference's workspace option; it never changes results
    /// and this implementation always uses compact sort keys.
    explicit GpuAggregation(bool compactKeys = false)
        : compact_(compactKeys), ctx_(std::make_unique<b200::Context>(b200::currentDevice())) {}
    ~GpuAggregation() = default;
    GpuAggregation(const GpuAggregation &) = delete;
    GpuAggregation &operator=(const GpuAggregation &) = delete;

    /// Sorted, duplicate-summed copy (explicit zeros kept).
    CsrMatrix<double> canonical(const CsrMatrix<double> &a) {
        if (!a.rowCount() || a.rowCount() >= std::size_t(INT_MAX) || a.rowCount() != a.columnCount() ||
            a.nonZeroCount() > std::size_t(INT_MAX / 2) || a.rowOffsets().deviceId() != device())
            throw std::invalid_argument("AMG requires nonempty square int32-capacity CSR on workspace device");
        return b200::onContext(*ctx_, [&] {
            const tf_csr v = b200::describe(a);
            tf_dcsr *out = nullptr;
            b200::check(tf_canonicalize(ctx_->get(), &v, &out));
            return detail::adopt(out, *ctx_);
        });
    }

    /// Finite values, a nonzero diagonal with a finite reciprocal on every row.
    void validate(const CsrMatrix<double> &a) {
        b200::onContext(*ctx_, [&] { rowMaxima(a); });
    }

    /// Symmetric strength graph of a (max-merged couplings above threshold).
    CsrMatrix<double> strength(const CsrMatrix<double> &a, double threshold) {
        if (!std::isfinite(threshold) || threshold < 0 || threshold > 1)
            throw std::invalid_argument("Invalid strength threshold");
        return b200::onContext(*ctx_, [&] {
            CudaBuffer<double> rowMax = rowMaxima(a);
            const tf_csr v = b200::describe(a);
            tf_dcsr *out = nullptr;
            b200::check(tf_strength(ctx_->get(), &v, detail::onDevice(rowMax), threshold, &out));
            return detail::adopt(out, *ctx_);
        });
    }

    /// Two-stage pairwise matching of the graph (rounds 1..8 each), optional
    /// singleton absorption, aggregates of at most four rows.
    AggregateTransfer aggregate(const CsrMatrix<double> &graph, int rounds, bool absorbSingletons) {
        if (rounds < 1 || rounds > 8 || !graph.rowCount()) throw std::invalid_argument("Invalid matching configuration");
        return b200::onContext(*ctx_, [&] {
            struct Free {
                void operator()(tf_transfer *t) const noexcept { tf_transfer_free(t); }
            };
            const tf_csr v = b200::describe(graph);
            tf_transfer *raw = nullptr;
            b200::check(tf_aggregate(ctx_->get(), &v, rounds, absorbSingletons ? 1 : 0, &raw));
            std::unique_ptr<tf_transfer, Free> t(raw);
            AggregateTransfer out;
            int32_t histogram[4] = {};
            b200::check(tf_transfer_info(raw, &out.fineRows_, &out.coarseRows_, histogram));
            for (int k = 0; k < 4; ++k) out.histogram_[static_cast<std::size_t>(k)] = histogram[k];
            const int32_t *map = nullptr, *off = nullptr, *mem = nullptr;
            b200::check(tf_transfer_arrays(raw, &map, &off, &mem));
            out.aggregate_ = CudaBuffer<int>(static_cast<std::size_t>(out.fineRows_));
            out.offsets_ = CudaBuffer<int>(static_cast<std::size_t>(out.coarseRows_) + 1);
            out.members_ = CudaBuffer<int>(static_cast<std::size_t>(out.fineRows_));
            copy(out.aggregate_.data(), map, out.aggregate_.sizeBytes());
            copy(out.offsets_.data(), off, out.offsets_.sizeBytes());
            copy(out.members_.data(), mem, out.members_.sizeBytes());
            ctx_->synchronize();
            return out;
        });
    }

    /// Ac = P^T A P for the piecewise-constant P of the transfer.
    CsrMatrix<double> galerkin(const CsrMatrix<double> &a, const AggregateTransfer &t) {
        if (a.rowCount() != std::size_t(t.fineRows_) || t.coarseRows_ < 1)
            throw std::invalid_argument("AMG transfer dimension mismatch");
        return b200::onContext(*ctx_, [&] {
            const tf_csr v = b200::describe(a);
            tf_dcsr *out = nullptr;
            b200::check(tf_galerkin_map(ctx_->get(), &v, detail::onDevice(t.aggregate_), t.coarseRows_, &out));
            return detail::adopt(out, *ctx_);
        });
    }

  private:
    int device() const noexcept { return ctx_->device(); }

    void copy(void *dst, const void *src, std::size_t bytes) {
        if (bytes)
            thermofem::detail::cudaCall(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx_->stream()),
                                        "cudaMemcpyAsync");
    }
    CudaBuffer<double> rowMaxima(const CsrMatrix<double> &a) {
        CudaBuffer<double> rowMax(a.rowCount());
        const tf_csr v = b200::describe(a);
        int bad = 0;
        b200::check(tf_row_stats(ctx_->get(), &v, rowMax.data(), &bad));
        if (bad)
            throw std::invalid_argument("Native AMG: missing/zero diagonal, non-finite value or reciprocal in hierarchy");
        return rowMax;
    }

    bool compact_;
    std::unique_ptr<b200::Context> ctx_;
};

namespace detail {

template <linalg::Scalar T>
void checkTransfer(const AggregateTransfer &t, const Vector<T> &fine, const Vector<T> &coarse) {
    const int owner = t.aggregate_.deviceId();
    if (fine.size() != std::size_t(t.fineRows_) || coarse.size() != std::size_t(t.coarseRows_) ||
        fine.deviceId() != owner || coarse.deviceId() != owner || fine.memoryType() != MemoryType::Global ||
        coarse.memoryType() != MemoryType::Global || fine.data() == coarse.data())
        throw std::invalid_argument("Invalid aggregate transfer vectors");
}

}  // namespace detail

/// coarse[c] = sum of fine over the members of aggregate c (member order).
template <linalg::Scalar T>
void restrictAggregates(const AggregateTransfer &t, const Vector<T> &fine, Vector<T> &coarse) {
    detail::checkTransfer(t, fine, coarse);
    auto &ctx = b200::ambient(t.aggregate_.deviceId());
    b200::onContext(ctx, [&] {
        b200::check(tf_restrict(ctx.get(), b200::valueType<T>(), t.coarseRows_, detail::onDevice(t.offsets_),
                                detail::onDevice(t.members_), fine.data(), coarse.data()));
    });
}

/// fine[i] += coarse[aggregate of i].
template <linalg::Scalar T>
void prolongAggregates(const AggregateTransfer &t, const Vector<T> &coarse, Vector<T> &fine) {
    detail::checkTransfer(t, fine, coarse);
    auto &ctx = b200::ambient(t.aggregate_.deviceId());
    b200::onContext(ctx, [&] {
        b200::check(tf_prolong(ctx.get(), b200::valueType<T>(), t.fineRows_, detail::onDevice(t.aggregate_),
                               coarse.data(), fine.data()));
    });
}

/// Dense partial-pivot LU of a small canonical matrix (1..256 rows), pivot
/// threshold 64 eps max|A|; a singular matrix gives singular_ = true.
inline CoarseFactor factorCoarse(const CsrMatrix<double> &a) {
    if (!a.rowCount() || a.rowCount() > 256 || a.rowCount() != a.columnCount())
        throw std::invalid_argument("GPU LU requires order 1..256");
    const int device = a.rowOffsets().deviceId();
    linalg::detail::OperationScope scope(device);
    CoarseFactor f;
    f.rows_ = static_cast<int>(a.rowCount());
    f.lu_ = CudaBuffer<double>(a.rowCount() * a.rowCount());
    f.pivots_ = CudaBuffer<int>(a.rowCount());
    auto &ctx = b200::ambient(device);
    int factored = 0;
    const tf_csr v = b200::describe(a);
    b200::onContext(ctx, [&] { b200::check(tf_coarse_lu_factor(ctx.get(), &v, f.lu_.data(), f.pivots_.data(), &factored)); });
    f.factored_ = factored != 0;
    f.singular_ = !f.factored_;
    return f;
}

/// x = A^-1 rhs from the factor (rhs and x may alias).
template <linalg::Scalar T>
void solveCoarse(const CoarseFactor &factor, const Vector<T> &rhs, Vector<T> &x) {
    const int owner = factor.lu_.deviceId();
    if (!factor.factored_ || rhs.size() != std::size_t(factor.rows_) || x.size() != rhs.size() ||
        rhs.deviceId() != owner || x.deviceId() != owner || rhs.memoryType() != MemoryType::Global ||
        x.memoryType() != MemoryType::Global)
        throw std::invalid_argument("Invalid GPU coarse solve");
    auto &ctx = b200::ambient(owner);
    b200::onContext(ctx, [&] {
        b200::check(tf_coarse_lu_solve(ctx.get(), factor.rows_, factor.lu_.data(), factor.pivots_.data(),
                                       b200::valueType<T>(), rhs.data(), x.data()));
    });
}

namespace detail {

template <class To, class From>
CudaBuffer<To> convertBuffer(const CudaBuffer<From> &in, b200::Context &ctx) {
    CudaBuffer<To> out(in.size());
    if (!in.empty()) {
        constexpr int src = std::is_floating_point_v<From> ? b200::valueType<From>() : b200::indexType<From>();
        constexpr int dst = std::is_floating_point_v<To> ? b200::valueType<To>() : b200::indexType<To>();
        b200::check(tf_convert(ctx.get(), static_cast<int64_t>(in.size()), src, in.deviceData(), dst, out.data()));
    }
    return out;
}

template <class TO, class IO, class TI, class II>
CsrMatrix<TO, IO> convertMatrix(const CsrMatrix<TI, II> &a) {
    if (a.rowCount() >= std::size_t(INT_MAX) || a.nonZeroCount() > std::size_t(INT_MAX / 2))
        throw std::length_error("AMG native index capacity exceeded");
    const int device = a.rowOffsets().deviceId();
    linalg::detail::OperationScope scope(device);
    CsrMatrix<TI, II> global;
    const CsrMatrix<TI, II> *m = &a;
    if (a.memoryType() != MemoryType::Global) {
        global = a;
        global.changeMemoryType(GlobalMemory{});
        m = &global;
    }
    auto &ctx = b200::ambient(device);
    return b200::onContext(ctx, [&] {
        auto rp = convertBuffer<IO>(m->rowOffsets(), ctx);
        auto ci = convertBuffer<IO>(m->columnIndices(), ctx);
        auto val = convertBuffer<TO>(m->values(), ctx);
        ctx.synchronize();
        return CsrMatrix<TO, IO>::fromBuffers(a.rowCount(), a.columnCount(), std::move(rp), std::move(ci),
                                              std::move(val));
    });
}

}  // namespace detail

template <linalg::Scalar T, CsrIndex I>
CsrMatrix<T, I> fromNativeMatrix(const CsrMatrix<double> &a) {
    return detail::convertMatrix<T, I>(a);
}

template <linalg::Scalar T, CsrIndex I>
CsrMatrix<double> toNativeMatrix(const CsrMatrix<T, I> &a) {
    return detail::convertMatrix<double, int>(a);
}

}  // namespace thermofem::multigrid
