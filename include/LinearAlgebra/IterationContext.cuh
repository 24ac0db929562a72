// IterationContext.cuh -- the per-operator execution resources of the
// iteration kernels (drop-in for include/LinearAlgebra/IterationContext.cuh
// of Mgepahmge/ThermoFEM, lines 42-79: the same methods, checks and
// messages).  The reference keeps cuBLAS/cuSPARSE handles and an SpMV
// descriptor here; this one keeps a tf_ctx and calls the library's own
// kernels: tf_spmv, tf_residual (one pass instead of SpMV + scale + axpy),
// tf_axpby, tf_dot_multi (FP64 accumulation, deterministic order) and
// tf_jacobi_update.
//
// Contract kept: construction takes a canonical (row-sorted, duplicates
// summed) global snapshot of the matrix, so the caller may change or destroy
// the matrix afterwards; vectors must be global vectors on the snapshot's
// device; calls are synchronous and restore the caller's device; SpMV and
// residual outputs must not alias their inputs; one instance is not for
// concurrent use.
#pragma once

#include <LinearAlgebra/Operations.cuh>

#include <cmath>
#include <memory>

namespace thermofem::linalg {

template <Scalar T, CsrIndex I = int>
class IterationContext {
  public:
    explicit IterationContext(const CsrMatrix<T, I> &matrix) {
        detail::librarySize(matrix.rowCount());
        detail::librarySize(matrix.columnCount());
        const int owner = matrix.rowOffsets().deviceId();
        detail::OperationScope scope(owner);
        impl_ = std::make_unique<Impl>(matrix, owner >= 0 ? owner : b200::currentDevice());
    }
    ~IterationContext() noexcept = default;
    IterationContext(const IterationContext &) = delete;
    IterationContext &operator=(const IterationContext &) = delete;

    const CsrMatrix<T, I> &matrix() const noexcept { return impl_->matrix; }

    /// y = A x.
    void multiply(const Vector<T> &x, Vector<T> &y) {
        auto &s = *impl_;
        s.accept(x);
        s.accept(y);
        if (x.size() != s.matrix.columnCount() || y.size() != s.matrix.rowCount() ||
            (!x.empty() && x.data() == y.data()))
            throw std::invalid_argument("SpMV shape or alias mismatch");
        s.run([&] {
            if (!s.matrix.nonZeroCount()) return s.zero(y);
            b200::check(tf_spmv(s.ctx.get(), &s.view, x.data(), y.data()));
        });
    }

    /// out = rhs - A x in one pass.
    void residual(const Vector<T> &rhs, const Vector<T> &x, Vector<T> &out) {
        auto &s = *impl_;
        s.accept(rhs);
        if (rhs.size() != out.size() || (!rhs.empty() && rhs.data() == out.data()))
            throw std::invalid_argument("Residual shape or alias mismatch");
        s.accept(x);
        s.accept(out);
        if (x.size() != s.matrix.columnCount() || out.size() != s.matrix.rowCount() ||
            (!x.empty() && x.data() == out.data()))
            throw std::invalid_argument("SpMV shape or alias mismatch");
        s.run([&] {
            if (!s.matrix.nonZeroCount()) {
                if (!out.empty())
                    thermofem::detail::cudaCall(cudaMemcpyAsync(out.data(), rhs.data(), out.sizeBytes(),
                                                                cudaMemcpyDeviceToDevice, s.ctx.stream()),
                                                "cudaMemcpyAsync");
                return;
            }
            b200::check(tf_residual(s.ctx.get(), &s.view, rhs.data(), x.data(), out.data()));
        });
    }

    void clear(Vector<T> &x) {
        auto &s = *impl_;
        s.accept(x);
        s.run([&] { s.zero(x); });
    }

    /// y += alpha x.
    void axpy(T alpha, const Vector<T> &x, Vector<T> &y) {
        auto &s = *impl_;
        s.accept(x);
        s.accept(y);
        if (x.size() != y.size()) throw std::invalid_argument("AXPY shape mismatch");
        if (x.empty()) return;
        s.run([&] {
            b200::check(tf_axpby(s.ctx.get(), b200::valueType<T>(), static_cast<int64_t>(x.size()), alpha, x.data(),
                                 1.0, y.data()));
        });
    }

    /// x *= alpha (the old value is not multiplied by zero: x = alpha x).
    void scale(T alpha, Vector<T> &x) {
        auto &s = *impl_;
        s.accept(x);
        if (x.empty()) return;
        s.run([&] {
            b200::check(tf_axpby(s.ctx.get(), b200::valueType<T>(), static_cast<int64_t>(x.size()), alpha, x.data(),
                                 0.0, x.data()));
        });
    }

    T dot(const Vector<T> &x, const Vector<T> &y) {
        auto &s = *impl_;
        s.accept(x);
        s.accept(y);
        if (x.size() != y.size()) throw std::invalid_argument("Dot shape mismatch");
        if (x.empty()) return T{};
        return static_cast<T>(s.dot(x.data(), y.data(), x.size()));
    }

    T norm(const Vector<T> &x) {
        auto &s = *impl_;
        s.accept(x);
        if (x.empty()) return T{};
        return static_cast<T>(std::sqrt(s.dot(x.data(), x.data(), x.size())));
    }

    /// x += weight * inverse * (rhs - product), product = A x formed before.
    void jacobi(T weight, const Vector<T> &inverse, const Vector<T> &rhs, const Vector<T> &product, Vector<T> &x) {
        auto &s = *impl_;
        s.accept(inverse);
        s.accept(rhs);
        s.accept(product);
        s.accept(x);
        if (inverse.size() != x.size() || rhs.size() != x.size() || product.size() != x.size())
            throw std::invalid_argument("Jacobi shape mismatch");
        if (x.empty()) return;
        s.run([&] {
            b200::check(tf_jacobi_update(s.ctx.get(), b200::valueType<T>(), static_cast<int64_t>(x.size()), weight,
                                         inverse.data(), rhs.data(), product.data(), x.data()));
        });
    }

  private:
    struct Impl {
        int device;
        b200::Context ctx;
        CsrMatrix<T, I> matrix;
        tf_csr view{};
        CudaBuffer<double> scalar;

        Impl(const CsrMatrix<T, I> &input, int owner) : device(owner), ctx(owner), scalar(1) {
            CsrMatrix<T, I> global(input);
            if (global.memoryType() != MemoryType::Global) global.changeMemoryType(GlobalMemory{});
            int flags = 0;
            if (global.nonZeroCount()) {
                const tf_csr v = b200::describe(global);
                b200::onContext(ctx, [&] { b200::check(tf_csr_check_canonical(ctx.get(), &v, &flags)); });
            }
            if (flags & 2) throw std::invalid_argument("Matrix contains nonfinite entries");
            matrix = (flags & 1) ? detail::canonical<I>(global) : std::move(global);
            view = b200::describe(matrix);
        }

        void accept(const Vector<T> &v) const {
            detail::librarySize(v.size());
            if (v.memoryType() != MemoryType::Global || (!v.empty() && v.deviceId() != device))
                throw std::invalid_argument("Iteration workspace requires same-device global vectors");
        }
        template <class F>
        void run(F &&f) {
            b200::onContext(ctx, std::forward<F>(f));
        }
        void zero(Vector<T> &v) {
            if (!v.empty())
                thermofem::detail::cudaCall(cudaMemsetAsync(v.data(), 0, v.sizeBytes(), ctx.stream()),
                                            "cudaMemsetAsync");
        }
        double dot(const T *x, const T *y, std::size_t n) {
            double result = 0;
            const void *xs[1] = {x}, *ys[1] = {y};
            run([&] {
                b200::check(tf_dot_multi(ctx.get(), b200::valueType<T>(), static_cast<int64_t>(n), 1, xs, ys,
                                         scalar.data()));
                thermofem::detail::cudaCall(cudaMemcpyAsync(&result, scalar.data(), sizeof(double),
                                                            cudaMemcpyDeviceToHost, ctx.stream()),
                                            "cudaMemcpyAsync");
            });
            return result;
        }
    };
    std::unique_ptr<Impl> impl_;
};

}  // namespace thermofem::linalg
