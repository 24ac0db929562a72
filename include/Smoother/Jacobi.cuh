// Jacobi.cuh -- the weighted Jacobi smoother, `sweeps` times
// x += w D^-1 (rhs - A x) from the current x (drop-in for
// include/Smoother/Jacobi.cuh:26-93 of Mgepahmge/ThermoFEM: the same
// constructor defaults and checks, transactional setup, rhs/x aliasing).
// Runs on the library's Jacobi component (tf_jacobi_*): each sweep is one
// fused SpMV + update kernel over the setup's snapshot of the matrix and its
// inverse diagonal.
#pragma once

#include <LinearAlgebra/Diagonal.cuh>
#include <Solver/Interfaces.cuh>

#include <cmath>

namespace thermofem {

template <linalg::Scalar T, CsrIndex I = int>
class Jacobi final : public Smoother<T, I> {
  public:
    explicit Jacobi(int sweeps = 2, T weight = T(2) / T(3)) : sweeps_(sweeps), weight_(weight) {
        if (sweeps < 1 || !std::isfinite(weight) || weight <= 0 || weight >= 2)
            throw std::invalid_argument("Invalid Jacobi parameters");
    }

    /// Builds the new state completely before replacing the old one, so a
    /// failed setup leaves the previous matrix in use.
    void setup(const CsrMatrix<T, I> &matrix) override {
        iteration::validateMatrix(matrix);
        const int device = matrix.rowOffsets().deviceId();
        linalg::detail::OperationScope scope(device);
        auto next = std::make_unique<State>(device, matrix.rowCount());
        CsrMatrix<T, I> global;
        const CsrMatrix<T, I> *m = &matrix;
        if (matrix.memoryType() != MemoryType::Global) {
            global = matrix;
            global.changeMemoryType(GlobalMemory{});
            m = &global;
        }
        const tf_csr view = b200::describe(*m);
        b200::onContext(next->ctx, [&] {
            tf_jacobi *h = nullptr;
            b200::check(tf_jacobi_create(next->ctx.get(), b200::valueType<T>(), b200::indexType<I>(), sweeps_,
                                         static_cast<double>(weight_), &h));
            next->handle.reset(h);
            const int status = tf_jacobi_setup(h, &view);
            if (status == TF_ERR_INVALID) {
                const std::string why = tf_last_error();
                throw std::invalid_argument(why.find("nonfinite") != std::string::npos ? why
                                                                                        : "Missing or invalid diagonal");
            }
            b200::check(status);
        });
        state_ = std::move(next);
    }

    void apply(const Vector<T> &rhs, Vector<T> &x) override {
        if (!state_) throw std::logic_error("Jacobi requires setup");
        auto &s = *state_;
        iteration::validateVectors(s.rows, s.ctx.device(), rhs, x);
        linalg::detail::OperationScope scope(s.ctx.device());
        b200::DeviceSide<T> in(rhs, true), out(x, true);
        b200::onContext(s.ctx, [&] { b200::check(tf_jacobi_apply(s.handle.get(), in.get(), out.get())); });
        out.writeBack(x);
    }

  private:
    struct Release {
        void operator()(tf_jacobi *j) const noexcept { tf_jacobi_destroy(j); }
    };
    struct State {
        b200::Context ctx;
        std::size_t rows;
        std::unique_ptr<tf_jacobi, Release> handle;
        State(int device, std::size_t n) : ctx(device), rows(n) {}
    };
    int sweeps_;
    T weight_;
    std::unique_ptr<State> state_;
};

}  // namespace thermofem
