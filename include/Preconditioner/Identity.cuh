// Identity.cuh -- the identity preconditioner, x = rhs (drop-in for
// include/Preconditioner/Identity.cuh:17-36 of Mgepahmge/ThermoFEM).  Setup
// checks the matrix is a nonempty square matrix with finite values (on its
// device); apply checks shapes and devices.  A solver given this
// preconditioner runs it inside its own fused device loop.
#pragma once

#include <Solver/Interfaces.cuh>

namespace thermofem {

template <linalg::Scalar T, CsrIndex I = int>
class Identity final : public Preconditioner<T, I> {
  public:
    void setup(const CsrMatrix<T, I> &matrix) override {
        iteration::validateMatrix(matrix);
        const int device = matrix.rowOffsets().deviceId();
        if (matrix.nonZeroCount()) {
            linalg::detail::OperationScope scope(device);
            CsrMatrix<T, I> global;
            const CsrMatrix<T, I> *m = &matrix;
            if (matrix.memoryType() != MemoryType::Global) {
                global = matrix;
                global.changeMemoryType(GlobalMemory{});
                m = &global;
            }
            const tf_csr view = b200::describe(*m);
            int flags = 0;
            auto &ctx = b200::ambient(device);
            b200::onContext(ctx, [&] { b200::check(tf_csr_check_canonical(ctx.get(), &view, &flags)); });
            if (flags & 2) throw std::invalid_argument("Nonfinite identity setup matrix");
        }
        size_ = matrix.rowCount();
        device_ = device;
    }
    void apply(const Vector<T> &rhs, Vector<T> &x) override {
        if (!size_) throw std::logic_error("Identity requires setup");
        iteration::validateVectors(size_, device_, rhs, x);
        x.copyDataFrom(rhs);
    }

  private:
    std::size_t size_{0};
    int device_{-1};
};

}  // namespace thermofem
