// component_test.cpp -- the C++ component layer's paths that the reference's
// own tests do not reach: solvers driven from the host because their
// preconditioner is the caller's (a class of its own, or Amg with a smoother
// factory), checked against the fused device path on the same problems, and
// the iteration context's kernels against host arithmetic.
//   tests/cxx/bin/component-tests [--gtest_filter=...]
#include <Preconditioner/Amg.cuh>
#include <Solver/BiCgStab.cuh>
#include <Solver/Cg.cuh>
#include <gtest/gtest.h>

#include <cmath>
#include <numeric>

namespace {

using namespace thermofem;

bool haveDevice() {
    int count = 0;
    return cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
}

// 3-D 7-point Laplacian with a varying diagonal shift on an m^3 grid.
template <class T, class I = int>
CsrMatrix<T, I> grid3(int m, double shift = 0.0) {
    const int n = m * m * m;
    std::vector<I> off{0}, col;
    std::vector<T> val;
    for (int i = 0; i < n; ++i) {
        const int x = i % m, y = (i / m) % m, z = i / (m * m);
        const int nb[6] = {z > 0 ? i - m * m : -1, y > 0 ? i - m : -1, x > 0 ? i - 1 : -1,
                           x < m - 1 ? i + 1 : -1, y < m - 1 ? i + m : -1, z < m - 1 ? i + m * m : -1};
        for (int k = 0; k < 3; ++k)
            if (nb[k] >= 0) col.push_back(nb[k]), val.push_back(T(-1));
        col.push_back(i);
        val.push_back(T(6.0 + shift * (1 + (i % 7))));
        for (int k = 3; k < 6; ++k)
            if (nb[k] >= 0) col.push_back(nb[k]), val.push_back(T(-1));
        off.push_back(static_cast<I>(val.size()));
    }
    return CsrMatrix<T, I>(n, n, off, col, val);
}

template <class T>
std::vector<T> rhsOf(std::size_t n) {
    std::vector<T> b(n);
    for (std::size_t i = 0; i < n; ++i) b[i] = T(std::sin(0.37 * double(i)) + 0.5);
    return b;
}

// A preconditioner of the caller's own: x = D^-1 rhs, written with the public
// API only (the iteration context's Jacobi update from x = 0 with A x = 0).
template <class T, class I = int>
class DiagonalScaling final : public Preconditioner<T, I> {
  public:
    void setup(const CsrMatrix<T, I> &a) override {
        context_ = std::make_unique<linalg::IterationContext<T, I>>(a);
        inverse_ = linalg::inverseDiagonal(a);
        zeros_ = Vector<T>(a.rowCount());
        context_->clear(zeros_);
        ++setups;
    }
    void apply(const Vector<T> &rhs, Vector<T> &x) override {
        context_->clear(x);
        context_->jacobi(T(1), inverse_, rhs, zeros_, x);
        ++applies;
    }
    int setups = 0, applies = 0;

  private:
    std::unique_ptr<linalg::IterationContext<T, I>> context_;
    Vector<T> inverse_, zeros_;
};

// The identity, as a caller's class: the host loop must then take the
// fused Identity solve's iterations.
template <class T, class I = int>
class CopyThrough final : public Preconditioner<T, I> {
  public:
    void setup(const CsrMatrix<T, I> &) override {}
    void apply(const Vector<T> &rhs, Vector<T> &x) override { x.copyDataFrom(rhs); }
};

template <class T>
double relDiff(const std::vector<T> &a, const std::vector<T> &b) {
    double num = 0, den = 0;
    for (std::size_t i = 0; i < a.size(); ++i) {
        num += (double(a[i]) - double(b[i])) * (double(a[i]) - double(b[i]));
        den += double(b[i]) * double(b[i]);
    }
    return std::sqrt(num / den);
}

class ComponentTest : public ::testing::Test {
  protected:
    void SetUp() override {
        if (!haveDevice()) GTEST_SKIP() << "CUDA unavailable";
        ASSERT_EQ(cudaSetDevice(0), cudaSuccess);
    }
};

TEST_F(ComponentTest, callerPreconditionerCgMatchesTheFusedIdentitySolve) {
    const auto a = grid3<double>(12);
    const auto b = rhsOf<double>(a.rowCount());
    const std::vector<double> zero(a.rowCount(), 0.0);
    Vector<double> rhs{std::span<const double>(b)};
    Vector<double> x1{std::span<const double>(zero)}, x2{std::span<const double>(zero)};
    Cg<double> fused({}, std::make_unique<Identity<double>>());
    Cg<double> host({}, std::make_unique<CopyThrough<double>>());
    fused.setup(a);
    host.setup(a);
    const auto r1 = fused.apply(rhs, x1);
    const auto r2 = host.apply(rhs, x2);
    ASSERT_EQ(r1.status_, SolveStatus::Converged);
    ASSERT_EQ(r2.status_, SolveStatus::Converged);
    EXPECT_LE(std::abs(r1.iterations_ - r2.iterations_), 1);
    EXPECT_LT(relDiff(linalg::detail::hostCopy(x2), linalg::detail::hostCopy(x1)), 1e-9);
    EXPECT_LE(r2.relativeResidual_, 1e-8);
}

TEST_F(ComponentTest, callerDiagonalPreconditionerIsUsedAndConverges) {
    const auto a = grid3<double>(10, 3.0);
    const auto b = rhsOf<double>(a.rowCount());
    const std::vector<double> zero(a.rowCount(), 0.0);
    auto owned = std::make_unique<DiagonalScaling<double>>();
    auto *pre = owned.get();
    CgOptions<double> o;
    o.relativeTolerance_ = 1e-10;
    Cg<double> cg(o, std::move(owned));
    cg.setup(a);
    EXPECT_EQ(pre->setups, 1);
    Vector<double> rhs{std::span<const double>(b), PinnedMemory{}}, x{std::span<const double>(zero), PinnedMemory{}};
    const auto r = cg.apply(rhs, x);
    ASSERT_EQ(r.status_, SolveStatus::Converged);
    EXPECT_EQ(pre->applies, r.iterations_);
    EXPECT_EQ(x.memoryType(), MemoryType::Pinned);
    // the true residual, on the host
    const auto xs = linalg::detail::hostCopy(x);
    const auto off = linalg::detail::hostCopy(a.rowOffsets());
    const auto col = linalg::detail::hostCopy(a.columnIndices());
    const auto val = linalg::detail::hostCopy(a.values());
    double rr = 0, bb = 0;
    for (std::size_t i = 0; i < b.size(); ++i) {
        double ax = 0;
        for (int j = off[i]; j < off[i + 1]; ++j) ax += val[j] * xs[col[j]];
        rr += (b[i] - ax) * (b[i] - ax);
        bb += b[i] * b[i];
    }
    EXPECT_LE(std::sqrt(rr / bb), 1.01e-10);
    EXPECT_NEAR(r.residualNorm_, std::sqrt(rr), 1e-9 * std::sqrt(bb));
}

template <class T, class I>
void factoryAmgMatchesDefaultAmg() {
    const auto a = grid3<T, I>(16, 0.5);
    const auto b = rhsOf<T>(a.rowCount());
    const std::vector<T> zero(a.rowCount(), T(0));
    AmgOptions<T> ao;
    ao.jacobiWeight_ = T(2) / T(3);
    int made = 0;
    auto factory = [&made, w = ao.jacobiWeight_]() -> std::unique_ptr<Smoother<T, I>> {
        ++made;
        return std::make_unique<Jacobi<T, I>>(1, w);
    };
    BiCgStabOptions<T> so;
    so.relativeTolerance_ = std::same_as<T, float> ? T(1e-5) : T(1e-9);
    BiCgStab<T, I> fused(so, std::make_unique<Amg<T, I>>(ao));
    auto owned = std::make_unique<Amg<T, I>>(ao, factory);
    auto *amg = owned.get();
    BiCgStab<T, I> host(so, std::move(owned));
    fused.setup(a);
    host.setup(a);
    EXPECT_EQ(static_cast<std::size_t>(made), 2 * (amg->levelCount() - 1));
    Vector<T> rhs{std::span<const T>(b)}, x1{std::span<const T>(zero)}, x2{std::span<const T>(zero)};
    const auto r1 = fused.apply(rhs, x1);
    const auto r2 = host.apply(rhs, x2);
    ASSERT_EQ(r1.status_, SolveStatus::Converged);
    ASSERT_EQ(r2.status_, SolveStatus::Converged);
    // the same hierarchy and the same smoothing: the same solve up to rounding
    EXPECT_LE(std::abs(r1.iterations_ - r2.iterations_), 1);
    EXPECT_LT(relDiff(linalg::detail::hostCopy(x2), linalg::detail::hostCopy(x1)),
              (std::same_as<T, float> ? 1e-3 : 1e-7));
    // the cycle itself: one apply of each on the same right-hand side
    Amg<T, I> plain(ao), injected(ao, factory);
    plain.setup(a);
    injected.setup(a);
    Vector<T> z1(a.rowCount()), z2(a.rowCount());
    plain.apply(rhs, z1);
    injected.apply(rhs, z2);
    EXPECT_LT(relDiff(linalg::detail::hostCopy(z2), linalg::detail::hostCopy(z1)),
              (std::same_as<T, float> ? 1e-5 : 1e-12));
    EXPECT_EQ(plain.lastCycleVisits(), injected.lastCycleVisits());
}

TEST_F(ComponentTest, factorySmoothersDriveTheHostCycleLikeTheFusedOne) { factoryAmgMatchesDefaultAmg<double, int>(); }
TEST_F(ComponentTest, factorySmoothersDriveTheHostCycleLikeTheFusedOneFloatWide) {
    factoryAmgMatchesDefaultAmg<float, std::int64_t>();
}

TEST_F(ComponentTest, cgWithFactoryAmgTakesTheHostLoop) {
    const auto a = grid3<double>(14);
    const auto b = rhsOf<double>(a.rowCount());
    const std::vector<double> zero(a.rowCount(), 0.0);
    AmgOptions<double> ao;
    ao.cycle_ = multigrid::Cycle::W;
    Cg<double> fused({}, std::make_unique<Amg<double>>(ao));
    Cg<double> host({}, std::make_unique<Amg<double>>(ao, [] { return std::make_unique<Jacobi<double>>(1, 0.75); }));
    fused.setup(a);
    host.setup(a);
    Vector<double> rhs{std::span<const double>(b)}, x1{std::span<const double>(zero)}, x2{std::span<const double>(zero)};
    const auto r1 = fused.apply(rhs, x1), r2 = host.apply(rhs, x2);
    ASSERT_EQ(r1.status_, SolveStatus::Converged);
    ASSERT_EQ(r2.status_, SolveStatus::Converged);
    EXPECT_EQ(r1.iterations_, r2.iterations_);
    EXPECT_LT(relDiff(linalg::detail::hostCopy(x2), linalg::detail::hostCopy(x1)), 1e-10);
}

TEST_F(ComponentTest, iterationContextKernelsMatchHostArithmetic) {
    const auto a = grid3<double, std::int64_t>(9, 1.0);
    const std::size_t n = a.rowCount();
    std::vector<double> xv(n), yv(n);
    for (std::size_t i = 0; i < n; ++i) xv[i] = std::cos(0.1 * double(i)), yv[i] = std::sin(0.2 * double(i)) + 2;
    linalg::IterationContext<double, std::int64_t> ctx(a);
    Vector<double> x{std::span<const double>(xv)}, y{std::span<const double>(yv)}, out(n);
    ctx.multiply(x, out);
    const auto off = linalg::detail::hostCopy(a.rowOffsets());
    const auto col = linalg::detail::hostCopy(a.columnIndices());
    const auto val = linalg::detail::hostCopy(a.values());
    const auto got = linalg::detail::hostCopy(out);
    double dot = 0;
    for (std::size_t i = 0; i < n; ++i) {
        double ax = 0;
        for (auto j = off[i]; j < off[i + 1]; ++j) ax += val[j] * xv[col[j]];
        EXPECT_NEAR(got[i], ax, 1e-13 * (1 + std::abs(ax)));
        dot += xv[i] * yv[i];
    }
    EXPECT_NEAR(ctx.dot(x, y), dot, 1e-12 * std::abs(dot));
    ctx.residual(y, x, out);
    const auto res = linalg::detail::hostCopy(out);
    for (std::size_t i = 0; i < n; ++i) EXPECT_NEAR(res[i], yv[i] - got[i], 1e-13 * (1 + std::abs(yv[i])));
    ctx.scale(-2.0, out);
    ctx.axpy(0.5, x, out);
    const auto s = linalg::detail::hostCopy(out);
    for (std::size_t i = 0; i < n; ++i) EXPECT_NEAR(s[i], -2.0 * res[i] + 0.5 * xv[i], 1e-12);
    EXPECT_THROW(ctx.multiply(x, x), std::invalid_argument);
    Vector<double> pinned(n, PinnedMemory{});
    EXPECT_THROW(ctx.multiply(x, pinned), std::invalid_argument);
}

}  // namespace
