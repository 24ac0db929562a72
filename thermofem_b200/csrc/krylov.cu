// krylov.cu -- PCG and right-preconditioned BiCGStab with the scalar
// recurrences on the device.
//
// The control flow is the reference's (PCG: include/Solver/Cg.cuh:123-189;
// BiCGStab: include/Solver/BiCgStab.cuh:144-247), including the
// breakdown/non-finite checks, the true-residual confirmation of a candidate
// convergence and the periodic refresh with restart.  The difference is
// where it runs: each scalar decision runs in the last CTA of the reduction
// it consumes (a device ticket; tile::finish), which adds the partial sums in
// a fixed order and updates a device-resident state record, and the vector
// kernels are gated on that record, so one iteration is a fixed kernel
// sequence captured once into a CUDA graph.  Reductions are fused
// into the producing pass (p.Ap into the SpMV that makes Ap, ||r||^2 into the
// x/r update, t.t and t.s into the SpMV that makes t).  The host reads one
// word per iteration to stop the loop.
#include "engine.cuh"
#include "tile.cuh"

namespace tfb {
namespace {

enum : int { kRunning = -1 };

struct KState {
    double normB, tol, res, rho, rho_prev, alpha, omega, beta, curv;
    int it, status, running, fresh, pmode, refresh, early, normal, copy_shadow, max_it, interval;
    unsigned tickets[8];  // last-CTA tickets of the reductions (zero between launches)
};

constexpr int kParts = 1184;  // upper bound of grid-stride partial sums

int parts_for(int64_t n) {
    int64_t p = (n + 2047) / 2048;
    return static_cast<int>(p < 1 ? 1 : (p > kParts ? kParts : p));
}

// Fixed-order sum of K partial arrays [K][parts]; valid in thread 0.  Thread
// t < 256 adds entries t, t + 256, t + 512, ... in that order, the loads
// issued eight at a time (they come from L2, written by other CTAs).  The
// stride is fixed, not blockDim: the finisher runs in the last CTA of
// whichever kernel produced the partials (256 threads for the sliced SpMV,
// 288 for the pipelined CSR one, 1024 for the one-CTA steps), and the sum
// must not depend on which.  Threads past 256 contribute +0.0, which leaves
// the block reduction's value unchanged.  Needs blockDim.x >= 256.
template <int K>
__device__ __forceinline__ void sum_partials(const double *part, int parts, double (&v)[K]) {
    constexpr int kBatch = 8;
    constexpr int step = tile::kThreads;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        v[k] = 0.0;
        if (threadIdx.x >= step) continue;
        for (int p0 = threadIdx.x; p0 < parts; p0 += step * kBatch) {
            double t[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int p = p0 + u * step;
                t[u] = p < parts ? __ldcg(part + k * parts + p) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u) v[k] += t[u];
        }
    }
    tile::block_reduce<K>(v);
}

__device__ __forceinline__ void stop(KState *s, int status) {
    s->status = status;
    s->running = 0;
}

// ---- shared steps --------------------------------------------------------

// After r = b - A x0 and ||b||^2 partials: initial decisions (Cg.cuh:125-137).
__global__ void k_init(KState *s, const double *pb, int nb, const double *pr, int nr, int bicg) {
    pdl_enter();
    double vb[1], vr[1];
    sum_partials<1>(pb, nb, vb);
    __syncthreads();
    sum_partials<1>(pr, nr, vr);
    if (threadIdx.x) return;
    s->normB = sqrt(vb[0]);
    s->tol = fmax(s->tol, s->res * s->normB);  // s->res carries rtol in, tol carries atol in
    s->res = sqrt(vr[0]);
    s->it = 0;
    s->fresh = 1;
    s->refresh = s->early = s->copy_shadow = 0;
    s->normal = 1;
    s->rho_prev = 1;
    s->alpha = 1;
    s->omega = 1;
    if (!isfinite(s->normB) || !isfinite(s->res)) stop(s, TF_NONFINITE);
    else if (s->res <= s->tol) stop(s, TF_CONVERGED);
    else {
        s->status = kRunning;
        s->running = 1;
        s->copy_shadow = bicg;  // BiCGStab: shadow = r
    }
}

// Final report from the true residual (Cg.cuh:105-121, BiCgStab.cuh:122-136).
__global__ void k_finish(KState *s, const double *pr, int nr) {
    pdl_enter();
    double v[1];
    sum_partials<1>(pr, nr, v);
    if (threadIdx.x) return;
    const double res = sqrt(v[0]);
    int status = s->status == kRunning ? TF_MAX_ITERATIONS : s->status;
    if (!isfinite(res) || !isfinite(s->normB)) status = TF_NONFINITE;
    else if (res <= s->tol) status = TF_CONVERGED;
    else if (status == TF_CONVERGED) status = TF_MAX_ITERATIONS;
    s->status = status;
    s->res = res;
    s->running = 0;
}

template <class T>
__global__ void k_copy_if(const int *flag, int64_t n, const T *__restrict__ src, T *__restrict__ dst) {
    pdl_enter();
    if (!*flag) return;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dst[i] = src[i];
}

// Loads the initial state of a solve (batched graphs carry it as a parameter).
__global__ void k_reset(KState *s, KState init) {
    pdl_enter();
    *s = init;
}

// Re-arms the WHILE node of the solve graph: one more iteration while the
// recurrence is running and below the iteration limit.
__global__ void k_set_continue(cudaGraphConditionalHandle handle, const KState *s) {
    pdl_enter();
    cudaGraphSetConditional(handle, (s->running && s->it < s->max_it) ? 1u : 0u);
}

template <class T, class Fin = tile::NoFinal>
__global__ void k_dot(int64_t n, const T *__restrict__ x, const T *__restrict__ y, double *part, Fin fin = {}) {
    pdl_enter();
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        v[0] += static_cast<double>(x[i]) * static_cast<double>(y[i]);
    tile::block_reduce<1>(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    tile::finish(fin, part, gridDim.x);
}

// z = T(xs) (the preconditioner's output in its own storage) and
// sum_i r_i z_i, in the grid and order of k_dot: the conversion that ends
// the preconditioner fused into the dot that follows it (same bits).
template <class T, class S, class Fin>
__global__ void k_dot_from(int64_t n, const T *__restrict__ r, const S *__restrict__ xs, T *__restrict__ z,
                           double *part, Fin fin) {
    pdl_enter();
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const T zi = static_cast<T>(xs[i]);
        if (z) z[i] = zi;  // (null: the next step reads xs itself)
        v[0] += static_cast<double>(r[i]) * static_cast<double>(zi);
    }
    tile::block_reduce<1>(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    tile::finish(fin, part, gridDim.x);
}

// x_j read from the preconditioner's output in its own storage S.
template <class T, class S>
struct ConvertX {
    const S *__restrict__ x;
    __device__ __forceinline__ T operator()(int64_t j) const { return static_cast<T>(__ldg(x + j)); }
    struct View {
        const S *__restrict__ p;
        __device__ __forceinline__ T operator()(int c) const { return static_cast<T>(__ldg(p + c)); }
    };
    __device__ __forceinline__ View row(int64_t i) const { return {x + i}; }
};

// Epi that also stores each row's own converted x_i into z: the SpMV that
// follows the preconditioner writes the converted vector the later steps
// read (in place of a separate conversion kernel).
template <class T, class Epi>
struct StoreOwnX {
    static constexpr int kReduce = Epi::kReduce;
    struct Pre {
        typename Epi::Pre inner;
        T xi;
    };
    Epi inner;
    T *__restrict__ z;
    double *partial;
    decltype(Epi::fin) fin;
    bool rarely_runs() const { return tile::rarely_runs(inner, 0); }
    __device__ __forceinline__ bool skip() const { return inner.skip(); }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &xs) const {
        return {inner.pre(i, xs), xs(i)};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p,
                                               double (&red)[kReduce > 0 ? kReduce : 1]) const {
        z[i] = p.xi;
        inner(i, acc, p.inner, red);
    }
};
template <class T, class Epi>
StoreOwnX<T, Epi> store_own_x(const Epi &e, T *z) {
    return StoreOwnX<T, Epi>{e, z, e.partial, e.fin};
}

// y = A x with sum_i w_i y_i; gated on *gate.
template <class T, class Fin = tile::NoFinal>
struct SpmvDot {
    static constexpr int kReduce = 1;
    struct Pre {
        T w;
    };
    T *__restrict__ y;
    const T *__restrict__ w;
    const int *gate;
    double *partial;
    Fin fin{};  // scalar step run by the last CTA
    __device__ __forceinline__ bool skip() const { return gate && !*gate; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &) const {
        return {w[i]};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&red)[1]) const {
        y[i] = acc;
        red[0] += static_cast<double>(p.w) * static_cast<double>(acc);
    }
};

// t = A x with sum t_i^2 and sum t_i s_i; gated.
template <class T, class Fin = tile::NoFinal>
struct SpmvDot2 {
    static constexpr int kReduce = 2;
    struct Pre {
        T s;
    };
    T *__restrict__ y;
    const T *__restrict__ s;
    const int *gate;
    double *partial;
    Fin fin{};  // scalar step run by the last CTA
    __device__ __forceinline__ bool skip() const { return gate && !*gate; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &) const {
        return {s[i]};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&red)[2]) const {
        y[i] = acc;
        const double t = static_cast<double>(acc);
        red[0] += t * t;
        red[1] += t * static_cast<double>(p.s);
    }
};

// r = b - A x with sum r_i^2; gated (gate may be null).
template <class T, class Fin = tile::NoFinal>
struct ResidualNorm {
    static constexpr int kReduce = 1;
    struct Pre {
        T b;
    };
    const T *__restrict__ b;
    T *__restrict__ r;
    const int *gate;
    double *partial;
    Fin fin{};  // scalar step run by the last CTA
    // Gated launches (residual refresh, early exit) rarely run: their
    // kernels do not stream the matrix before the gate is read.
    bool rarely_runs() const { return gate != nullptr; }
    __device__ __forceinline__ bool skip() const { return gate && !*gate; }
    template <class XS>
    __device__ __forceinline__ Pre pre(int64_t i, const XS &) const {
        return {b[i]};
    }
    __device__ __forceinline__ void operator()(int64_t i, T acc, const Pre &p, double (&red)[1]) const {
        const T v = p.b - acc;
        r[i] = v;
        red[0] += static_cast<double>(v) * static_cast<double>(v);
    }
};

// ---- PCG -----------------------------------------------------------------

__device__ void cg_rho_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    s->it += 1;
    const double rho = v[0];
    s->rho = rho;
    if (!isfinite(rho)) return stop(s, TF_NONFINITE);
    if (rho <= 0) return stop(s, TF_BREAKDOWN);
    if (s->fresh) {
        s->pmode = 0;
        s->fresh = 0;
    } else {
        const double beta = rho / s->rho_prev;
        if (!isfinite(beta)) return stop(s, TF_NONFINITE);
        s->beta = beta;
        s->pmode = 1;
    }
}

template <class T, class S = T>
__global__ void cg_p(const KState *s, int64_t n, const S *__restrict__ z, T *__restrict__ p) {
    pdl_enter();
    if (!s->running) return;
    const int mode = s->pmode;
    const T beta = static_cast<T>(s->beta);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const T zi = static_cast<T>(z[i]);  // exact: z is the preconditioner's output in its storage S
        p[i] = mode ? zi + beta * p[i] : zi;
    }
}

__device__ void cg_curv_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    const double c = v[0];
    s->curv = c;
    if (!isfinite(c)) return stop(s, TF_NONFINITE);
    if (c <= 0) return stop(s, TF_BREAKDOWN);
    const double alpha = s->rho / c;
    if (!isfinite(alpha)) return stop(s, TF_NONFINITE);
    s->alpha = alpha;
}

template <class T, class Fin>
__global__ void cg_xr(const KState *s, int64_t n, const T *__restrict__ p, const T *__restrict__ ap, T *__restrict__ x,
                      T *__restrict__ r, double *part, Fin fin) {
    pdl_enter();
    if (!s->running) return;
    const T alpha = static_cast<T>(s->alpha);
    double v[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        x[i] += alpha * p[i];
        const T ri = r[i] - alpha * ap[i];
        r[i] = ri;
        v[0] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    tile::block_reduce<1>(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    tile::finish(fin, part, gridDim.x);
}

// ||r|| check and refresh decision (Cg.cuh:170-178); without a refresh the
// iteration closes here (Cg.cuh:185-189).
__device__ void cg_res_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    const double res = sqrt(v[0]);
    s->res = res;
    if (!isfinite(res)) return stop(s, TF_NONFINITE);
    if (res <= s->tol || s->it % s->interval == 0) {
        s->refresh = 1;
        return;
    }
    s->rho_prev = s->rho;
    if (s->it >= s->max_it) stop(s, TF_MAX_ITERATIONS);
}

// After the gated true residual: confirm or restart (Cg.cuh:178-185), then
// close the iteration.
__device__ void cg_refresh_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    s->refresh = 0;
    const double res = sqrt(v[0]);
    s->res = res;
    if (!isfinite(res) || res <= s->tol) return stop(s, TF_MAX_ITERATIONS);
    s->fresh = 1;
    s->rho_prev = s->rho;
    if (s->it >= s->max_it) stop(s, TF_MAX_ITERATIONS);
}

// Scalar steps as last-CTA handoffs (tile::finish) of the reductions they
// consume.
#define TF_KRYLOV_FINAL(Name, step)                                                    \
    struct Name {                                                                      \
        static constexpr bool kActive = true;                                          \
        KState *s;                                                                     \
        unsigned *ticket;                                                              \
        __device__ void operator()(const double *p, int n) const { step(s, p, n); }    \
    };
TF_KRYLOV_FINAL(CgRho, cg_rho_step)
TF_KRYLOV_FINAL(CgCurv, cg_curv_step)
TF_KRYLOV_FINAL(CgRes, cg_res_step)
TF_KRYLOV_FINAL(CgRefresh, cg_refresh_step)

// ---- BiCGStab ------------------------------------------------------------

__device__ void bi_rho_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    s->it += 1;
    s->normal = 1;
    s->early = 0;
    s->copy_shadow = 0;
    const double rho = v[0];
    s->rho = rho;
    if (!isfinite(rho)) return stop(s, TF_NONFINITE);
    if (rho == 0) return stop(s, TF_BREAKDOWN);
    if (s->fresh) {
        s->pmode = 0;
        s->fresh = 0;
    } else {
        const double beta = (rho / s->rho_prev) * (s->alpha / s->omega);
        if (!isfinite(beta)) return stop(s, TF_NONFINITE);
        s->beta = beta;
        s->pmode = 1;
    }
}

// p = r (fresh) or p = r + beta (p - omega v) (BiCgStab.cuh:176-184).
template <class T>
__global__ void bi_p(const KState *s, int64_t n, const T *__restrict__ r, const T *__restrict__ v, T *__restrict__ p) {
    pdl_enter();
    if (!s->running) return;
    const int mode = s->pmode;
    const T beta = static_cast<T>(s->beta), omega = static_cast<T>(s->omega);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (mode) {
            const T t = p[i] - omega * v[i];
            p[i] = r[i] + beta * t;
        } else {
            p[i] = r[i];
        }
    }
}

__device__ void bi_alpha_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    const double den = v[0];
    if (!isfinite(den)) return stop(s, TF_NONFINITE);
    if (den == 0) return stop(s, TF_BREAKDOWN);
    const double alpha = s->rho / den;
    if (!isfinite(alpha)) return stop(s, TF_NONFINITE);
    s->alpha = alpha;
}

// s = r - alpha v, x += alpha phat, sum s_i^2.
template <class T, class Fin>
__global__ void bi_s(const KState *st, int64_t n, const T *__restrict__ r, const T *__restrict__ v,
                     const T *__restrict__ ph, T *__restrict__ sv, T *__restrict__ x, double *part, Fin fin) {
    pdl_enter();
    if (!st->running) return;
    const T alpha = static_cast<T>(st->alpha);
    double acc[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const T si = r[i] - alpha * v[i];
        sv[i] = si;
        x[i] += alpha * ph[i];
        acc[0] += static_cast<double>(si) * static_cast<double>(si);
    }
    tile::block_reduce<1>(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
    tile::finish(fin, part, gridDim.x);
}

// ||s|| check: candidate convergence takes the early path (BiCgStab.cuh:199-211).
__device__ void bi_snorm_step(KState *s, const double *part, int parts) {
    if (!s->running) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    const double ns = sqrt(v[0]);
    if (!isfinite(ns)) return stop(s, TF_NONFINITE);
    if (ns <= s->tol) {
        s->early = 1;
        s->normal = 0;
    }
}

// Early path after the gated true residual: confirm or restart, skipping the
// omega half and the rho_prev update of this iteration.
__device__ void bi_early_step(KState *s, const double *part, int parts) {
    if (!s->running || !s->early) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    const double res = sqrt(v[0]);
    s->res = res;
    if (res <= s->tol || !isfinite(res)) return stop(s, TF_MAX_ITERATIONS);
    s->copy_shadow = 1;
    s->fresh = 1;
}

__device__ void bi_omega_step(KState *s, const double *part, int parts) {
    if (!s->running || !s->normal) return;
    double v[2];
    sum_partials<2>(part, parts, v);
    if (threadIdx.x) return;
    const double tt = v[0], ts = v[1];
    if (!isfinite(tt) || !isfinite(ts)) return stop(s, TF_NONFINITE);
    if (tt == 0) return stop(s, TF_BREAKDOWN);
    const double omega = ts / tt;
    if (!isfinite(omega)) return stop(s, TF_NONFINITE);
    if (omega == 0) return stop(s, TF_BREAKDOWN);
    s->omega = omega;
}

// x += omega shat, r = s - omega t, sum r_i^2.
template <class T, class Fin>
__global__ void bi_xr(const KState *st, int64_t n, const T *__restrict__ sh, const T *__restrict__ sv,
                      const T *__restrict__ t, T *__restrict__ x, T *__restrict__ r, double *part, Fin fin) {
    pdl_enter();
    if (!st->running || !st->normal) return;
    const T omega = static_cast<T>(st->omega);
    double acc[1] = {0.0};
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        x[i] += omega * sh[i];
        const T ri = sv[i] - omega * t[i];
        r[i] = ri;
        acc[0] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    tile::block_reduce<1>(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
    tile::finish(fin, part, gridDim.x);
}

__device__ void bi_res_step(KState *s, const double *part, int parts) {
    if (!s->running || !s->normal) return;
    double v[1];
    sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    const double res = sqrt(v[0]);
    s->res = res;
    if (!isfinite(res)) return stop(s, TF_NONFINITE);
    if (res <= s->tol || s->it % s->interval == 0) s->refresh = 1;
}

__global__ void bi_end(KState *s, const double *part, int parts) {
    pdl_enter();
    if (!s->running) return;
    double v[1];
    const bool refresh = s->normal && s->refresh;
    if (refresh) sum_partials<1>(part, parts, v);
    if (threadIdx.x) return;
    if (refresh) {
        s->refresh = 0;
        const double res = sqrt(v[0]);
        s->res = res;
        if (res <= s->tol || !isfinite(res)) return stop(s, TF_MAX_ITERATIONS);
        s->copy_shadow = 1;
        s->fresh = 1;
    }
    if (s->normal) s->rho_prev = s->rho;
    if (s->it >= s->max_it) stop(s, TF_MAX_ITERATIONS);
}

TF_KRYLOV_FINAL(BiRho, bi_rho_step)
TF_KRYLOV_FINAL(BiAlpha, bi_alpha_step)
TF_KRYLOV_FINAL(BiSnorm, bi_snorm_step)
TF_KRYLOV_FINAL(BiEarly, bi_early_step)
TF_KRYLOV_FINAL(BiOmega, bi_omega_step)
TF_KRYLOV_FINAL(BiRes, bi_res_step)
#undef TF_KRYLOV_FINAL

// ---- solver object --------------------------------------------------------

template <class T, class I>
class KrylovImpl final : public Krylov {
  public:
    KrylovImpl(int kind, const tf_solver_options &opt, int precond, const tf_amg_options *amg)
        : kind_(kind), opt_(opt), precond_(precond) {
        validate_solver_options(opt);
        if (precond == TF_PRECOND_AMG) {
            require(amg != nullptr, "AMG options required");
            amg_cfg_ = std::make_unique<AmgConfig>(*amg);
        } else {
            require(precond == TF_PRECOND_IDENTITY, "unknown preconditioner");
        }
    }
    ~KrylovImpl() override {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (solve_exec_) cudaGraphExecDestroy(solve_exec_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
    }

    void setup(tf_ctx *ctx, const tf_csr &a) override {
        ready_ = false;
        const char *f = std::getenv("THERMOFEM_B200_FUSE");
        const char *fo = std::getenv("THERMOFEM_B200_FUSE_OUTER");
        fuse_ = (f ? std::atoi(f) : 1) != 0 && !(fo && fo[0] == '0') ? 1 : 0;
        if (exec_) {
            cudaGraphExecDestroy(exec_);
            exec_ = nullptr;
        }
        if (solve_exec_) {
            cudaGraphExecDestroy(solve_exec_);
            solve_exec_ = nullptr;
        }
        capture_failed_ = solve_graph_failed_ = false;
        check_csr(&a);
        require(a.rows > 0 && a.rows == a.cols, "Solver requires a nonempty square matrix");
        require(sizeof(T) == type_size(a.value_type) && sizeof(I) == type_size(a.index_type),
                "matrix types differ from the solver's");
        // Snapshot: canonical copy (duplicates summed), finite values.
        std::unique_ptr<tf_dcsr> native;
        try {
            native = to_native(ctx, a);
        } catch (const Failure &f) {
            if (f.code == TF_ERR_INVALID) fail(TF_ERR_INVALID, "Matrix contains nonfinite entries");
            throw;
        }
        n_ = a.rows;
        nnz_ = native->nnz;
        rp_.allocate(static_cast<size_t>(n_) + 1);
        ci_.allocate(static_cast<size_t>(nnz_));
        val_.allocate(static_cast<size_t>(nnz_));
        const auto nc = csr_of(*native);
        convert(ctx, n_ + 1, nc.rp, rp_.data());
        convert(ctx, nnz_, nc.ci, ci_.data());
        convert(ctx, nnz_, nc.val, val_.data());
        cd_.release();
        if (delta_columns_enabled() && nnz_ > 0) {
            cd_.allocate(static_cast<size_t>(nnz_));
            if (!delta_columns(ctx, n_, rp_.data(), ci_.data(), cd_.data())) cd_.release();
        }
        sl_.release();
        if constexpr (std::is_same_v<I, int32_t>) {
            // a banded copy where the operator's slices share their column
            // offsets (stencils), else the 2-byte-offset sliced copy
            if (sliced_enabled() && !(banded_enabled() && build_banded(ctx, csr(), sl_)) && cd_.data())
                build_sliced(ctx, csr(), sl_, false);
        }
        hier_.reset();
        if (precond_ == TF_PRECOND_AMG) {
            const int storage = amg_cfg_->o.hierarchy_type == -1 ? (sizeof(T) == 8 ? TF_F64 : TF_F32)
                                                                 : amg_cfg_->o.hierarchy_type;
            hier_ = build_hierarchy(ctx, *amg_cfg_, storage, *native);
        }
        for (auto *b : {&rhs_, &x_, &r_, &z_, &p_, &q_, &shadow_, &s_, &t_, &sh_})
            b->allocate(static_cast<size_t>(n_));
        tiles_ = tile::partials(n_);
        fill_zero(ctx, n_, x_.data());
        tune_spmv(ctx, csr(), static_cast<const T *>(x_.data()), q_.data());
        parts_ = parts_for(n_);
        part_.allocate(static_cast<size_t>(2 * std::max(tiles_, parts_)));
        partb_.allocate(static_cast<size_t>(std::max(tiles_, parts_)));
        state_.allocate(1);
        if (!ev0_) {
            cuda_check(cudaEventCreate(&ev0_), "event");
            cuda_check(cudaEventCreate(&ev1_), "event");
        }
        cuda_check(cudaStreamSynchronize(ctx->stream), "solver setup");
        ready_ = true;
        ++generation_;
    }

    tf_solve_result solve(tf_ctx *ctx, const void *rhs, void *x) override {
        if (!ready_) fail(TF_ERR_LOGIC, kind_ == TF_SOLVER_CG ? "CG requires setup" : "BiCGStab requires setup");
        StableScope stable(ctx);  // the operator and the hierarchy are read-only during a solve
        cuda_check(cudaEventRecord(ev0_, ctx->stream), "event");
        copy_async(ctx, rhs_.data(), rhs, n_ * sizeof(T));
        copy_async(ctx, x_.data(), x, n_ * sizeof(T));
        const KState init = initial_state();
        cuda_check(cudaMemcpyAsync(state_.data(), &init, sizeof(KState), cudaMemcpyHostToDevice, ctx->stream),
                   "state upload");
        if (graph_mode == 1 && !solve_exec_ && !solve_graph_failed_) build_solve_graph(ctx);
        const bool whole = graph_mode == 1 && solve_exec_;
        if (whole) {
            // the whole solve, loop included, is one graph launch
            cuda_check(cudaGraphLaunch(solve_exec_, ctx->stream), "solve graph");
            last_execution = 2;
        } else {
            enqueue_prefix(ctx);
            int *running = static_cast<int *>(ctx->pinned);
            cuda_check(cudaMemcpyAsync(running, &state_.data()->running, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream),
                       "state readback");
            cuda_check(cudaStreamSynchronize(ctx->stream), "solve init");
            for (int k = 0; k < opt_.max_iterations && *running; ++k) {
                run_iteration(ctx);
                cuda_check(cudaMemcpyAsync(running, &state_.data()->running, sizeof(int), cudaMemcpyDeviceToHost,
                                           ctx->stream),
                           "state readback");
                cuda_check(cudaStreamSynchronize(ctx->stream), "iteration");
            }
            enqueue_suffix(ctx);
        }
        copy_async(ctx, x, x_.data(), n_ * sizeof(T));
        KState fin;
        cuda_check(cudaMemcpyAsync(ctx->pinned, state_.data(), sizeof(KState) <= 256 ? sizeof(KState) : 256,
                                   cudaMemcpyDeviceToHost, ctx->stream),
                   "state readback");
        cuda_check(cudaEventRecord(ev1_, ctx->stream), "event");
        cuda_check(cudaStreamSynchronize(ctx->stream), "solve");
        std::memcpy(&fin, ctx->pinned, sizeof(KState));
        if (whole) ctx->launches += prefix_launches_ + suffix_launches_ + per_iteration_ * fin.it;
        check_faults(ctx);
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0_, ev1_);
        last_ms = ms;
        tf_solve_result out;
        out.status = fin.status;
        out.iterations = fin.it;
        out.residual_norm = fin.res;
        out.relative_residual = fin.normB > 0 ? fin.res / fin.normB : fin.res;
        return out;
    }

    Hierarchy *amg() override { return hier_.get(); }

    // ---- batches: many solvers' whole solves as branches of one graph ----
    void batch_nodes(tf_ctx *ctx, cudaGraph_t g) override {
        if (!ready_) fail(TF_ERR_LOGIC, kind_ == TF_SOLVER_CG ? "CG requires setup" : "BiCGStab requires setup");
        StableScope stable(ctx);
        add_solve_nodes(ctx, g, true);
    }
    int64_t batch_launches(int iterations) const override {
        return prefix_launches_ + suffix_launches_ + per_iteration_ * iterations;
    }
    void batch_stage(tf_ctx *ctx, const void *rhs, const void *x) override {
        copy_async(ctx, rhs_.data(), rhs, n_ * sizeof(T));
        copy_async(ctx, x_.data(), x, n_ * sizeof(T));
    }
    void batch_finish(tf_ctx *ctx, void *x, void *state_host) override {
        copy_async(ctx, x, x_.data(), n_ * sizeof(T));
        cuda_check(cudaMemcpyAsync(state_host, state_.data(), sizeof(KState), cudaMemcpyDeviceToHost, ctx->stream),
                   "state readback");
    }
    size_t state_bytes() const override { return sizeof(KState); }
    tf_solve_result batch_result(const void *state_host) const override {
        KState fin;
        std::memcpy(&fin, state_host, sizeof(KState));
        tf_solve_result out;
        out.status = fin.status;
        out.iterations = fin.it;
        out.residual_norm = fin.res;
        out.relative_residual = fin.normB > 0 ? fin.res / fin.normB : fin.res;
        return out;
    }
    int64_t generation() const override { return generation_; }
    void spmv(tf_ctx *ctx, const void *x, void *y) override {
        if (!ready_) fail(TF_ERR_LOGIC, "solver requires setup");
        StableScope stable(ctx);
        tfb::spmv(ctx, csr(), static_cast<const T *>(x), static_cast<T *>(y));
    }
    int spmv_layout(tf_ctx *ctx, int64_t *entries) const override {
        if (!ready_) fail(TF_ERR_LOGIC, "solver requires setup");
        if (!streams_sliced(ctx, csr(), sl_.entries, entries)) return cd_.data() ? 0 : 4;
        return sl_.banded() ? 3 : 1;
    }
    int64_t rows() const override { return n_; }

  private:
    Csr<T, I> csr() const {
        Csr<T, I> c;
        c.rows = c.cols = n_;
        c.nnz = nnz_;
        c.rp = rp_.data();
        c.ci = ci_.data();
        c.val = val_.data();
        c.cd = cd_.data();
        sl_.attach(c);
        return c;
    }

    // The preconditioner's last conversion fused into the kernel after it
    // (THERMOFEM_B200_FUSE=0 or THERMOFEM_B200_FUSE_OUTER=0 keep them apart;
    // the same bits either way).
    bool fuse_outer() const { return hier_ && fuse_ != 0; }

    // out = M^-1 in, then the operator SpMV of out with epi: the gathers read
    // the preconditioner's output in its own storage and every row also
    // stores its converted value into out.
    template <class Epi>
    void preconditioned_spmv(tf_ctx *ctx, const T *in, T *out, const Epi &epi, const char *name) {
        const void *zs = hier_->apply_open(ctx, in);
        if (hier_->storage_type() == TF_F32)
            tile::launch(ctx, csr(), ConvertX<T, float>{static_cast<const float *>(zs)}, store_own_x(epi, out), name);
        else
            tile::launch(ctx, csr(), ConvertX<T, double>{static_cast<const double *>(zs)}, store_own_x(epi, out),
                         name);
    }

    void precondition(tf_ctx *ctx, const T *in, T *out) {
        if (hier_) hier_->apply(ctx, in, out);
        else copy_async(ctx, out, in, n_ * sizeof(T));
    }

    // ||b||^2, r = b - A x with ||r||^2, initial decisions.
    void enqueue_prefix(tf_ctx *ctx) {
        launch_kernel(ctx, "dot", k_dot<T>, parts_, 256, 0, n_, rhs_.data(), rhs_.data(), partb_.data(),
                      tile::NoFinal{});
        tile::launch(ctx, csr(), tile::PlainX<T>{x_.data()},
                     ResidualNorm<T>{rhs_.data(), r_.data(), nullptr, part_.data()}, "residual_norm");
        launch_kernel(ctx, "k_init", k_init, 1, 1024, 0, state_.data(), partb_.data(), parts_, part_.data(), tiles_,
                      kind_ == TF_SOLVER_BICGSTAB ? 1 : 0);
        if (kind_ == TF_SOLVER_BICGSTAB) {
            launch_kernel(ctx, "copy_if", k_copy_if<T>, parts_, 256, 0, &state_.data()->copy_shadow, n_, r_.data(),
                          shadow_.data());
        }
    }

    // Final true residual and report.
    void enqueue_suffix(tf_ctx *ctx) {
        tile::launch(ctx, csr(), tile::PlainX<T>{x_.data()},
                     ResidualNorm<T>{rhs_.data(), r_.data(), nullptr, part_.data()}, "residual_norm");
        launch_kernel(ctx, "k_finish", k_finish, 1, 1024, 0, state_.data(), part_.data(), tiles_);
    }

    // One graph for the whole solve: prefix, then a conditional WHILE node
    // whose body is one iteration (it re-arms the condition from the device
    // state at its end), then the suffix.  Falls back to the host loop when
    // the driver refuses any step.
    // Adds the whole solve to graph g as one independent branch: (with
    // reset, a kernel that loads the initial state) prefix, a conditional
    // WHILE node whose body is one iteration (it re-arms the condition from
    // the device state at its end), suffix.  Throws when CUDA refuses a
    // step; the caller ends any capture left open.
    void add_solve_nodes(tf_ctx *ctx, cudaGraph_t g, bool reset) {
        const int64_t before = ctx->launches;
        cudaGraphConditionalHandle handle;
        cuda_check(cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault), "condition");
        cuda_check(cudaStreamBeginCaptureToGraph(ctx->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                   "capture prefix");
        if (reset) launch_kernel(ctx, "k_reset", k_reset, 1, 1, 0, state_.data(), initial_state());
        enqueue_prefix(ctx);
        launch_kernel(ctx, "set_continue", k_set_continue, 1, 1, 0, handle, state_.data());
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        cuda_check(cudaStreamGetCaptureInfo(ctx->stream, &st, nullptr, nullptr, &deps, &ndeps), "capture info");
        std::vector<cudaGraphNode_t> last(deps, deps + ndeps);
        cudaGraph_t out = nullptr;
        cuda_check(cudaStreamEndCapture(ctx->stream, &out), "capture prefix end");
        prefix_launches_ = ctx->launches - before;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        cuda_check(cudaGraphAddNode(&loop, g, last.data(), last.size(), &cp), "while node");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        const int64_t b0 = ctx->launches;
        cuda_check(cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal),
                   "capture body");
        enqueue_iteration(ctx);
        launch_kernel(ctx, "set_continue", k_set_continue, 1, 1, 0, handle, state_.data());
        cuda_check(cudaStreamEndCapture(ctx->stream, &out), "capture body end");
        per_iteration_ = ctx->launches - b0;
        const int64_t s0 = ctx->launches;
        cuda_check(cudaStreamBeginCaptureToGraph(ctx->stream, g, &loop, nullptr, 1, cudaStreamCaptureModeThreadLocal),
                   "capture suffix");
        enqueue_suffix(ctx);
        cuda_check(cudaStreamEndCapture(ctx->stream, &out), "capture suffix end");
        suffix_launches_ = ctx->launches - s0;
        ctx->launches = before;
    }

    void build_solve_graph(tf_ctx *ctx) {
        cudaGraph_t g = nullptr;
        try {
            cuda_check(cudaGraphCreate(&g, 0), "graph create");
            add_solve_nodes(ctx, g, false);
            cuda_check(cudaGraphInstantiate(&solve_exec_, g, 0), "solve graph instantiate");
        } catch (const Failure &) {
            end_open_capture(ctx);
            solve_exec_ = nullptr;
            solve_graph_failed_ = true;
        }
        if (g) cudaGraphDestroy(g);
    }

    static void end_open_capture(tf_ctx *ctx) { end_capture_into_graph(ctx); }

    KState initial_state() const {
        KState init{};
        init.tol = opt_.absolute_tolerance;
        init.res = opt_.relative_tolerance;
        init.max_it = opt_.max_iterations;
        init.interval = opt_.residual_refresh_interval;
        init.status = TF_MAX_ITERATIONS;
        return init;
    }

    void run_iteration(tf_ctx *ctx) {
        if (!exec_ && !capture_failed_) {
            if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const int64_t before = ctx->launches;
                cudaGraph_t g = nullptr;
                try {
                    enqueue_iteration(ctx);
                } catch (const Failure &) {
                    // a step the driver cannot capture: run uncaptured from now on
                    cudaStreamEndCapture(ctx->stream, &g);
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    ctx->launches = before;
                    capture_failed_ = true;
                    enqueue_iteration(ctx);
                    return;
                }
                per_iteration_ = ctx->launches - before;
                ctx->launches = before;
                cuda_check(cudaStreamEndCapture(ctx->stream, &g), "iteration capture");
                if (cudaGraphInstantiate(&exec_, g, 0) != cudaSuccess) {
                    cudaGetLastError();
                    exec_ = nullptr;
                    capture_failed_ = true;
                }
                cudaGraphDestroy(g);
            } else {
                cudaGetLastError();
                capture_failed_ = true;
            }
        }
        if (exec_) {
            cuda_check(cudaGraphLaunch(exec_, ctx->stream), "iteration graph");
            ctx->launches += per_iteration_;
            last_execution = 1;
        } else {
            enqueue_iteration(ctx);
            last_execution = 0;
        }
    }

    void enqueue_iteration(tf_ctx *ctx) {
        KState *s = state_.data();
        double *part = part_.data();
        unsigned *tk = s->tickets;
        const unsigned pg = static_cast<unsigned>(parts_);
        if (kind_ == TF_SOLVER_CG) {
            if (fuse_outer()) {
                // z = M^-1 r stays in the hierarchy's finest level (its
                // storage): the dot and the direction update read it there
                const void *zs = hier_->apply_open(ctx, static_cast<const T *>(r_.data()));
                if (hier_->storage_type() == TF_F32) {
                    launch_kernel(ctx, "dot_rho_from", k_dot_from<T, float, CgRho>, pg, 256, 0, n_, r_.data(),
                                  static_cast<const float *>(zs), static_cast<T *>(nullptr), part, CgRho{s, tk + 0});
                    launch_kernel(ctx, "cg_p", cg_p<T, float>, pg, 256, 0, s, n_, static_cast<const float *>(zs),
                                  p_.data());
                } else {
                    launch_kernel(ctx, "dot_rho_from", k_dot_from<T, double, CgRho>, pg, 256, 0, n_, r_.data(),
                                  static_cast<const double *>(zs), static_cast<T *>(nullptr), part, CgRho{s, tk + 0});
                    launch_kernel(ctx, "cg_p", cg_p<T, double>, pg, 256, 0, s, n_, static_cast<const double *>(zs),
                                  p_.data());
                }
            } else {
                precondition(ctx, r_.data(), z_.data());
                launch_kernel(ctx, "dot_rho", k_dot<T, CgRho>, pg, 256, 0, n_, r_.data(), z_.data(), part,
                              CgRho{s, tk + 0});
                launch_kernel(ctx, "cg_p", cg_p<T>, pg, 256, 0, s, n_, z_.data(), p_.data());
            }
            tile::launch(ctx, csr(), tile::PlainX<T>{p_.data()},
                         SpmvDot<T, CgCurv>{q_.data(), p_.data(), &s->running, part, CgCurv{s, tk + 1}},
                         "spmv_dot_curv");
            launch_kernel(ctx, "cg_xr_res", cg_xr<T, CgRes>, pg, 256, 0, s, n_, p_.data(), q_.data(), x_.data(),
                          r_.data(), part, CgRes{s, tk + 2});
            tile::launch(ctx, csr(), tile::PlainX<T>{x_.data()},
                         ResidualNorm<T, CgRefresh>{rhs_.data(), r_.data(), &s->refresh, part, CgRefresh{s, tk + 3}},
                         "residual_refresh");
            return;
        }
        // BiCGStab: v = q_, phat = z_
        launch_kernel(ctx, "dot_rho", k_dot<T, BiRho>, pg, 256, 0, n_, shadow_.data(), r_.data(), part,
                      BiRho{s, tk + 0});
        launch_kernel(ctx, "bi_p", bi_p<T>, pg, 256, 0, s, n_, r_.data(), q_.data(), p_.data());
        const SpmvDot<T, BiAlpha> alpha_epi{q_.data(), shadow_.data(), &s->running, part, BiAlpha{s, tk + 1}};
        if (fuse_outer())
            preconditioned_spmv(ctx, p_.data(), z_.data(), alpha_epi, "spmv_dot_alpha_from");
        else {
            precondition(ctx, p_.data(), z_.data());
            tile::launch(ctx, csr(), tile::PlainX<T>{z_.data()}, alpha_epi, "spmv_dot_alpha");
        }
        launch_kernel(ctx, "bi_s_norm", bi_s<T, BiSnorm>, pg, 256, 0, s, n_, r_.data(), q_.data(), z_.data(),
                      s_.data(), x_.data(), part, BiSnorm{s, tk + 2});
        tile::launch(ctx, csr(), tile::PlainX<T>{x_.data()},
                     ResidualNorm<T, BiEarly>{rhs_.data(), r_.data(), &s->early, part, BiEarly{s, tk + 3}},
                     "residual_early");
        const SpmvDot2<T, BiOmega> omega_epi{t_.data(), s_.data(), &s->normal, part, BiOmega{s, tk + 4}};
        if (fuse_outer())
            preconditioned_spmv(ctx, s_.data(), sh_.data(), omega_epi, "spmv_dot2_omega_from");
        else {
            precondition(ctx, s_.data(), sh_.data());
            tile::launch(ctx, csr(), tile::PlainX<T>{sh_.data()}, omega_epi, "spmv_dot2_omega");
        }
        launch_kernel(ctx, "bi_xr_res", bi_xr<T, BiRes>, pg, 256, 0, s, n_, sh_.data(), s_.data(), t_.data(),
                      x_.data(), r_.data(), part, BiRes{s, tk + 5});
        tile::launch(ctx, csr(), tile::PlainX<T>{x_.data()}, ResidualNorm<T>{rhs_.data(), r_.data(), &s->refresh, part},
                     "residual_norm");
        launch_kernel(ctx, "bi_end", bi_end, 1, 1024, 0, s, part, tiles_);
        launch_kernel(ctx, "copy_if", k_copy_if<T>, pg, 256, 0, &s->copy_shadow, n_, r_.data(), shadow_.data());
    }

    int kind_;
    int fuse_{1};
    tf_solver_options opt_;
    int precond_;
    std::unique_ptr<AmgConfig> amg_cfg_;
    std::unique_ptr<Hierarchy> hier_;
    bool ready_{false};
    int64_t n_{0}, nnz_{0};
    DeviceBuffer<I> rp_, ci_;
    DeviceBuffer<int16_t> cd_;  // columns as row offsets, when they fit
    SlicedCopy<T> sl_;          // sliced copy for the SpMV family, when built
    DeviceBuffer<T> val_;
    DeviceBuffer<T> rhs_, x_, r_, z_, p_, q_, shadow_, s_, t_, sh_;
    DeviceBuffer<double> part_, partb_;
    DeviceBuffer<KState> state_;
    int tiles_{1}, parts_{1};
    cudaGraphExec_t exec_{nullptr};
    cudaGraphExec_t solve_exec_{nullptr};
    bool solve_graph_failed_{false};
    int64_t prefix_launches_{0}, suffix_launches_{0};
    int64_t generation_{0};
    bool capture_failed_{false};
    int64_t per_iteration_{0};
    cudaEvent_t ev0_{nullptr}, ev1_{nullptr};
};

}  // namespace

void validate_solver_options(const tf_solver_options &o) {
    if (o.max_iterations < 0 || o.residual_refresh_interval < 1 || !std::isfinite(o.relative_tolerance) ||
        o.relative_tolerance < 0 || o.relative_tolerance >= 1 || !std::isfinite(o.absolute_tolerance) ||
        o.absolute_tolerance < 0)
        fail(TF_ERR_INVALID, "Invalid solver options");
}

std::unique_ptr<Krylov> make_krylov(int kind, int value_type, int index_type, const tf_solver_options &opt,
                                    int precond, const tf_amg_options *amg_opt) {
    require(kind == TF_SOLVER_CG || kind == TF_SOLVER_BICGSTAB, "unknown solver kind");
    if (value_type == TF_F64 && index_type == TF_I32)
        return std::make_unique<KrylovImpl<double, int32_t>>(kind, opt, precond, amg_opt);
    if (value_type == TF_F64 && index_type == TF_I64)
        return std::make_unique<KrylovImpl<double, int64_t>>(kind, opt, precond, amg_opt);
    if (value_type == TF_F32 && index_type == TF_I32)
        return std::make_unique<KrylovImpl<float, int32_t>>(kind, opt, precond, amg_opt);
    if (value_type == TF_F32 && index_type == TF_I64)
        return std::make_unique<KrylovImpl<float, int64_t>>(kind, opt, precond, amg_opt);
    fail(TF_ERR_INVALID, "unsupported solver types");
}

}  // namespace tfb
