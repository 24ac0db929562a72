// mlp.cu -- learned per-row Jacobi damping: row features, a 2-layer MLP
// (4 -> 32 -> 1, BF16 weights, FP32 accumulation) with hand-written forward,
// backward and SGD kernels, and its use by the AMG setup.
//
// The network maps the features of a row of a level operator
//   x0 = log(|a_ii| / mean |a_jj| of the level), x1 = sum_j!=i |a_ij| / |a_ii|,
//   x2 = row nonzeros / 8, x3 = level index / 10
// to a damping factor omega_i = lo + (hi - lo) * sigmoid(z),
//   z = w2 . relu(W1 x + b1) + b2.
// Training minimises the mean squared error to per-row targets (the damping
// that the solver measured to reduce the error of that row most); the
// gradient of a batch is reduced in a fixed order (per warp, per CTA, over
// CTAs), so it does not depend on the GPU.  The master weights are FP32; the
// forward and backward passes use their BF16 rounding, as inference does.
// A hierarchy built with a model multiplies each level's inverse diagonal by
// omega_i and sweeps with weight 1 (fixed-omega Jacobi is the fallback).
#include <cmath>
#include <cstring>
#include <vector>

#include "mlp.cuh"

namespace tfb {
namespace {

constexpr int kF = TF_MLP_FEATURES, kH = TF_MLP_HIDDEN, kP = TF_MLP_PARAMS;
constexpr int kGradSlots = kP + 1;  // gradient sums and the loss sum
constexpr int kMlpBlock = 256;
constexpr int kMaxGrid = 1184;

// Parameter layout: W1[kH][kF], b1[kH], w2[kH], b2.
constexpr int kW1 = 0, kB1 = kH * kF, kW2 = kB1 + kH, kB2 = kW2 + kH;

__device__ __forceinline__ float bf16_to_float(uint16_t b) { return __uint_as_float(static_cast<uint32_t>(b) << 16); }

uint16_t float_to_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t lsb = (u >> 16) & 1u;  // round to nearest, ties to even
    u += 0x7fffu + lsb;
    return static_cast<uint16_t>(u >> 16);
}

__device__ __forceinline__ void load_params(const uint16_t *bf, float *sp) {
    for (int k = threadIdx.x; k < kP; k += blockDim.x) sp[k] = bf16_to_float(bf[k]);
    __syncthreads();
}

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

template <class T, class I>
__global__ void abs_diag_kernel(int64_t n, const I *__restrict__ rp, const I *__restrict__ ci,
                                const T *__restrict__ val, double *part) {
    pdl_enter();
    double s = 0.0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double d = 0.0;
        for (I j = rp[i]; j < rp[i + 1]; ++j)
            if (static_cast<int64_t>(ci[j]) == i) d += static_cast<double>(val[j]);
        s += fabs(d);
    }
    double v[1] = {s};
    tile::block_reduce<1>(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

template <class T, class I>
__global__ void features_kernel(int64_t n, const I *__restrict__ rp, const I *__restrict__ ci,
                                const T *__restrict__ val, int level, double mean_diag, float *__restrict__ out) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double d = 0.0, off = 0.0;
        for (I j = rp[i]; j < rp[i + 1]; ++j) {
            const double v = static_cast<double>(val[j]);
            if (static_cast<int64_t>(ci[j]) == i) d += v;
            else off += fabs(v);
        }
        const double ad = fabs(d);
        float *f = out + i * kF;
        f[0] = ad > 0 && mean_diag > 0 ? static_cast<float>(log(ad / mean_diag)) : 0.0f;
        f[1] = ad > 0 ? static_cast<float>(off / ad) : 0.0f;
        f[2] = static_cast<float>(rp[i + 1] - rp[i]) * 0.125f;
        f[3] = static_cast<float>(level) * 0.1f;
    }
}

__global__ void forward_kernel(int64_t n, const float *__restrict__ x, const uint16_t *__restrict__ bf, float lo,
                               float hi, float *__restrict__ omega) {
    pdl_enter();
    __shared__ float sp[kP];
    load_params(bf, sp);
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float *f = x + i * kF;
        const float x0 = f[0], x1 = f[1], x2 = f[2], x3 = f[3];
        float z = sp[kB2];
#pragma unroll 8
        for (int j = 0; j < kH; ++j) {
            const float *w = sp + kW1 + j * kF;
            const float a = sp[kB1 + j] + w[0] * x0 + w[1] * x1 + w[2] * x2 + w[3] * x3;
            z += sp[kW2 + j] * fmaxf(a, 0.0f);
        }
        omega[i] = lo + (hi - lo) * sigmoid(z);
    }
}

// Per-CTA sums of the gradient of sum_i (omega_i - t_i)^2 and of the loss:
// each warp reduces its 32 rows per parameter with shuffles, lane 0 adds the
// warp sum to its slot, and the slots are added in warp order.
__global__ void __launch_bounds__(kMlpBlock) backward_kernel(int64_t n, const float *__restrict__ x,
                                                             const float *__restrict__ target,
                                                             const uint16_t *__restrict__ bf, float lo, float hi,
                                                             double *__restrict__ partial) {
    pdl_enter();
    __shared__ float sp[kP];
    __shared__ double slot[kMlpBlock / 32][kGradSlots];
    load_params(bf, sp);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = lane; k < kGradSlots; k += 32) slot[warp][k] = 0.0;
    __syncwarp();
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t base = blockIdx.x * static_cast<int64_t>(blockDim.x) + warp * 32; base < n; base += stride) {
        const int64_t i = base + lane;
        const bool on = i < n;
        float xv[kF] = {0.f, 0.f, 0.f, 0.f};
        float t = 0.f;
        if (on) {
            for (int k = 0; k < kF; ++k) xv[k] = x[i * kF + k];
            t = target[i];
        }
        float a[kH];
        float z = sp[kB2];
#pragma unroll
        for (int j = 0; j < kH; ++j) {
            const float *w = sp + kW1 + j * kF;
            a[j] = sp[kB1 + j] + w[0] * xv[0] + w[1] * xv[1] + w[2] * xv[2] + w[3] * xv[3];
            z += sp[kW2 + j] * fmaxf(a[j], 0.0f);
        }
        const float s = sigmoid(z);
        const float om = lo + (hi - lo) * s;
        const float e = on ? om - t : 0.0f;
        const float dz = 2.0f * e * (hi - lo) * s * (1.0f - s);
        auto add = [&](int k, float g) {
            for (int o = 16; o > 0; o >>= 1) g += __shfl_down_sync(0xffffffffu, g, o);
            if (lane == 0) slot[warp][k] += static_cast<double>(g);
        };
        add(kP, e * e);
        add(kB2, dz);
#pragma unroll
        for (int j = 0; j < kH; ++j) {
            const float h = fmaxf(a[j], 0.0f);
            add(kW2 + j, dz * h);
            const float dh = a[j] > 0.0f ? dz * sp[kW2 + j] : 0.0f;
            add(kB1 + j, dh);
#pragma unroll
            for (int k = 0; k < kF; ++k) add(kW1 + j * kF + k, dh * xv[k]);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kGradSlots; k += blockDim.x) {
        double v = 0.0;
        for (int w = 0; w < kMlpBlock / 32; ++w) v += slot[w][k];
        partial[static_cast<int64_t>(blockIdx.x) * kGradSlots + k] = v;
    }
}

// grad[k] += sum over CTAs of partial[cta][k], in CTA order.
__global__ void gradient_sum_kernel(int parts, const double *__restrict__ partial, double *__restrict__ grad) {
    pdl_enter();
    for (int k = threadIdx.x; k < kGradSlots; k += blockDim.x) {
        double v = 0.0;
        for (int c = 0; c < parts; ++c) v += partial[static_cast<int64_t>(c) * kGradSlots + k];
        grad[k] += v;
    }
}

// Momentum SGD on the FP32 master weights with the mean gradient of the
// rows accumulated since the last step; refreshes the BF16 copy and clears
// the accumulator.
__global__ void sgd_kernel(float *__restrict__ p, float *__restrict__ vel, double *__restrict__ grad, double rows,
                           float lr, float momentum, uint16_t *__restrict__ bf) {
    pdl_enter();
    for (int k = threadIdx.x; k < kP; k += blockDim.x) {
        const float g = static_cast<float>(grad[k] / rows);
        const float v = momentum * vel[k] + g;
        vel[k] = v;
        const float w = p[k] - lr * v;
        p[k] = w;
        uint32_t u = __float_as_uint(w);
        u += 0x7fffu + ((u >> 16) & 1u);
        bf[k] = static_cast<uint16_t>(u >> 16);
        grad[k] = 0.0;
    }
    if (threadIdx.x == 0) grad[kP] = 0.0;
}

template <class T>
__global__ void scale_kernel(int64_t n, const float *__restrict__ omega, T *__restrict__ dinv) {
    pdl_enter();
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        dinv[i] = static_cast<T>(omega[i]) * dinv[i];
}

unsigned grid_rows(int64_t n) {
    int64_t g = (n + kMlpBlock - 1) / kMlpBlock;
    if (g < 1) g = 1;
    if (g > kMaxGrid) g = kMaxGrid;
    return static_cast<unsigned>(g);
}

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

}  // namespace

std::vector<float> mlp_initial_params(uint64_t seed, double lo, double hi, double start) {
    std::vector<float> p(kP, 0.0f);
    uint64_t s = seed;
    auto uni = [&] { return static_cast<double>(splitmix(s) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0; };
    const double a1 = std::sqrt(6.0 / (kF + kH)), a2 = std::sqrt(6.0 / (kH + 1));
    for (int k = 0; k < kH * kF; ++k) p[kW1 + k] = static_cast<float>(a1 * uni());
    for (int j = 0; j < kH; ++j) p[kW2 + j] = static_cast<float>(0.01 * a2 * uni());
    // the output starts near `start` everywhere (the fixed-omega method)
    const double q = (start - lo) / (hi - lo);
    p[kB2] = static_cast<float>(std::log(q / (1.0 - q)));
    return p;
}

std::vector<uint16_t> mlp_bf16(const std::vector<float> &p) {
    std::vector<uint16_t> b(p.size());
    for (size_t k = 0; k < p.size(); ++k) b[k] = float_to_bf16(p[k]);
    return b;
}

template <class T, class I>
void row_features(tf_ctx *ctx, const Csr<T, I> &a, int level, float *out) {
    require(a.rows > 0 && a.rows == a.cols, "row features need a nonempty square matrix");
    require(level >= 0, "level must be non-negative");
    const unsigned g = grid_rows(a.rows);
    double *part = static_cast<double *>(ctx->arena(sizeof(double) * g, 1));
    launch_kernel(ctx, "abs_diag", abs_diag_kernel<T, I>, g, kMlpBlock, 0, a.rows, a.rp, a.ci, a.val, part);
    std::vector<double> h(g);
    cuda_check(cudaMemcpyAsync(h.data(), part, sizeof(double) * g, cudaMemcpyDeviceToHost, ctx->stream),
               "diagonal readback");
    cuda_check(cudaStreamSynchronize(ctx->stream), "diagonal readback");
    double s = 0.0;
    for (double v : h) s += v;
    launch_kernel(ctx, "row_features", features_kernel<T, I>, g, kMlpBlock, 0, a.rows, a.rp, a.ci, a.val, level,
                  s / static_cast<double>(a.rows), out);
}

void mlp_forward(tf_ctx *ctx, const uint16_t *bf16, float lo, float hi, int64_t n, const float *features,
                 float *omega) {
    if (n <= 0) return;
    launch_kernel(ctx, "mlp_forward", forward_kernel, grid_rows(n), kMlpBlock, 0, n, features, bf16, lo, hi, omega);
}

template <class T, class I>
void learned_damping(tf_ctx *ctx, const DampingModel &m, const Csr<T, I> &a, int level, T *dinv) {
    DeviceBuffer<uint16_t> bf(static_cast<size_t>(kP));
    cuda_check(cudaMemcpyAsync(bf.data(), m.bf16.data(), kP * sizeof(uint16_t), cudaMemcpyHostToDevice, ctx->stream),
               "model upload");
    DeviceBuffer<float> feat(static_cast<size_t>(a.rows) * kF), omega(static_cast<size_t>(a.rows));
    row_features(ctx, a, level, feat.data());
    mlp_forward(ctx, bf.data(), m.omega_min, m.omega_max, a.rows, feat.data(), omega.data());
    launch_kernel(ctx, "damping_scale", scale_kernel<T>, grid_rows(a.rows), kMlpBlock, 0, a.rows,
                  static_cast<const float *>(omega.data()), dinv);
    cuda_check(cudaStreamSynchronize(ctx->stream), "learned damping");
}

#define TF_MLP_INST(T, I)                                                                            \
    template void row_features<T, I>(tf_ctx *, const Csr<T, I> &, int, float *);                    \
    template void learned_damping<T, I>(tf_ctx *, const DampingModel &, const Csr<T, I> &, int, T *);
TF_MLP_INST(float, int32_t)
TF_MLP_INST(double, int32_t)
TF_MLP_INST(float, int64_t)
TF_MLP_INST(double, int64_t)
#undef TF_MLP_INST

}  // namespace tfb

// ---- C ABI ------------------------------------------------------------------

struct tf_mlp {
    tf_ctx *ctx{nullptr};
    float omega_min{0}, omega_max{0};
    tfb::DeviceBuffer<float> params, velocity;
    tfb::DeviceBuffer<uint16_t> bf16;
    tfb::DeviceBuffer<double> grad, partial;
    double rows{0};  // rows accumulated in grad since the last step
};

using namespace tfb;

namespace {

void upload(tf_mlp *m, const std::vector<float> &p) {
    const std::vector<uint16_t> b = mlp_bf16(p);
    cuda_check(cudaMemcpyAsync(m->params.data(), p.data(), kP * sizeof(float), cudaMemcpyHostToDevice,
                               m->ctx->stream),
               "params upload");
    cuda_check(cudaMemcpyAsync(m->bf16.data(), b.data(), kP * sizeof(uint16_t), cudaMemcpyHostToDevice,
                               m->ctx->stream),
               "params upload");
    cuda_check(cudaStreamSynchronize(m->ctx->stream), "params upload");
}

void check_mlp(const tf_mlp *m) { require(m != nullptr, "null model"); }

}  // namespace

extern "C" {

int tf_mlp_create(tf_ctx *ctx, uint64_t seed, double omega_min, double omega_max, tf_mlp **out) {
    return guard([&] {
        require(out != nullptr, "null argument");
        *out = nullptr;
        check_ctx(ctx);
        require(std::isfinite(omega_min) && std::isfinite(omega_max) && omega_min > 0 && omega_min < omega_max &&
                    omega_max <= 2.0,
                "damping bounds must satisfy 0 < omega_min < omega_max <= 2");
        DeviceScope scope(ctx->device);
        auto m = std::make_unique<tf_mlp>();
        m->ctx = ctx;
        m->omega_min = static_cast<float>(omega_min);
        m->omega_max = static_cast<float>(omega_max);
        m->params.allocate(kP);
        m->velocity.allocate(kP);
        m->bf16.allocate(kP);
        m->grad.allocate(kGradSlots);
        m->partial.allocate(static_cast<size_t>(kMaxGrid) * kGradSlots);
        memset_async(ctx, m->velocity.data(), 0, kP * sizeof(float));
        memset_async(ctx, m->grad.data(), 0, kGradSlots * sizeof(double));
        const double start = std::min(std::max(2.0 / 3.0, omega_min + 0.01 * (omega_max - omega_min)),
                                      omega_max - 0.01 * (omega_max - omega_min));
        upload(m.get(), mlp_initial_params(seed, omega_min, omega_max, start));
        *out = m.release();
    });
}

int tf_mlp_destroy(tf_mlp *m) {
    return guard([&] {
        if (!m) return;
        DeviceScope scope(m->ctx->device);
        delete m;
    });
}

int tf_mlp_get_params(const tf_mlp *m, float *host) {
    return guard([&] {
        check_mlp(m);
        require(host != nullptr, "null argument");
        DeviceScope scope(m->ctx->device);
        cuda_check(cudaMemcpyAsync(host, m->params.data(), kP * sizeof(float), cudaMemcpyDeviceToHost, m->ctx->stream),
                   "params readback");
        cuda_check(cudaStreamSynchronize(m->ctx->stream), "params readback");
    });
}

int tf_mlp_set_params(tf_mlp *m, const float *host) {
    return guard([&] {
        check_mlp(m);
        require(host != nullptr, "null argument");
        DeviceScope scope(m->ctx->device);
        std::vector<float> p(host, host + kP);
        for (float v : p) require(std::isfinite(v), "parameters must be finite");
        upload(m, p);
        memset_async(m->ctx, m->velocity.data(), 0, kP * sizeof(float));
    });
}

int tf_mlp_bounds(const tf_mlp *m, double *omega_min, double *omega_max) {
    return guard([&] {
        check_mlp(m);
        if (omega_min) *omega_min = m->omega_min;
        if (omega_max) *omega_max = m->omega_max;
    });
}

int tf_row_features(tf_ctx *ctx, const tf_csr *a, int level, float *features) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        require(features != nullptr, "null features");
        DeviceScope scope(ctx->device);
        if (a->value_type == TF_F64) {
            if (a->index_type == TF_I32) row_features(ctx, csr_of<double, int32_t>(*a), level, features);
            else row_features(ctx, csr_of<double, int64_t>(*a), level, features);
        } else {
            if (a->index_type == TF_I32) row_features(ctx, csr_of<float, int32_t>(*a), level, features);
            else row_features(ctx, csr_of<float, int64_t>(*a), level, features);
        }
    });
}

int tf_mlp_forward(tf_mlp *m, int64_t n, const float *features, float *omega) {
    return guard([&] {
        check_mlp(m);
        require(n >= 0 && (n == 0 || (features && omega)), "null argument");
        DeviceScope scope(m->ctx->device);
        mlp_forward(m->ctx, m->bf16.data(), m->omega_min, m->omega_max, n, features, omega);
    });
}

int tf_mlp_backward(tf_mlp *m, int64_t n, const float *features, const float *target, double *loss) {
    return guard([&] {
        check_mlp(m);
        require(n >= 1 && features && target, "null argument or empty batch");
        DeviceScope scope(m->ctx->device);
        tf_ctx *ctx = m->ctx;
        const unsigned g = grid_rows(n);
        const double before = loss ? read_scalar(ctx, m->grad.data() + kP) : 0.0;
        launch_kernel(ctx, "mlp_backward", backward_kernel, g, kMlpBlock, 0, n, features, target,
                      static_cast<const uint16_t *>(m->bf16.data()), m->omega_min, m->omega_max, m->partial.data());
        launch_kernel(ctx, "mlp_gradient_sum", gradient_sum_kernel, 1, kMlpBlock, 0, static_cast<int>(g),
                      static_cast<const double *>(m->partial.data()), m->grad.data());
        m->rows += static_cast<double>(n);
        if (loss) *loss = (read_scalar(ctx, m->grad.data() + kP) - before) / static_cast<double>(n);
    });
}

int tf_mlp_get_gradient(const tf_mlp *m, double *host) {
    return guard([&] {
        check_mlp(m);
        require(host != nullptr, "null argument");
        DeviceScope scope(m->ctx->device);
        cuda_check(cudaMemcpyAsync(host, m->grad.data(), kP * sizeof(double), cudaMemcpyDeviceToHost, m->ctx->stream),
                   "gradient readback");
        cuda_check(cudaStreamSynchronize(m->ctx->stream), "gradient readback");
    });
}

int tf_mlp_sgd(tf_mlp *m, double lr, double momentum) {
    return guard([&] {
        check_mlp(m);
        require(std::isfinite(lr) && lr > 0 && momentum >= 0 && momentum < 1, "lr > 0 and 0 <= momentum < 1");
        require(m->rows > 0, "no gradient accumulated");
        DeviceScope scope(m->ctx->device);
        launch_kernel(m->ctx, "mlp_sgd", sgd_kernel, 1, kMlpBlock, 0, m->params.data(), m->velocity.data(),
                      m->grad.data(), m->rows, static_cast<float>(lr), static_cast<float>(momentum), m->bf16.data());
        m->rows = 0;
        cuda_check(cudaStreamSynchronize(m->ctx->stream), "sgd");
    });
}

}  // extern "C"

namespace tfb {

std::shared_ptr<const DampingModel> damping_model_of(const tf_mlp *m) {
    if (!m) return nullptr;
    float host[kP];
    DeviceScope scope(m->ctx->device);
    cuda_check(cudaMemcpyAsync(host, m->params.data(), kP * sizeof(float), cudaMemcpyDeviceToHost, m->ctx->stream),
               "model readback");
    cuda_check(cudaStreamSynchronize(m->ctx->stream), "model readback");
    auto d = std::make_shared<DampingModel>();
    d->bf16 = mlp_bf16(std::vector<float>(host, host + kP));
    d->omega_min = m->omega_min;
    d->omega_max = m->omega_max;
    return d;
}

}  // namespace tfb
