// capi.cu -- extern "C" entry points of the kernel layer (thermofem_b200.h).
// Each validates its POD arguments, dispatches on element types and calls
// the typed entry points of ops.cuh on the context's stream.
#include "ops.cuh"

#include <cstdio>
#include <cstdlib>
#include <initializer_list>

namespace tfb {

namespace {
thread_local std::string g_last_error;
thread_local int g_last_cuda = 0;
}

void set_last_error(const char *msg, int cuda) {
    g_last_error = msg ? msg : "";
    g_last_cuda = cuda;
}


namespace {

template <class F>
void with_csr_types(const tf_csr *a, F &&f) {
    check_csr(a);
    if (a->value_type == TF_F64) {
        if (a->index_type == TF_I32) f(double{}, int32_t{});
        else f(double{}, int64_t{});
    } else {
        if (a->index_type == TF_I32) f(float{}, int32_t{});
        else f(float{}, int64_t{});
    }
}

template <class F>
void with_value_type(int t, F &&f) {
    if (t == TF_F64) f(double{});
    else if (t == TF_F32) f(float{});
    else fail(TF_ERR_INVALID, "value type must be TF_F32 or TF_F64");
}

// Device vector arguments: a length that is not negative, and pointers that
// are not NULL unless the vectors are empty (a NULL vector would otherwise
// reach a kernel as an invalid address).
void require_vectors(int64_t n, std::initializer_list<const void *> vectors, const char *what) {
    require(n >= 0, what);
    if (n > 0)
        for (const void *v : vectors) require(v != nullptr, what);
}

// The device check of a CSR's structure (row offsets from 0 to nnz, never
// decreasing; columns in [0, cols)).
void validate_structure(tf_ctx *ctx, const tf_csr *a) {
    const bool ok = a->index_type == TF_I32
                        ? csr_structure_ok(ctx, a->rows, a->cols, a->nnz, static_cast<const int32_t *>(a->offsets),
                                           static_cast<const int32_t *>(a->indices))
                        : csr_structure_ok(ctx, a->rows, a->cols, a->nnz, static_cast<const int64_t *>(a->offsets),
                                           static_cast<const int64_t *>(a->indices));
    if (!ok) fail(TF_ERR_INVALID, "Invalid device CSR structure");
}

// Checked contexts (THERMOFEM_B200_CHECKED=1 at tf_ctx_create) validate a
// caller's CSR before a kernel-layer entry point gathers through it, so a
// column or offset out of range comes back as TF_ERR_INVALID instead of an
// out-of-bounds access.  Setups always validate their input.
void check_operand(tf_ctx *ctx, const tf_csr *a) {
    if (ctx->checked) validate_structure(ctx, a);
}

Csr<double, int32_t> native_csr(const tf_csr *a) {
    check_csr(a);
    require(a->value_type == TF_F64 && a->index_type == TF_I32, "native setup stages take FP64 values and int32 indices");
    require(a->rows == a->cols, "square matrix required");
    return csr_of<double, int32_t>(*a);
}

}  // namespace
}  // namespace tfb

using namespace tfb;

extern "C" {

const char *tf_version(void) { return "thermofem_b200 0.1.0 (sm_100a)"; }
const char *tf_last_error(void) { return g_last_error.c_str(); }
int tf_last_cuda_error(void) { return g_last_cuda; }

const char *tf_status_string(int status) {
    switch (status) {
        case TF_OK: return "ok";
        case TF_ERR_INVALID: return "invalid argument";
        case TF_ERR_CUDA: return "CUDA error";
        case TF_ERR_LENGTH: return "length error";
        case TF_ERR_LOGIC: return "logic error";
        case TF_ERR_TIMEOUT: return "device wait timed out";
        case TF_ERR_NOMEM: return "out of memory";
        case TF_ERR_RUNTIME: return "runtime error";
    }
    return "unknown status";
}

int tf_device_count(int *count) {
    return guard([&] {
        require(count != nullptr, "null output");
        int c = 0;
        cudaError_t e = cudaGetDeviceCount(&c);
        if (e != cudaSuccess) {
            cudaGetLastError();
            c = 0;
        }
        *count = c;
    });
}

int tf_ctx_create(int device, void *stream, tf_ctx **out) {
    return guard([&] {
        require(out != nullptr, "null output");
        *out = nullptr;
        int count = 0;
        cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        require(device >= 0 && device < count, "device ordinal out of range");
        DeviceScope scope(device);  // outlives ctx: a failed create releases on this device
        auto ctx = std::make_unique<tf_ctx>();
        ctx->device = device;
        cuda_check(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device), "SM count");
        // THERMOFEM_B200_PDL=0 launches every kernel with plain stream order.
        const char *pdl = std::getenv("THERMOFEM_B200_PDL");
        ctx->pdl = !(pdl && pdl[0] == '0');
        // THERMOFEM_B200_CHECKED=1 validates caller CSR operands on every kernel-layer call.
        const char *checked = std::getenv("THERMOFEM_B200_CHECKED");
        ctx->checked = checked && checked[0] == '1';
        if (stream) {
            ctx->stream = static_cast<cudaStream_t>(stream);
        } else {
            cuda_check(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ctx->own_stream = true;
        }
        cuda_check(cudaMallocHost(&ctx->pinned, 256), "cudaMallocHost");
        cuda_check(cudaMalloc(&ctx->fault, sizeof(int)), "cudaMalloc");
        cuda_check(cudaMemsetAsync(ctx->fault, 0, sizeof(int), ctx->stream), "cudaMemsetAsync");
        cuda_check(cudaStreamSynchronize(ctx->stream), "context setup");
        *out = ctx.release();
    });
}

int tf_ctx_destroy(tf_ctx *ctx) {
    return guard([&] {
        if (!ctx) return;
        DeviceScope scope(ctx->device);
        delete ctx;
    });
}

int tf_ctx_synchronize(tf_ctx *ctx) {
    return guard([&] {
        check_ctx(ctx);
        cuda_check(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
        check_faults(ctx);
    });
}

int tf_ctx_check_bounded_wait(tf_ctx *ctx, int64_t polls) {
    return guard([&] {
        check_ctx(ctx);
        DeviceScope scope(ctx->device);
        bounded_wait_check(ctx, polls);
    });
}

void *tf_ctx_stream(tf_ctx *ctx) { return ctx ? static_cast<void *>(ctx->stream) : nullptr; }
int tf_ctx_device(tf_ctx *ctx) { return ctx ? ctx->device : -1; }
int64_t tf_ctx_launch_count(tf_ctx *ctx) { return ctx ? ctx->launches : -1; }

int tf_dcsr_view(const tf_dcsr *m, tf_csr *out) {
    return guard([&] {
        require(m && out, "null argument");
        *out = m->view();
    });
}

int tf_dcsr_free(tf_dcsr *m) {
    return guard([&] { delete m; });
}

int tf_csr_validate(tf_ctx *ctx, const tf_csr *a) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        DeviceScope scope(ctx->device);
        validate_structure(ctx, a);
    });
}

int tf_csr_check_canonical(tf_ctx *ctx, const tf_csr *a, int *flags) {
    return guard([&] {
        check_ctx(ctx);
        require(flags != nullptr, "null output");
        DeviceScope scope(ctx->device);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            *flags = csr_canonical_flags(ctx, csr_of<T, I>(*a));
        });
    });
}

int tf_canonicalize(tf_ctx *ctx, const tf_csr *a, tf_dcsr **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out != nullptr, "null output");
        *out = nullptr;
        auto c = native_csr(a);
        require(c.rows > 0 && c.rows < INT32_MAX && c.nnz <= INT32_MAX / 2,
                "AMG requires nonempty square int32-capacity CSR on workspace device");
        DeviceScope scope(ctx->device);
        const int flags = csr_canonical_flags(ctx, c);
        if (flags & 2) fail(TF_ERR_INVALID, "AMG invalid CSR or nonfinite coefficient");
        if (flags == 0) {
            auto m = std::make_unique<tf_dcsr>();
            m->rows = m->cols = c.rows;
            m->nnz = c.nnz;
            m->offsets.allocate((c.rows + 1) * sizeof(int32_t));
            m->indices.allocate(c.nnz * sizeof(int32_t));
            m->values.allocate(c.nnz * sizeof(double));
            copy_async(ctx, m->offsets.data(), c.rp, (c.rows + 1) * sizeof(int32_t));
            copy_async(ctx, m->indices.data(), c.ci, c.nnz * sizeof(int32_t));
            copy_async(ctx, m->values.data(), c.val, c.nnz * sizeof(double));
            cuda_check(cudaStreamSynchronize(ctx->stream), "canonical copy");
            *out = m.release();
        } else {
            auto m = canonicalize(ctx, c);
            cuda_check(cudaStreamSynchronize(ctx->stream), "canonicalize");
            *out = m.release();
        }
    });
}

int tf_convert(tf_ctx *ctx, int64_t n, int src_type, const void *src, int dst_type, void *dst) {
    return guard([&] {
        check_ctx(ctx);
        require(n >= 0 && (n == 0 || (src && dst)), "invalid conversion arguments");
        DeviceScope scope(ctx->device);
        auto go = [&](auto s, auto d) {
            using S = decltype(s);
            using D = decltype(d);
            convert(ctx, n, static_cast<const S *>(src), static_cast<D *>(dst));
        };
        if (src_type == TF_F32 && dst_type == TF_F64) go(float{}, double{});
        else if (src_type == TF_F64 && dst_type == TF_F32) go(double{}, float{});
        else if (src_type == TF_F32 && dst_type == TF_F32) go(float{}, float{});
        else if (src_type == TF_F64 && dst_type == TF_F64) go(double{}, double{});
        else if (src_type == TF_I32 && dst_type == TF_I64) go(int32_t{}, int64_t{});
        else if (src_type == TF_I64 && dst_type == TF_I32) go(int64_t{}, int32_t{});
        else if (src_type == TF_I32 && dst_type == TF_I32) go(int32_t{}, int32_t{});
        else if (src_type == TF_I64 && dst_type == TF_I64) go(int64_t{}, int64_t{});
        else fail(TF_ERR_INVALID, "unsupported conversion");
    });
}

int tf_spmv(tf_ctx *ctx, const tf_csr *a, const void *x, void *y) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        require_vectors(a->cols, {x}, "null SpMV vector");
        require_vectors(a->rows, {y}, "null SpMV vector");
        require(x != y || a->rows == 0, "SpMV shape or alias mismatch");
        DeviceScope scope(ctx->device);
        check_operand(ctx, a);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            spmv(ctx, csr_of<T, I>(*a), static_cast<const T *>(x), static_cast<T *>(y));
        });
    });
}

int tf_spmv_f64(tf_ctx *ctx, int64_t rows, int64_t cols, int64_t nnz, const int32_t *offsets, const int32_t *indices,
                const double *values, const double *x, double *y) {
    tf_csr a{rows, cols, nnz, TF_I32, TF_F64, offsets, indices, values};
    return tf_spmv(ctx, &a, x, y);
}

int tf_spmv_f32(tf_ctx *ctx, int64_t rows, int64_t cols, int64_t nnz, const int32_t *offsets, const int32_t *indices,
                const float *values, const float *x, float *y) {
    tf_csr a{rows, cols, nnz, TF_I32, TF_F32, offsets, indices, values};
    return tf_spmv(ctx, &a, x, y);
}

int tf_autotune_spmv(tf_ctx *ctx, const tf_csr *a, const void *x, void *y, int *stages, int *ctas_per_sm,
                     int *cap_pct, int *rows_per_thread, float *ms) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        require_vectors(a->cols, {x}, "null SpMV vector");
        require_vectors(a->rows, {y}, "null SpMV vector");
        require(x != y || a->rows == 0, "SpMV shape or alias mismatch");
        DeviceScope scope(ctx->device);
        check_operand(ctx, a);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            autotune_spmv(ctx, csr_of<T, I>(*a), static_cast<const T *>(x), static_cast<T *>(y), stages, ctas_per_sm,
                          cap_pct, rows_per_thread, ms);
        });
    });
}

int tf_spmv_set_config(tf_ctx *ctx, const tf_csr *a, int stages, int ctas_per_sm, int cap_pct, int rows_per_thread) {
    return guard([&] {
        check_ctx(ctx);
        DeviceScope scope(ctx->device);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            set_spmv_config(ctx, csr_of<T, I>(*a), stages, ctas_per_sm, cap_pct, rows_per_thread);
        });
    });
}

int tf_residual(tf_ctx *ctx, const tf_csr *a, const void *b, const void *x, void *r) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        require(a->rows == a->cols, "residual needs a square matrix");
        require_vectors(a->rows, {b, x, r}, "null residual vector");
        require(r != b && r != x, "Residual shape or alias mismatch");
        DeviceScope scope(ctx->device);
        check_operand(ctx, a);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            residual(ctx, csr_of<T, I>(*a), static_cast<const T *>(b), static_cast<const T *>(x), static_cast<T *>(r));
        });
    });
}

int tf_jacobi_sweep(tf_ctx *ctx, const tf_csr *a, const void *dinv, const void *b, const void *x, void *x_out,
                    double weight, const float *row_weight, const int32_t *map, const void *coarse) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        require(a->rows == a->cols, "Jacobi needs a square matrix");
        require_vectors(a->rows, {dinv, b, x, x_out}, "null Jacobi vector");
        require(x_out != x || a->rows == 0, "Jacobi sweep output must not alias its input");
        require((map == nullptr) == (coarse == nullptr), "map and coarse go together");
        DeviceScope scope(ctx->device);
        check_operand(ctx, a);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            jacobi_sweep(ctx, csr_of<T, I>(*a), static_cast<const T *>(dinv), static_cast<const T *>(b),
                         static_cast<const T *>(x), static_cast<T *>(x_out), static_cast<T>(weight), row_weight, map,
                         static_cast<const T *>(coarse));
        });
    });
}

int tf_jacobi_zero(tf_ctx *ctx, int64_t n, int value_type, const void *dinv, const void *b, void *x, double weight,
                   const float *row_weight) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(n, {dinv, b, x}, "invalid zero-guess sweep arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            jacobi_zero(ctx, n, static_cast<const T *>(dinv), static_cast<const T *>(b), static_cast<T *>(x),
                        static_cast<T>(weight), row_weight);
        });
    });
}

int tf_jacobi_update(tf_ctx *ctx, int value_type, int64_t n, double weight, const void *dinv, const void *b,
                     const void *ax, void *x) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(n, {dinv, b, ax, x}, "invalid Jacobi update arguments");
        require(n == 0 || (x != ax && x != b && x != dinv), "Jacobi update output aliases an input");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            jacobi_update(ctx, n, static_cast<T>(weight), static_cast<const T *>(dinv), static_cast<const T *>(b),
                          static_cast<const T *>(ax), static_cast<T *>(x));
        });
    });
}

int tf_inverse_diagonal(tf_ctx *ctx, const tf_csr *a, void *dinv) {
    return guard([&] {
        check_ctx(ctx);
        check_csr(a);
        require_vectors(a->rows, {dinv}, "null inverse diagonal");
        DeviceScope scope(ctx->device);
        check_operand(ctx, a);
        with_csr_types(a, [&](auto t, auto i) {
            using T = decltype(t);
            using I = decltype(i);
            inverse_diagonal(ctx, csr_of<T, I>(*a), static_cast<T *>(dinv));
        });
    });
}

int tf_restrict(tf_ctx *ctx, int value_type, int64_t coarse_rows, const int32_t *offsets, const int32_t *members,
                const void *fine, void *coarse) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(coarse_rows, {offsets, members, fine, coarse}, "Invalid aggregate transfer vectors");
        require(fine != coarse || coarse_rows == 0, "Invalid aggregate transfer vectors");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            restrict_sum(ctx, coarse_rows, offsets, members, static_cast<const T *>(fine), static_cast<T *>(coarse));
        });
    });
}

int tf_prolong(tf_ctx *ctx, int value_type, int64_t fine_rows, const int32_t *map, const void *coarse, void *fine) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(fine_rows, {map, coarse, fine}, "Invalid aggregate transfer vectors");
        require(fine != coarse || fine_rows == 0, "Invalid aggregate transfer vectors");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            prolong_add(ctx, fine_rows, map, static_cast<const T *>(coarse), static_cast<T *>(fine));
        });
    });
}

int tf_dot_multi(tf_ctx *ctx, int value_type, int64_t n, int count, const void *const *xs, const void *const *ys,
                 double *out) {
    return guard([&] {
        check_ctx(ctx);
        require(xs && ys && out && count >= 1 && count <= 4 && n >= 0, "invalid dot arguments");
        for (int k = 0; k < count; ++k) require_vectors(n, {xs[k], ys[k]}, "null dot vector");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            const T *x[4], *y[4];
            for (int k = 0; k < count; ++k) {
                x[k] = static_cast<const T *>(xs[k]);
                y[k] = static_cast<const T *>(ys[k]);
            }
            dot_multi(ctx, n, count, x, y, out);
        });
    });
}

int tf_axpby(tf_ctx *ctx, int value_type, int64_t n, double a, const void *x, double b, void *y) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(n, {x, y}, "invalid axpby arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            axpby(ctx, n, a, static_cast<const T *>(x), b, static_cast<T *>(y));
        });
    });
}

int tf_krylov_cg_update(tf_ctx *ctx, int value_type, int64_t n, double alpha, const void *p, const void *ap,
                        void *x, void *r, double *rr) {
    return guard([&] {
        check_ctx(ctx);
        require(n >= 0 && p && ap && x && r && rr && x != r, "invalid CG update arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            krylov_cg_update(ctx, n, alpha, static_cast<const T *>(p), static_cast<const T *>(ap), static_cast<T *>(x),
                             static_cast<T *>(r), rr);
        });
    });
}

int tf_krylov_cg_direction(tf_ctx *ctx, int value_type, int64_t n, double beta, int restart, const void *z, void *p) {
    return guard([&] {
        check_ctx(ctx);
        require(n >= 0 && z && p && z != p, "invalid CG direction arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            krylov_cg_direction(ctx, n, beta, restart, static_cast<const T *>(z), static_cast<T *>(p));
        });
    });
}

int tf_krylov_bicgstab_direction(tf_ctx *ctx, int value_type, int64_t n, double beta, double omega, int restart,
                                 const void *r, const void *v, void *p) {
    return guard([&] {
        check_ctx(ctx);
        require(n >= 0 && r && v && p && p != r && p != v, "invalid BiCGStab direction arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            krylov_bicgstab_direction(ctx, n, beta, omega, restart, static_cast<const T *>(r),
                                      static_cast<const T *>(v), static_cast<T *>(p));
        });
    });
}

int tf_krylov_bicgstab_s(tf_ctx *ctx, int value_type, int64_t n, double alpha, const void *r, const void *v,
                         const void *phat, void *x, void *s, double *ss) {
    return guard([&] {
        check_ctx(ctx);
        require(n >= 0 && r && v && phat && x && s && ss && x != s, "invalid BiCGStab s-step arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            krylov_bicgstab_s(ctx, n, alpha, static_cast<const T *>(r), static_cast<const T *>(v),
                              static_cast<const T *>(phat), static_cast<T *>(x), static_cast<T *>(s), ss);
        });
    });
}

int tf_krylov_bicgstab_update(tf_ctx *ctx, int value_type, int64_t n, double omega, const void *shat,
                              const void *s, const void *t, void *x, void *r, double *rr) {
    return guard([&] {
        check_ctx(ctx);
        require(n >= 0 && shat && s && t && x && r && rr && x != r, "invalid BiCGStab update arguments");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto tv) {
            using T = decltype(tv);
            krylov_bicgstab_update(ctx, n, omega, static_cast<const T *>(shat), static_cast<const T *>(s),
                                   static_cast<const T *>(t), static_cast<T *>(x), static_cast<T *>(r), rr);
        });
    });
}

int tf_row_stats(tf_ctx *ctx, const tf_csr *a, double *row_max, int *bad) {
    return guard([&] {
        check_ctx(ctx);
        require(bad != nullptr, "null output");
        auto c = native_csr(a);
        require_vectors(c.rows, {row_max}, "null row maximum");
        DeviceScope scope(ctx->device);
        *bad = row_stats(ctx, c, row_max) ? 0 : 1;
    });
}

int tf_strength(tf_ctx *ctx, const tf_csr *a, const double *row_max, double threshold, tf_dcsr **graph) {
    return guard([&] {
        check_ctx(ctx);
        require(graph != nullptr && row_max != nullptr, "null argument");
        *graph = nullptr;
        auto c = native_csr(a);
        require(c.rows > 0, "empty matrix");
        DeviceScope scope(ctx->device);
        auto g = strength_graph(ctx, c, row_max, threshold);
        cuda_check(cudaStreamSynchronize(ctx->stream), "strength");
        *graph = g.release();
    });
}

int tf_match(tf_ctx *ctx, const tf_csr *graph, int rounds, int32_t *map, int *count) {
    return guard([&] {
        check_ctx(ctx);
        require(map && count, "null argument");
        auto g = native_csr(graph);
        require(g.rows > 0, "empty graph");
        DeviceScope scope(ctx->device);
        *count = match_pairs(ctx, g, rounds, map);
    });
}

int tf_contract(tf_ctx *ctx, const tf_csr *graph, const int32_t *map, int count, tf_dcsr **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out && map && count >= 1, "invalid contraction arguments");
        *out = nullptr;
        auto g = native_csr(graph);
        DeviceScope scope(ctx->device);
        auto c = contract_graph(ctx, g, map, count);
        cuda_check(cudaStreamSynchronize(ctx->stream), "contract");
        *out = c.release();
    });
}

int tf_aggregate(tf_ctx *ctx, const tf_csr *graph, int rounds, int absorb_singletons, tf_transfer **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out != nullptr, "null output");
        *out = nullptr;
        require(rounds >= 1 && rounds <= 8 && graph && graph->rows > 0, "Invalid matching configuration");
        auto g = native_csr(graph);
        DeviceScope scope(ctx->device);
        *out = aggregate(ctx, g, rounds, absorb_singletons != 0).release();
    });
}

int tf_transfer_info(const tf_transfer *t, int *fine_rows, int *coarse_rows, int32_t histogram[4]) {
    return guard([&] {
        require(t != nullptr, "null transfer");
        if (fine_rows) *fine_rows = t->fine_rows;
        if (coarse_rows) *coarse_rows = t->coarse_rows;
        if (histogram)
            for (int k = 0; k < 4; ++k) histogram[k] = t->histogram[k];
    });
}

int tf_transfer_arrays(const tf_transfer *t, const int32_t **map, const int32_t **offsets, const int32_t **members) {
    return guard([&] {
        require(t != nullptr, "null transfer");
        if (map) *map = t->map.data();
        if (offsets) *offsets = t->offsets.data();
        if (members) *members = t->members.data();
    });
}

int tf_transfer_free(tf_transfer *t) {
    return guard([&] { delete t; });
}

int tf_galerkin(tf_ctx *ctx, const tf_csr *a, const tf_transfer *t, tf_dcsr **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out && t, "null argument");
        *out = nullptr;
        auto c = native_csr(a);
        require(c.rows == t->fine_rows && t->coarse_rows >= 1, "AMG transfer dimension mismatch");
        DeviceScope scope(ctx->device);
        auto m = galerkin(ctx, c, t->map.data(), t->coarse_rows);
        cuda_check(cudaStreamSynchronize(ctx->stream), "galerkin");
        *out = m.release();
    });
}

int tf_galerkin_map(tf_ctx *ctx, const tf_csr *a, const int32_t *map, int coarse_rows, tf_dcsr **out) {
    return guard([&] {
        check_ctx(ctx);
        require(out && map, "null argument");
        *out = nullptr;
        auto c = native_csr(a);
        require(coarse_rows >= 1 && coarse_rows <= c.rows, "AMG transfer dimension mismatch");
        DeviceScope scope(ctx->device);
        if (indices_out_of_range(ctx, c.rows, map, coarse_rows))
            fail(TF_ERR_INVALID, "aggregate map entry outside 0..coarse_rows-1");
        auto m = galerkin(ctx, c, map, coarse_rows);
        cuda_check(cudaStreamSynchronize(ctx->stream), "galerkin");
        *out = m.release();
    });
}

int tf_radix_sort_pairs_u64f64(tf_ctx *ctx, int64_t n, const uint64_t *keys_in, const double *values_in,
                               uint64_t *keys_out, double *values_out, int end_bit) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(n, {keys_in, values_in, keys_out, values_out}, "invalid sort arguments");
        require(n == 0 || (keys_in != keys_out && values_in != values_out), "sort outputs must not alias inputs");
        DeviceScope scope(ctx->device);
        radix_sort_pairs(ctx, n, keys_in, values_in, keys_out, values_out, end_bit);
    });
}

int tf_reduce_by_key_u64f64(tf_ctx *ctx, int64_t n, const uint64_t *keys, const double *values, int op,
                            uint64_t *keys_out, double *values_out, int64_t *count) {
    return guard([&] {
        check_ctx(ctx);
        require(count != nullptr && (op == 0 || op == 1), "invalid reduce arguments");
        require_vectors(n, {keys, values, keys_out, values_out}, "invalid reduce arguments");
        DeviceScope scope(ctx->device);
        *count = reduce_by_key(ctx, n, keys, values, op, keys_out, values_out);
    });
}

int tf_scan_exclusive_i32(tf_ctx *ctx, int64_t n, const int32_t *in, int32_t *out) {
    return guard([&] {
        check_ctx(ctx);
        require_vectors(n, {in, out}, "invalid scan arguments");
        DeviceScope scope(ctx->device);
        scan_exclusive(ctx, n, in, out);
    });
}

int tf_coarse_lu_factor(tf_ctx *ctx, const tf_csr *a, double *lu, int32_t *pivots, int *factored) {
    return guard([&] {
        check_ctx(ctx);
        require(lu && pivots && factored, "null argument");
        auto c = native_csr(a);
        DeviceScope scope(ctx->device);
        *factored = coarse_lu_factor(ctx, c, lu, pivots) ? 1 : 0;
    });
}

int tf_coarse_lu_solve(tf_ctx *ctx, int rows, const double *lu, const int32_t *pivots, int value_type, const void *b,
                       void *x) {
    return guard([&] {
        check_ctx(ctx);
        require(lu && pivots && b && x, "null argument");
        DeviceScope scope(ctx->device);
        with_value_type(value_type, [&](auto t) {
            using T = decltype(t);
            coarse_lu_solve(ctx, rows, lu, pivots, static_cast<const T *>(b), static_cast<T *>(x));
        });
    });
}

}  // extern "C"
