// coarse_cycle.cu -- the small levels of an AMG cycle in one cooperative
// launch.
//
// Below a few hundred thousand rows every level operation of the cycle is a
// few microseconds of launch latency for well under a microsecond of work.
// The host records the level steps of the sub-cycle that starts at the first
// small level (the same recursion as the large levels: Cycle.cuh:35-63) into
// a program; one cooperative kernel (all CTAs co-resident) walks the program
// with a grid-wide barrier between steps.  Values written inside the kernel
// are read back with ld.global.cg (L2, never a stale L1 line).  The barrier
// is bounded: a CTA that waits too long raises the context's fault word and
// every CTA leaves at its next barrier.
//
// Step semantics match the launched kernels exactly: sweeps x_out =
// x~ + w d (b - A x~) with x~ = x (+ e[map]), residual-restriction
// coarse[c] = sum over members m (in member order) of (b_m - (A x)_m) with each
// residual rounded to the level type first, prolongation x += e[map], the
// dense coarse inverse.
#include "coarse_cycle.cuh"

namespace tfb {
namespace {

template <class T>
__device__ __forceinline__ T ldcg(const T *p) {
    return __ldcg(p);
}

__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded sense barrier over all CTAs of the grid: one atomic arrival per CTA,
// waiters poll the generation word with acquire loads.  Returns false when
// the wait expired or another CTA already gave up.
__device__ bool grid_barrier(unsigned *count, unsigned *generation, unsigned *abort_flag, int *fault) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned gen = load_acquire(generation);
        __threadfence();
        if (atomicAdd(count, 1u) == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(generation, 1u);
        } else {
            long long spins = 0;
            while (load_acquire(generation) == gen) {
                if ((++spins & 255) == 0 && (load_acquire(abort_flag) || spins > (1ll << 24))) {
                    atomicExch(abort_flag, 1u);
                    atomicExch(fault, 1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (load_acquire(abort_flag)) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// Row i of A times x (x~ when map/e are set), left to right, eight gathers in flight.
template <class S>
__device__ __forceinline__ S row_dot(const CoarseStep<S> &st, int i, const S *x) {
    const int s = __ldg(st.rp + i), e = __ldg(st.rp + i + 1);
    S acc = S(0);
    for (int j0 = s; j0 < e; j0 += 8) {
        S y[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = j0 + u;
            if (j < e) {
                const int c = __ldg(st.ci + j);
                y[u] = ldcg(x + c);
                if (st.map) y[u] += ldcg(st.e + __ldg(st.map + c));
            } else {
                y[u] = S(0);
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = j0 + u;
            acc += (j < e ? __ldg(st.val + j) : S(0)) * y[u];
        }
    }
    return acc;
}

template <class S>
__global__ void __launch_bounds__(kCoarseThreads) coarse_program_kernel(const CoarseStep<S> *program, int steps,
                                                                         unsigned *barrier, int *fault) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int k = 0; k < steps; ++k) {
        const CoarseStep<S> st = program[k];
        switch (st.op) {
            case kStepZero:
                for (int i = tid; i < st.n; i += stride) st.xout[i] = S(0);
                break;
            case kStepJacobiZero:
                for (int i = tid; i < st.n; i += stride) st.xout[i] = st.w * __ldg(st.dinv + i) * ldcg(st.rhs + i);
                break;
            case kStepSweep:
                for (int i = tid; i < st.n; i += stride) {
                    const S ax = row_dot(st, i, st.xin);
                    S xi = ldcg(st.xin + i);
                    if (st.map) xi += ldcg(st.e + __ldg(st.map + i));
                    st.xout[i] = xi + st.w * __ldg(st.dinv + i) * (ldcg(st.rhs + i) - ax);
                }
                break;
            case kStepResidualRestrict: {
                // a quad of lanes per coarse row, one member (<= 4) per lane;
                // lane 0 of the quad adds the member residuals in member order
                const int quads = stride >> 2, quad = tid >> 2, k4 = tid & 3;
                for (int base = 0; base < st.nc; base += quads) {
                    const int c = base + quad;
                    int count = 0;
                    S r = S(0);
                    if (c < st.nc) {
                        const int j0 = __ldg(st.off + c);
                        count = __ldg(st.off + c + 1) - j0;
                        if (k4 < count) {
                            const int m = __ldg(st.mem + j0 + k4);
                            r = ldcg(st.rhs + m) - row_dot(st, m, st.xin);
                        }
                    }
                    const S r1 = __shfl_sync(0xffffffffu, r, 1, 4);
                    const S r2 = __shfl_sync(0xffffffffu, r, 2, 4);
                    const S r3 = __shfl_sync(0xffffffffu, r, 3, 4);
                    if (c < st.nc && k4 == 0) {
                        S sum = S(0);
                        if (count > 0) sum += r;
                        if (count > 1) sum += r1;
                        if (count > 2) sum += r2;
                        if (count > 3) sum += r3;
                        st.coarse_rhs[c] = sum;
                    }
                }
                break;
            }
            case kStepRestrict:
                for (int c = tid; c < st.nc; c += stride) {
                    S sum = S(0);
                    for (int j = __ldg(st.off + c); j < __ldg(st.off + c + 1); ++j) sum += ldcg(st.rhs + __ldg(st.mem + j));
                    st.coarse_rhs[c] = sum;
                }
                break;
            case kStepProlong:
                for (int i = tid; i < st.n; i += stride) st.xout[i] = ldcg(st.xin + i) + ldcg(st.e + __ldg(st.map + i));
                break;
            case kStepDense: {
                // one warp per row of the dense inverse (rows <= 256)
                const int warp = tid >> 5, lane = tid & 31, warps = stride >> 5;
                for (int i = warp; i < st.n; i += warps) {
                    double s = 0;
                    for (int j = lane; j < st.n; j += 32)
                        s += __ldg(st.inv + static_cast<int64_t>(i) * st.n + j) * static_cast<double>(ldcg(st.rhs + j));
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                    if (lane == 0) st.xout[i] = static_cast<S>(s);
                }
                break;
            }
            default:
                break;
        }
        if (k + 1 < steps && !grid_barrier(barrier, barrier + 1, barrier + 2, fault)) return;
    }
}

}  // namespace

// One thread per row of the largest level of the region (at least one CTA,
// at most one per SM): fewer CTAs make every barrier cheaper.
template <class S>
int coarse_grid_size(int sm_count, int64_t max_rows) {
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, coarse_program_kernel<S>, kCoarseThreads, 0),
               "coarse occupancy");
    if (per_sm < 1) fail(TF_ERR_CUDA, "coarse-cycle kernel cannot be resident");
    int64_t g = (max_rows + kCoarseThreads - 1) / kCoarseThreads;
    if (g < 1) g = 1;
    if (g > sm_count) g = sm_count;
    return static_cast<int>(g);
}

template <class S>
void launch_coarse_program(tf_ctx *ctx, const CoarseStep<S> *program, int steps, unsigned *barrier, int grid) {
    if (steps <= 0) return;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(kCoarseThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cuda_check(cudaLaunchKernelEx(&cfg, coarse_program_kernel<S>, program, steps, barrier, ctx->fault),
               "coarse-cycle launch");
    launched(ctx, "coarse_program");
}

template int coarse_grid_size<float>(int, int64_t);
template int coarse_grid_size<double>(int, int64_t);
template void launch_coarse_program<float>(tf_ctx *, const CoarseStep<float> *, int, unsigned *, int);
template void launch_coarse_program<double>(tf_ctx *, const CoarseStep<double> *, int, unsigned *, int);

}  // namespace tfb
