// coarse_cycle.cu -- the small levels of an AMG cycle in one cluster launch.
//
// Below a few ten thousand rows every level operation of the cycle is a few
// microseconds of launch and memory latency for well under a microsecond of
// work.  The host records the level steps of the sub-cycle that starts at the
// first small level (the same recursion as the large levels: Cycle.cuh:35-63)
// into a program; one thread-block cluster walks the program with the
// hardware cluster barrier (barrier.cluster, release/acquire) between steps.
// All CTAs of a cluster are co-scheduled by construction, so the barrier
// needs no spin loop and cannot wait on a CTA that is not running.  Values
// written inside the kernel are read back with ld.global.cg (L2, never a
// stale L1 line).
//
// Step semantics match the launched kernels exactly: sweeps x_out =
// x~ + w d (b - A x~) with x~ = x (+ e[map]), residual-restriction
// coarse[c] = sum over members m (in member order) of (b_m - (A x)_m) with
// each residual rounded to the level type first, the zero-guess sweep
// x = w d b, prolongation x += e[map] (or fine[m] += x_c over the members m
// of c), the dense coarse inverse.
#include "coarse_cycle.cuh"

namespace tfb {
namespace {

template <class T>
__device__ __forceinline__ T ldcg(const T *p) {
    return __ldcg(p);
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// Row i of A times x with kGroup lanes per row: lane k of the group loads
// entries k, k + kGroup, ... (all loads of a row in flight at once), and the
// group's lane 0 adds the products left to right from shuffles (the order
// and the FMAs of the row-tile kernels, so the same bits).  Every lane of the
// warp calls it (lanes without a row pass i = -1); the result is valid in the
// group's lane 0.  x~ = x + e[map] when the step has map/e.
constexpr int kGroup = 8;
template <class S>
__device__ __forceinline__ S row_dot_group(const CoarseStep<S> &st, int i, const S *x) {
    const int g = threadIdx.x & (kGroup - 1);
    int s = 0, e = 0;
    if (i >= 0) {
        s = __ldg(st.rp + i);
        e = __ldg(st.rp + i + 1);
    }
    const int len = e - s;
    const int warp_len = __reduce_max_sync(0xffffffffu, len);
    S acc = S(0);
    for (int base = 0; base < warp_len; base += kGroup) {
        const int j = s + base + g;
        S v = S(0), y = S(0);
        if (base + g < len) {
            const int c = __ldg(st.ci + j);
            v = __ldg(st.val + j);
            y = ldcg(x + c);
            if (st.map) y += ldcg(st.e + __ldg(st.map + c));
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            const S vu = __shfl_sync(0xffffffffu, v, u, kGroup);
            const S yu = __shfl_sync(0xffffffffu, y, u, kGroup);
            if (base + u < len) acc += vu * yu;
        }
    }
    return acc;
}

// sum of src over the members of aggregate c (restrict_kernel's order)
template <class S>
__device__ __forceinline__ S member_sum(const int32_t *off, const int32_t *mem, const S *src, int c) {
    S s = S(0);
    for (int j = __ldg(off + c); j < __ldg(off + c + 1); ++j) s += ldcg(src + __ldg(mem + j));
    return s;
}

template <class S>
__device__ __forceinline__ void scatter(const ProgramIO<S> &io, int c, S v, int lane, int lanes) {
    for (int k = __ldg(io.soff + c) + lane; k < __ldg(io.soff + c + 1); k += lanes) {
        const int m = __ldg(io.smem + k);
        io.sfine[m] = ldcg(io.sfine + m) + v;
    }
}

template <class S>
__global__ void __launch_bounds__(kClusterThreads, 1)
    coarse_cluster_kernel(const CoarseStep<S> *program, int steps, ProgramIO<S> io) {
    extern __shared__ __align__(16) unsigned char prog_smem[];
    // the program (read by every thread at every step) is staged once
    CoarseStep<S> *prog = reinterpret_cast<CoarseStep<S> *>(prog_smem);
    {
        const int words = static_cast<int>(steps * sizeof(CoarseStep<S>) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(program);
        int *dst = reinterpret_cast<int *>(prog_smem);
        for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = __ldg(src + k);
    }
    pdl_enter();
    __syncthreads();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    bool restricted = io.rsrc == nullptr;
    if (!restricted) {
        const CoarseStep<S> &first = prog[0];
        if (!(first.op == kStepJacobiZero && first.rhs == io.rrhs)) {
            for (int c = tid; c < io.rn; c += stride) io.rrhs[c] = member_sum(io.roff, io.rmem, io.rsrc, c);
            cluster_sync();
            restricted = true;
        }
    }
    for (int k = 0; k < steps; ++k) {
        const CoarseStep<S> &st = prog[k];
        const bool last = k + 1 == steps && io.sfine != nullptr;
        switch (st.op) {
            case kStepZero:
                for (int i = tid; i < st.n; i += stride) st.xout[i] = S(0);
                break;
            case kStepJacobiZero:
                for (int i = tid; i < st.n; i += stride) {
                    S b;
                    if (!restricted) {  // first step: the region's restriction fused in
                        b = member_sum(io.roff, io.rmem, io.rsrc, i);
                        io.rrhs[i] = b;
                    } else {
                        b = ldcg(st.rhs + i);
                    }
                    st.xout[i] = st.w * __ldg(st.dinv + i) * b;
                }
                restricted = true;
                break;
            case kStepSweep: {
                // kGroup lanes per row; warps stay converged for the shuffles
                const int groups = stride / kGroup, g0 = tid / kGroup, lane = tid & (kGroup - 1);
                for (int base = 0; base < st.n; base += groups) {
                    const int i = base + g0 < st.n ? base + g0 : -1;
                    const S ax = row_dot_group(st, i, st.xin);
                    if (i >= 0 && lane == 0) {
                        S xi = ldcg(st.xin + i);
                        if (st.map) xi += ldcg(st.e + __ldg(st.map + i));
                        const S v = xi + st.w * __ldg(st.dinv + i) * (ldcg(st.rhs + i) - ax);
                        st.xout[i] = v;
                        if (last) scatter(io, i, v, 0, 1);
                    }
                }
                break;
            }
            case kStepResidualRestrict: {
                // a warp per coarse row, kGroup lanes per member (<= 4); lane 0
                // adds the member residuals in member order
                const int warps = stride >> 5, wid = tid >> 5, k4 = (tid & 31) / kGroup;
                for (int base = 0; base < st.nc; base += warps) {
                    const int c = base + wid;
                    int count = 0, m = -1;
                    if (c < st.nc) {
                        const int j0 = __ldg(st.off + c);
                        count = __ldg(st.off + c + 1) - j0;
                        if (k4 < count) m = __ldg(st.mem + j0 + k4);
                    }
                    const S ax = row_dot_group(st, m, st.xin);
                    const S r = m >= 0 ? ldcg(st.rhs + m) - ax : S(0);
                    const S r1 = __shfl_sync(0xffffffffu, r, kGroup);
                    const S r2 = __shfl_sync(0xffffffffu, r, 2 * kGroup);
                    const S r3 = __shfl_sync(0xffffffffu, r, 3 * kGroup);
                    if (c < st.nc && (tid & 31) == 0) {
                        S sum = S(0);
                        if (count > 0) sum += r;
                        if (count > 1) sum += r1;
                        if (count > 2) sum += r2;
                        if (count > 3) sum += r3;
                        st.coarse_rhs[c] = sum;
                        if (st.cx) st.cx[c] = st.cw * __ldg(st.cdinv + c) * sum;
                    }
                }
                break;
            }
            case kStepRestrict:
                for (int c = tid; c < st.nc; c += stride) {
                    const S sum = member_sum(st.off, st.mem, st.rhs, c);
                    st.coarse_rhs[c] = sum;
                    if (st.cx) st.cx[c] = st.cw * __ldg(st.cdinv + c) * sum;
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
                    const S v = static_cast<S>(__shfl_sync(0xffffffffu, s, 0));
                    if (lane == 0) st.xout[i] = v;
                    if (last) scatter(io, i, v, lane, 32);
                }
                break;
            }
            default:
                break;
        }
        if (k + 1 < steps) cluster_sync();
    }
}

template <class S>
cudaLaunchConfig_t cluster_config(int cluster, cudaLaunchAttribute *attr, int &nattr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(cluster));
    cfg.blockDim = dim3(kClusterThreads);
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    nattr = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

}  // namespace

template <class S>
int coarse_cluster_size() {
    cuda_check(cudaFuncSetAttribute(coarse_cluster_kernel<S>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
               "cluster attribute");
    for (int c : {16, 8, 4, 2, 1}) {
        cudaLaunchAttribute attr[2];
        int nattr = 0;
        cudaLaunchConfig_t cfg = cluster_config<S>(c, attr, nattr);
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, coarse_cluster_kernel<S>, &cfg) == cudaSuccess && clusters >= 1)
            return c;
        cudaGetLastError();
    }
    fail(TF_ERR_CUDA, "small-level cycle: no thread-block cluster can be scheduled");
    return 1;
}

template <class S>
void launch_coarse_program(tf_ctx *ctx, const CoarseStep<S> *program, int steps, const ProgramIO<S> &io,
                           int cluster) {
    if (steps <= 0) return;
    cudaLaunchAttribute attr[2];
    int nattr = 0;
    cudaLaunchConfig_t cfg = cluster_config<S>(cluster, attr, nattr);
    cfg.stream = ctx->stream;
    cfg.dynamicSmemBytes = static_cast<size_t>(steps) * sizeof(CoarseStep<S>);
    require(cfg.dynamicSmemBytes <= 200 * 1024, "small-level program too long: lower small_level_rows");
    if (cfg.dynamicSmemBytes > 48 * 1024)
        cuda_check(cudaFuncSetAttribute(coarse_cluster_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(cfg.dynamicSmemBytes)),
                   "small-level program shared memory");
    if (ctx->pdl) {
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.numAttrs = 2;
    }
    cuda_check(cudaLaunchKernelEx(&cfg, coarse_cluster_kernel<S>, program, steps, io), "small-level cycle launch");
    launched(ctx, "coarse_program");
}

template int coarse_cluster_size<float>();
template int coarse_cluster_size<double>();
template void launch_coarse_program<float>(tf_ctx *, const CoarseStep<float> *, int, const ProgramIO<float> &, int);
template void launch_coarse_program<double>(tf_ctx *, const CoarseStep<double> *, int, const ProgramIO<double> &,
                                            int);

}  // namespace tfb
