// coarse_cycle.cuh -- program steps of the small-level cycle (one cluster launch).
#pragma once
#include "ops.cuh"

namespace tfb {

constexpr int kClusterThreads = 1024;

enum CoarseOp : int {
    kStepZero = 0,              // xout = 0
    kStepJacobiZero = 1,        // xout = w Dinv rhs
    kStepSweep = 2,             // xout = x~ + w Dinv (rhs - A x~), x~ = xin (+ e[map])
    kStepResidualRestrict = 3,  // coarse_rhs[c] = sum_members (rhs - A xin)
    kStepRestrict = 4,          // coarse_rhs[c] = sum_members rhs
    kStepProlong = 5,           // xout = xin + e[map]
    kStepDense = 6,             // xout = inv rhs (n <= 256)
};

// One step of a level (int32 indices, level type S).  Unused fields null.
template <class S>
struct CoarseStep {
    int op{0};
    int n{0}, nc{0};
    S w{0};
    const int32_t *rp{nullptr}, *ci{nullptr};
    const S *val{nullptr}, *dinv{nullptr};
    const S *rhs{nullptr};
    const S *xin{nullptr};
    S *xout{nullptr};
    const int32_t *map{nullptr};
    const S *e{nullptr};
    const int32_t *off{nullptr}, *mem{nullptr};
    S *coarse_rhs{nullptr};
    const double *inv{nullptr};
    // Restrictions only: with cx set, the coarse level's zero-guess sweep is
    // done in the same pass, cx[c] = cw * cdinv[c] * coarse_rhs[c].
    const S *cdinv{nullptr};
    S *cx{nullptr};
    S cw{0};
};

// Transfers around one launch of a program.  With rsrc set, the first
// step's level first receives rrhs[c] = sum of rsrc over the members
// roff/rmem of aggregate c (fused into the first step when that is the
// level's zero-guess sweep).  With sfine set, the last step (a sweep or the
// dense solve) adds each new value xout[c] to sfine at the members soff/smem
// of aggregate c.
template <class S>
struct ProgramIO {
    const S *rsrc{nullptr};
    const int32_t *roff{nullptr}, *rmem{nullptr};
    S *rrhs{nullptr};
    int rn{0};
    const int32_t *soff{nullptr}, *smem{nullptr};
    S *sfine{nullptr};
};

// CTAs of the cluster that runs the program: the largest cluster (16, 8, 4,
// 2 or 1 CTAs of kClusterThreads) the device can schedule.
template <class S>
int coarse_cluster_size();

template <class S>
void launch_coarse_program(tf_ctx *ctx, const CoarseStep<S> *program, int steps, const ProgramIO<S> &io,
                           int cluster);

}  // namespace tfb
