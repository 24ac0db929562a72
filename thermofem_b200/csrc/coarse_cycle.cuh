// coarse_cycle.cuh -- program steps of the cooperative small-level cycle.
#pragma once
#include "ops.cuh"

namespace tfb {

constexpr int kCoarseThreads = 512;

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
};

// CTAs of the cooperative launch (all resident at once).
template <class S>
int coarse_grid_size(int sm_count, int64_t max_rows);

// barrier: 3 device words (arrival count, generation, abort), zeroed once.
template <class S>
void launch_coarse_program(tf_ctx *ctx, const CoarseStep<S> *program, int steps, unsigned *barrier, int grid);

}  // namespace tfb
