// coarse_cycle.cuh -- the small levels of an AMG cycle as one thread-block
// cluster working out of distributed shared memory.
#pragma once
#include <memory>
#include <vector>

#include "ops.cuh"

namespace tfb {

constexpr int kTailThreads = 1024;
constexpr int kTailMaxLevels = 16;

// Steps of a recorded small-level sub-cycle (the host recursion's level
// operations, level type S, int32 indices).  Unused fields null.
enum CoarseOp : int {
    kStepZero = 0,              // xout = 0
    kStepJacobiZero = 1,        // xout = w Dinv rhs
    kStepSweep = 2,             // xout = x~ + w Dinv (rhs - A x~), x~ = xin (+ e[map])
    kStepResidualRestrict = 3,  // coarse_rhs[c] = sum_members (rhs - A xin)
    kStepRestrict = 4,          // coarse_rhs[c] = sum_members rhs
    kStepProlong = 5,           // xout = xin + e[map]
    kStepDense = 6,             // xout = inv rhs (n <= 256)
};

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

// Transfers around one launch of a region.  With rsrc set, the region's
// root first receives rrhs[c] = sum of rsrc over the members roff/rmem of
// aggregate c (else its rhs is read from memory).  With sfine set, each
// final root value x[c] is added to sfine at the members soff/smem of c.
// (The region kernel reads those maps from its plan: roff/rmem and
// soff/smem are the root's parent aggregates, TailParent.)
template <class S>
struct ProgramIO {
    const S *rsrc{nullptr};
    const int32_t *roff{nullptr}, *rmem{nullptr};
    S *rrhs{nullptr};
    int rn{0};
    const int32_t *soff{nullptr}, *smem{nullptr};
    S *sfine{nullptr};
};

// One level of a region, as the launched cycle keeps it in global memory.
template <class S>
struct TailLevel {
    int64_t n{0};
    const int32_t *rp{nullptr}, *ci{nullptr};
    const int16_t *cd{nullptr};  // columns as offsets from the row, when the level has them
    const S *val{nullptr}, *dinv{nullptr};
    S *rhs{nullptr}, *x0{nullptr}, *x1{nullptr};
    const int32_t *map{nullptr};             // row -> aggregate of the next level (null on the last)
    const int32_t *off{nullptr}, *mem{nullptr};  // aggregates of the next level -> rows of this level
};

// The root's aggregates in the level above it (that level's aggregate
// offsets and members over its n rows): the restriction into the root and
// the prolongation out of it.
struct TailParent {
    int64_t n{0};
    const int32_t *off{nullptr}, *mem{nullptr};
};

template <class S>
struct TailDevice;  // device-side plan (coarse_cycle.cu)

// The small levels of the cycle (a root level and every level below it),
// run by one CTA or one thread-block cluster: each CTA holds its share of
// every level's rows -- matrix rows, diagonal, right-hand side, iterates,
// transfer maps -- in its shared memory for the whole launch, and reads
// other CTAs' values through distributed shared memory, with the hardware
// cluster barrier between dependent steps.  Only the root's vectors are read
// from and written back to global memory.
template <class S>
class TailRegion {
  public:
    TailRegion();
    ~TailRegion();
    // Lays the levels (and room for max_steps steps) out over the largest
    // schedulable cluster; false when they do not fit in its shared memory
    // (nothing is kept then).
    bool plan(tf_ctx *ctx, const std::vector<TailLevel<S>> &levels, const TailParent &parent, const double *inv,
              int dense_n, S w, int max_steps);
    // Translates one recorded sub-cycle into region steps; false when a step
    // does not belong to the region's levels.
    bool add_entry(const std::vector<CoarseStep<S>> &steps, size_t first, size_t count);
    void upload(tf_ctx *ctx);
    // Runs entry `entry`; root_cur is the root buffer (0: x0, 1: x1) that
    // holds its result at the end, written back with both buffers and rhs.
    void launch(tf_ctx *ctx, int entry, const ProgramIO<S> &io, int root_cur) const;
    int cluster() const { return cluster_; }
    size_t shared_bytes() const { return smem_; }

  private:
    struct Step {
        int op, level, a, b, c;
    };
    std::vector<TailLevel<S>> levels_;
    std::vector<Step> steps_;
    std::vector<std::pair<int, int>> entries_;
    std::unique_ptr<TailDevice<S>> dev_;
    int cluster_{0}, max_steps_{0};
    size_t smem_{0};
};

}  // namespace tfb
