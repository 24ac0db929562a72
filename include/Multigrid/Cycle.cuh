// Cycle.cuh -- V, W and F multigrid schedules, independent of matrices,
// smoothers and how the steps run (drop-in for include/Multigrid/Cycle.cuh:
// 10-63 of Mgepahmge/ThermoFEM: the same enum, operations concept and
// executeCycle semantics).
//
// The schedule per level d (begin(d) counts a visit; x_d is cleared on entry
// when zeroInitial is set, and always for F):
//   coarsest  coarseSolve(d)
//   V         preSmooth, restrictResidual, V(d+1, zero), prolong, postSmooth
//   W         as V with a second W(d+1) that keeps the first's result
//   F         restrictRhs, F(d+1, zero), prolong (x_d was cleared, so this
//             sets x_d to the coarse solution), then a V correction on d
//             from that x_d
// Fixed visits and fixed smoothing keep the cycle a linear operator.
// Visits per level: V 1; W 2^d; F d+2 (the coarsest: the number of levels).
// In this library the hierarchy records these steps once into a CUDA graph
// (tf_amg_apply); the host recursion here drives the same steps for
// hierarchies with user-supplied smoothers.
#pragma once

#include <concepts>
#include <cstddef>
#include <stdexcept>

namespace thermofem::multigrid {

enum class Cycle { V, W, F };

template <class O>
concept CycleOperations = requires(O &ops, std::size_t level) {
    { ops.isCoarsest(level) } -> std::convertible_to<bool>;
    ops.begin(level);
    ops.clear(level);
    ops.coarseSolve(level);
    ops.preSmooth(level);
    ops.postSmooth(level);
    ops.restrictRhs(level);
    ops.restrictResidual(level);
    ops.prolong(level);
};

template <CycleOperations O>
void executeCycle(Cycle kind, std::size_t level, O &ops, bool zeroInitial = true) {
    switch (kind) {
        case Cycle::V:
        case Cycle::W:
        case Cycle::F: break;
        default: throw std::invalid_argument("Unknown AMG cycle");
    }
    ops.begin(level);
    if (zeroInitial || kind == Cycle::F) ops.clear(level);
    if (ops.isCoarsest(level)) {
        ops.coarseSolve(level);
        return;
    }
    const std::size_t coarser = level + 1;
    if (kind == Cycle::F) {
        // nested iteration: a coarse F solve as the initial guess, then a V correction
        ops.restrictRhs(level);
        executeCycle(Cycle::F, coarser, ops, true);
        ops.prolong(level);
        executeCycle(Cycle::V, level, ops, false);
        return;
    }
    ops.preSmooth(level);
    ops.restrictResidual(level);
    const int coarseVisits = kind == Cycle::W ? 2 : 1;
    for (int visit = 0; visit < coarseVisits; ++visit) executeCycle(kind, coarser, ops, visit == 0);
    ops.prolong(level);
    ops.postSmooth(level);
}

}  // namespace thermofem::multigrid
