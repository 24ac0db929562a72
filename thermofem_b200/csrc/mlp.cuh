// mlp.cuh -- learned per-row Jacobi damping (mlp.cu).
#pragma once
#include <memory>
#include <vector>

#include "ops.cuh"
#include "tile.cuh"

namespace tfb {

// A trained damping network as a hierarchy uses it: BF16 weights in the
// layout of tf_mlp (W1[32][4], b1[32], w2[32], b2) and the output bounds.
struct DampingModel {
    std::vector<uint16_t> bf16;
    float omega_min{0}, omega_max{0};
};

// Snapshot of a model's current weights (nullptr for a null model).
std::shared_ptr<const DampingModel> damping_model_of(const tf_mlp *m);

// n x 4 row features of a level operator (mlp.cu header comment).
template <class T, class I>
void row_features(tf_ctx *ctx, const Csr<T, I> &a, int level, float *out);

// dinv_i *= omega_i = model(features of row i at `level`).
template <class T, class I>
void learned_damping(tf_ctx *ctx, const DampingModel &m, const Csr<T, I> &a, int level, T *dinv);

}  // namespace tfb
