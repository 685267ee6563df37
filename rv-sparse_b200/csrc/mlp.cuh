// Row-size predictor: a 4-32-32-2 ReLU MLP over cheap per-row features.
//
// Features (per output row i, from the analysis pass): A-row nnz, the sum of
// the referenced B-row lengths (= intermediate products), their maximum, and
// the column span [first, last] those B rows cover. Each feature f enters as
// (log2(1 + f) - mean) / std with mean/std fixed by the training data.
// Outputs: mu = predicted log2(1 + nnz(C_i)) and s, the raw scale of a
// Gaussian on that log size, sigma = softplus(s) + 1e-3. The capacity used
// for row i is ceil(2^(mu + z * sigma) - 1), clamped to [1, ub_i] with
// ub_i = min(products, cols(B)); z is the stored safety quantile.
//
// Training minimises the Gaussian negative log-likelihood
//   w * (0.5 * ((y - mu) / sigma)^2 + log sigma)
// with Adam, on exact counts produced by the library's own exact path.

#pragma once

#include <cstdint>

namespace rvsp {

constexpr int MLP_IN = 4;
constexpr int MLP_H = 32;
constexpr int MLP_OUT = 2;
// parameter layout (floats)
constexpr int MLP_W1 = 0;                          // [H][IN]
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;    // [H]
constexpr int MLP_W2 = MLP_B1 + MLP_H;             // [H][H]
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;     // [H]
constexpr int MLP_W3 = MLP_B2 + MLP_H;             // [OUT][H]
constexpr int MLP_B3 = MLP_W3 + MLP_OUT * MLP_H;   // [OUT]
constexpr int MLP_NPARAM = MLP_B3 + MLP_OUT;       // 1282

// Model as stored in a checkpoint: normalisation, safety quantile, weights.
struct MlpModel {
    float mean[MLP_IN];
    float inv_std[MLP_IN];
    float z;
    float params[MLP_NPARAM];
};

__host__ __device__ inline float mlp_softplus(float s) {
    return s > 20.0f ? s : log1pf(expf(s));
}

}  // namespace rvsp
