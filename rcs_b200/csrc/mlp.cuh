// Rank model: a 6 -> 64 -> 64 -> 1 perceptron (ReLU hidden layers) that
// predicts log2(1 + rank) of a box's ACA skeleton from six features of the
// box and its interaction list.  The solver uses the prediction to size the
// ACA workspace of each box before the launch; the adaptive ACA
// (ACA.cpp:639-859) still decides the rank, and reruns a box with a larger
// workspace whenever the prediction was too small.
#pragma once
#include <vector>

#include "context.cuh"

namespace aifmm {

constexpr int MLP_IN = 6, MLP_H = 64;
// Parameter vector (FP32 master copy), in this order:
//   W1 [MLP_H x MLP_IN] row-major, b1 [MLP_H], W2 [MLP_H x MLP_H] row-major
//   (output unit, input unit), b2 [MLP_H], w3 [MLP_H], b3 [1].
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H,
              MLP_B2 = MLP_W2 + MLP_H * MLP_H, MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H,
              MLP_NP = MLP_B3 + 1;

// Raw features of one ACA problem (box k at level j against its interaction
// list): mean centre distance to the interaction-list boxes over the box side,
// wavenumber times the box side, log2(1 + rows), log2(1 + columns), the
// level, and 1 for a leaf.
struct RankFeatures {
  float f[MLP_IN];
};

}  // namespace aifmm

struct aifmm_mlp {
  aifmm_ctx* ctx = nullptr;
  std::vector<float> params;          // FP32 master weights (host copy, authoritative between calls)
  float mean[aifmm::MLP_IN] = {0, 0, 0, 0, 0, 0};
  float scale[aifmm::MLP_IN] = {1, 1, 1, 1, 1, 1};
  // Adam moments of the last training run
  std::vector<float> m1, m2;
  long adamStep = 0;
};

namespace aifmm {
// Predicted log2(1 + rank) for n feature rows (raw features; the model's
// normalisation is applied on the device).  Stream-ordered on the context.
void mlp_infer(aifmm_mlp* m, const std::vector<RankFeatures>& x, std::vector<float>& y);
}  // namespace aifmm
