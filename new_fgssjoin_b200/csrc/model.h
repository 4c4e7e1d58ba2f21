// model.h -- the learned cost model of the batched method: a 2-layer FP32 MLP
// (kFeat inputs -> kHidden ReLU -> 2 outputs) predicting, per query record,
// the log of the expected number of candidates it must verify and of result
// pairs it emits (Poisson regression on the exact counts).
// Training and inference are our own CUDA kernels (model.cu).  The model is
// advisory only: it sizes the result buffers and balances work items; an
// undersized buffer is detected on the device and the join re-runs exactly.
#pragma once

#include <stdint.h>

#include <vector>

#include "ctx.h"
#include "tiles.cuh"

namespace fgss {

constexpr int kHidden = 32;
constexpr int kOut = 2;
constexpr int kFeatM = 8;  // equals kFeat in join.h
// parameter block: W1[H][F] b1[H] W2[O][H] b2[O] calib[O]
constexpr int kParams = kHidden * kFeatM + kHidden + kOut * kHidden + kOut;
constexpr int kParamsAll = kParams + kOut;

}  // namespace fgss

struct fgss_model {
    std::vector<float> host;   // kParamsAll floats
    float* dev = nullptr;      // device copy
    float last_loss = 0.f;
    int trained = 0;
};

namespace fgss {

// pred[q] <- predicted candidates (u32); *res_sum += sum of predicted results (x calib);
// *cand_sum += sum of pred (when given)
void model_predict(Ctx& c, const float* feat, uint64_t n, uint32_t* pred, uint64_t* res_sum,
                   uint64_t* cand_sum = nullptr);
// The prediction for every join of a batch (tiles of 256 of its records):
// res_sums[j] / cand_sums[j] += join j's sums.
void model_predict_tiles(Ctx& c, const float* feat, const TileMap& m, uint32_t* pred, uint64_t* res_sums,
                         uint64_t* cand_sums);
// *out += sum of cost[0..n)
void model_sum_cost(Ctx& c, const uint32_t* cost, uint64_t n, uint64_t* out);
// Full-batch Adam training on (feat, target) rows already on the device;
// target rows are (log1p candidates, log1p results).  Returns the final loss.
float model_fit(Ctx& c, const float* feat, const float* target, uint64_t n, int epochs, float lr, uint64_t seed);
// One gradient evaluation (for tests): params (kParams) -> grads (kParams), returns loss.
float model_grad(Ctx& c, const float* feat, const float* target, uint64_t n, const float* params, float* grads);

}  // namespace fgss
