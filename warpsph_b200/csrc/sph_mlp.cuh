// Learned warm-start network: layout constants, packed weights, kernel args.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "sph_internal.cuh"

namespace sph {

constexpr int kH = 64;        // hidden width
// largest rise of asinh(p / (rho0 g h)) over the previous step's value that
// the warm start may predict
constexpr float kMaxRise = SPH_MLP_MAX_RISE;
constexpr int kIn = 16;       // kFeatures padded to one k-tile
constexpr int kW1Pitch = 24;  // row pitch (bf16) of w1f: 8 rows hit 8 distinct bank groups
constexpr int kWPitch = 72;   // row pitch (bf16) of the 64-wide matrices

// Parameter order inside the FP32 blob's parameter block and the gradient
// vector (SPH_MLP_* in include/wpsph.h):  W1 [11][64] (in, out), b1 [64],
// W2 [64][64] (in, out), b2 [64], w3 [64], b3.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kFeatures * kH;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH;
constexpr int kNumParams = kOffB3 + 1;  // 4993
constexpr int kOffLoss = kNumParams;    // gradient vector slot holding the loss
constexpr int kGradStride = kNumParams + 3;
// FP32 blob: mu[11], sd[11], t_scale, then the parameters.
constexpr int kBlobMu = 0;
constexpr int kBlobSd = kBlobMu + kFeatures;
constexpr int kBlobTScale = kBlobSd + kFeatures;
constexpr int kBlobParams = kBlobTScale + 1;
constexpr int kBlobSize = kBlobParams + kNumParams;  // 5016

// Weights as the kernels read them (bf16 matrices in fragment-friendly layouts).
struct MlpPacked {
  __nv_bfloat16 w1f[kH][kW1Pitch];  // [out][in]   forward B of layer 1
  __nv_bfloat16 w2f[kH][kWPitch];   // [out][in]   forward B of layer 2
  __nv_bfloat16 w2b[kH][kWPitch];   // [in][out]   backward B (dH1 = dZ2 W2^T)
  __nv_bfloat16 w3f[8][kWPitch];    // [out][in], row 0 = w3, rows 1..7 zero
  float b1[kH], b2[kH], b3;
  float mu[kIn], inv_sd[kIn];
  float t_scale;
};

struct MlpInferArgs {
  long long n;
  const MlpPacked* w;
  const float* feat;      // raw features: row-major n x kFeatures, or feature-major (feat_ld > 0)
  long long feat_ld;      // > 0: feature c of row r at feat[c * feat_ld + r]
  const float* rho;
  float p_unit;           // rho0 g h: pressure of one target unit
  float* p0;              // out: initial pressure
  float4* pos_q;          // out: .w = p0 / rho^2 of each sorted position record
  float* pred;            // optional out: raw network output
  int* flags;             // optional: SPH_F_TIMEOUT if a tensor-core wait ran out
  int withhold_mma;       // test hook: issue no MMA, so the first wait runs out
  const float* pprev;     // optional: previous-step pressure, sorted
  const int* restart;     // optional, per scene: 1 = start from pprev, not the prediction
  const SceneTable* scenes;  // scene of each row (null: one scene)
};

struct MlpGradArgs {
  long long n;
  const MlpPacked* w;
  const float* feat;      // n x kFeatures
  const float* target;    // n, in units of t_scale
  float* part;            // [gridDim.x][kGradStride]
};

struct MlpAdamArgs {
  const float* part;
  int nblocks;
  float* grad_out;        // optional kGradStride
  float* loss_out;        // optional
  float* master;          // blob (FP32); NULL = gradient only
  float* m;
  float* v;
  float lr, beta1, beta2, eps, beta1_t, beta2_t;  // beta*_t = beta^step
};

size_t mlp_grad_smem();
cudaError_t launch_mlp_pack(const float* blob, MlpPacked* out, cudaStream_t s);
cudaError_t launch_mlp_infer_tc(const MlpInferArgs& a, int sm_count, cudaStream_t s);  // tcgen05
cudaError_t launch_mlp_grad(const MlpGradArgs& a, int nblocks, cudaStream_t s);
cudaError_t launch_mlp_reduce_adam(const MlpAdamArgs& a, cudaStream_t s);
cudaError_t launch_gather_rows(long long n, const int* idx, const float* feat, const float* target,
                               float* feat_out, float* target_out, cudaStream_t s);

}  // namespace sph
