// C ABI of the learned warm-start network: training (Adam over shuffled
// minibatches) and evaluation (predictions + the mean-loss gradient, used to
// check the backward kernel against the CPU oracle).  No counterpart in the
// reference, whose pressure solve always starts from p = 0 (IISPH.py:166-174).
#include <algorithm>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "sph_mlp.cuh"

namespace {

struct Buffers {
  std::vector<void*> ptrs;
  ~Buffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t alloc(T*& p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(count, 1));
    if (e == cudaSuccess) ptrs.push_back(q);
    p = static_cast<T*>(q);
    return e;
  }
};

#define CKR(expr)                                  \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) {                       \
      cudaGetLastError();                          \
      return e_ == cudaErrorMemoryAllocation ? SPH_E_NOMEM : SPH_E_CUDA; \
    }                                              \
  } while (0)

int grad_blocks(long long rows, int sm_count) {
  long long b = (rows + 63) / 64;
  return int(std::max<long long>(1, std::min<long long>(b, 2ll * sm_count)));
}

}  // namespace

extern "C" {

int sph_mlp_train(const SphMlpTrainConfig* cfg, const float* feat, const float* target, int64_t n, float* blob,
                  float* epoch_loss) {
  using namespace sph;
  if (!cfg || !feat || !target || !blob || n <= 0 || cfg->epochs < 0 || cfg->batch < 16) return SPH_E_INVALID;
  if (!(blob[kBlobTScale] > 0)) return SPH_E_INVALID;
  for (int c = 0; c < kFeatures; ++c)
    if (!(blob[kBlobSd + c] > 0)) return SPH_E_INVALID;
  CKR(cudaSetDevice(cfg->device));
  int sm = 0;
  CKR(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, cfg->device));
  cudaStream_t s = nullptr;
  CKR(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{s};
  Buffers B;
  float *d_feat, *d_t, *d_bf, *d_bt, *d_master, *d_m, *d_v, *d_part, *d_loss;
  int* d_idx;
  MlpPacked* d_w;
  const long long batch = std::min<long long>(cfg->batch, n);
  const int nb = grad_blocks(batch, sm);
  CKR(B.alloc(d_feat, size_t(n) * kFeatures));
  CKR(B.alloc(d_t, size_t(n)));
  CKR(B.alloc(d_idx, size_t(n)));
  CKR(B.alloc(d_bf, size_t(batch) * kFeatures));
  CKR(B.alloc(d_bt, size_t(batch)));
  CKR(B.alloc(d_master, kBlobSize));
  CKR(B.alloc(d_m, kGradStride));
  CKR(B.alloc(d_v, kGradStride));
  CKR(B.alloc(d_part, size_t(nb) * kGradStride));
  CKR(B.alloc(d_loss, 1));
  CKR(B.alloc(d_w, 1));
  // targets in units of t_scale
  std::vector<float> tn(n);
  const float inv_ts = 1.0f / blob[kBlobTScale];
  for (int64_t i = 0; i < n; ++i) tn[i] = target[i] * inv_ts;
  CKR(cudaMemcpyAsync(d_feat, feat, sizeof(float) * n * kFeatures, cudaMemcpyHostToDevice, s));
  CKR(cudaMemcpyAsync(d_t, tn.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
  CKR(cudaMemcpyAsync(d_master, blob, sizeof(float) * kBlobSize, cudaMemcpyHostToDevice, s));
  CKR(cudaMemsetAsync(d_m, 0, sizeof(float) * kGradStride, s));
  CKR(cudaMemsetAsync(d_v, 0, sizeof(float) * kGradStride, s));
  CKR(launch_mlp_pack(d_master, d_w, s));

  std::mt19937_64 rng(cfg->seed);
  std::vector<int> perm(n);
  long long step = 0;
  double b1t = 1.0, b2t = 1.0;
  for (int ep = 0; ep < cfg->epochs; ++ep) {
    std::iota(perm.begin(), perm.end(), 0);
    std::shuffle(perm.begin(), perm.end(), rng);
    CKR(cudaMemcpyAsync(d_idx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    double loss_sum = 0.0;
    long long nbatches = 0;
    for (long long off = 0; off < n; off += batch) {
      const long long rows = std::min<long long>(batch, n - off);
      CKR(launch_gather_rows(rows, d_idx + off, d_feat, d_t, d_bf, d_bt, s));
      MlpGradArgs ga{rows, d_w, d_bf, d_bt, d_part};
      const int blocks = grad_blocks(rows, sm);
      CKR(launch_mlp_grad(ga, blocks, s));
      ++step;
      b1t *= cfg->beta1;
      b2t *= cfg->beta2;
      MlpAdamArgs aa{};
      aa.part = d_part;
      aa.nblocks = blocks;
      aa.loss_out = d_loss;
      aa.master = d_master;
      aa.m = d_m;
      aa.v = d_v;
      aa.lr = cfg->lr;
      aa.beta1 = cfg->beta1;
      aa.beta2 = cfg->beta2;
      aa.eps = cfg->eps;
      aa.beta1_t = float(b1t);
      aa.beta2_t = float(b2t);
      CKR(launch_mlp_reduce_adam(aa, s));
      CKR(launch_mlp_pack(d_master, d_w, s));
      if (epoch_loss) {
        float l = 0.f;
        CKR(cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        CKR(cudaStreamSynchronize(s));
        loss_sum += double(l);
      }
      ++nbatches;
    }
    if (epoch_loss) epoch_loss[ep] = float(loss_sum / double(std::max<long long>(nbatches, 1)));
  }
  CKR(cudaMemcpyAsync(blob, d_master, sizeof(float) * kBlobSize, cudaMemcpyDeviceToHost, s));
  CKR(cudaStreamSynchronize(s));
  return SPH_OK;
}

int sph_mlp_eval(const float* blob, const float* feat, const float* target, int64_t n, int32_t device,
                 float* pred, float* grad) {
  using namespace sph;
  if (!blob || !feat || n <= 0) return SPH_E_INVALID;
  CKR(cudaSetDevice(device));
  int sm = 0;
  CKR(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device));
  Buffers B;
  float *d_blob, *d_feat, *d_t = nullptr, *d_pred, *d_part, *d_grad;
  MlpPacked* d_w;
  const int nb = grad_blocks(n, sm);
  CKR(B.alloc(d_blob, kBlobSize));
  CKR(B.alloc(d_feat, size_t(n) * kFeatures));
  CKR(B.alloc(d_pred, size_t(n)));
  CKR(B.alloc(d_part, size_t(nb) * kGradStride));
  CKR(B.alloc(d_grad, kGradStride));
  CKR(B.alloc(d_w, 1));
  CKR(cudaMemcpy(d_blob, blob, sizeof(float) * kBlobSize, cudaMemcpyHostToDevice));
  CKR(cudaMemcpy(d_feat, feat, sizeof(float) * n * kFeatures, cudaMemcpyHostToDevice));
  CKR(launch_mlp_pack(d_blob, d_w, nullptr));
  int* d_flags;
  CKR(B.alloc(d_flags, 1));
  CKR(cudaMemset(d_flags, 0, sizeof(int)));
  MlpInferArgs ia{};
  ia.n = n;
  ia.w = d_w;
  ia.feat = d_feat;
  ia.pred = d_pred;
  ia.flags = d_flags;
  CKR(launch_mlp_infer_tc(ia, sm, nullptr));  // the step's inference kernel
  int flags = 0;
  CKR(cudaMemcpy(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost));
  if (flags & SPH_F_TIMEOUT) return SPH_E_TIMEOUT;
  if (pred) CKR(cudaMemcpy(pred, d_pred, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (grad) {
    if (!target) return SPH_E_INVALID;
    std::vector<float> tn(n);
    const float inv_ts = 1.0f / blob[kBlobTScale];
    for (int64_t i = 0; i < n; ++i) tn[i] = target[i] * inv_ts;
    CKR(B.alloc(d_t, size_t(n)));
    CKR(cudaMemcpy(d_t, tn.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    MlpGradArgs ga{n, d_w, d_feat, d_t, d_part};
    CKR(launch_mlp_grad(ga, nb, nullptr));
    MlpAdamArgs aa{};
    aa.part = d_part;
    aa.nblocks = nb;
    aa.grad_out = d_grad;
    CKR(launch_mlp_reduce_adam(aa, nullptr));
    CKR(cudaMemcpy(grad, d_grad, sizeof(float) * (kNumParams + 1), cudaMemcpyDeviceToHost));
  }
  CKR(cudaDeviceSynchronize());
  return SPH_OK;
}

}  // extern "C"
