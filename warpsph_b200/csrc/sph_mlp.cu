// Learned pressure warm start: a per-particle MLP 10 -> 64 -> 64 -> 1 (ReLU),
// BF16 operands on the tensor cores with FP32 accumulation: the training
// forward/backward here use warp-level mma.sync m16n8k16 tiles, the Adam
// update runs on the CUDA cores, and the inference the step runs is the
// tcgen05 kernel of sph_mlp_tc.cu (same BF16 rounding points).
//
// The network only proposes the Jacobi starting pressure p_0; the unchanged
// relaxed-Jacobi loop (IISPH.py:1200-1296) still decides convergence, so a bad
// prediction costs iterations, never accuracy.
//
// Fragment conventions of mma.m16n8k16 (g = lane / 4, t = lane % 4):
//   A (16x16, row-major): a0 (g, 2t..2t+1), a1 (g+8, 2t..), a2 (g, 2t+8..), a3 (g+8, 2t+8..)
//   B (16x8, k-major):    b0 (k = 2t..2t+1, n = g), b1 (k = 2t+8..2t+9, n = g)
//   C (16x8):             c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1)
// Two neighbouring C tiles (columns 16k..16k+15) are exactly the A fragment of
// k-tile k for the next layer, so hidden activations never leave registers in
// the forward pass.
#include <cuda_bf16.h>

#include "sph_internal.cuh"
#include "sph_mlp.cuh"

namespace sph {

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

using MlpSmem = MlpPacked;

__device__ __forceinline__ void load_weights(MlpSmem& s, const MlpPacked* __restrict__ w) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(w);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&s);
  constexpr int words = sizeof(MlpSmem) / 4;
  for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
}

// Forward pass of one warp over 16 rows.  x[r][c] = standardised features of
// row r (rows g and g+8 of this lane), columns 2t, 2t+1, 2t+8, 2t+9.
struct Fwd {
  float z1[8][4];  // layer-1 pre-activations (C layout)
  float z2[8][4];  // layer-2 pre-activations
  uint32_t h1[4][4], h2[4][4];  // bf16 A fragments of relu(z1), relu(z2)
  float y[4];      // output tile (column 0 valid)
};

__device__ __forceinline__ void forward(const MlpSmem& s, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                        Fwd& f) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float* d = f.z1[nt];
    d[0] = d[1] = d[2] = d[3] = 0.f;
    mma_bf16(f.z1[nt], a0, a1, a2, a3, lds32(&s.w1f[8 * nt + g][2 * t]), lds32(&s.w1f[8 * nt + g][2 * t + 8]));
    const float b0 = s.b1[8 * nt + 2 * t], b1 = s.b1[8 * nt + 2 * t + 1];
    d[0] += b0;
    d[1] += b1;
    d[2] += b0;
    d[3] += b1;
  }
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const float* c0 = f.z1[2 * kt];
    const float* c1 = f.z1[2 * kt + 1];
    f.h1[kt][0] = pack_bf16(fmaxf(c0[0], 0.f), fmaxf(c0[1], 0.f));
    f.h1[kt][1] = pack_bf16(fmaxf(c0[2], 0.f), fmaxf(c0[3], 0.f));
    f.h1[kt][2] = pack_bf16(fmaxf(c1[0], 0.f), fmaxf(c1[1], 0.f));
    f.h1[kt][3] = pack_bf16(fmaxf(c1[2], 0.f), fmaxf(c1[3], 0.f));
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float* d = f.z2[nt];
    d[0] = d[1] = d[2] = d[3] = 0.f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
      mma_bf16(f.z2[nt], f.h1[kt][0], f.h1[kt][1], f.h1[kt][2], f.h1[kt][3], lds32(&s.w2f[8 * nt + g][16 * kt + 2 * t]),
               lds32(&s.w2f[8 * nt + g][16 * kt + 2 * t + 8]));
    const float b0 = s.b2[8 * nt + 2 * t], b1 = s.b2[8 * nt + 2 * t + 1];
    d[0] += b0;
    d[1] += b1;
    d[2] += b0;
    d[3] += b1;
  }
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const float* c0 = f.z2[2 * kt];
    const float* c1 = f.z2[2 * kt + 1];
    f.h2[kt][0] = pack_bf16(fmaxf(c0[0], 0.f), fmaxf(c0[1], 0.f));
    f.h2[kt][1] = pack_bf16(fmaxf(c0[2], 0.f), fmaxf(c0[3], 0.f));
    f.h2[kt][2] = pack_bf16(fmaxf(c1[0], 0.f), fmaxf(c1[1], 0.f));
    f.h2[kt][3] = pack_bf16(fmaxf(c1[2], 0.f), fmaxf(c1[3], 0.f));
  }
  f.y[0] = f.y[1] = f.y[2] = f.y[3] = 0.f;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt)
    mma_bf16(f.y, f.h2[kt][0], f.h2[kt][1], f.h2[kt][2], f.h2[kt][3], lds32(&s.w3f[g][16 * kt + 2 * t]),
             lds32(&s.w3f[g][16 * kt + 2 * t + 8]));
  f.y[0] += s.b3;
  f.y[2] += s.b3;
}

// A fragment of the standardised feature tile of rows r0 (= g) and r0 + 8.
__device__ __forceinline__ void feature_frag(const MlpSmem& s, const float* __restrict__ feat, long long row0,
                                             long long nrows, uint32_t& a0, uint32_t& a1, uint32_t& a2,
                                             uint32_t& a3, float (*xs)[4] = nullptr) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float v[2][4];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const long long r = row0 + g + 8 * h;
    const int cols[4] = {2 * t, 2 * t + 1, 2 * t + 8, 2 * t + 9};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = cols[q];
      float x = 0.f;
      if (r < nrows && c < kFeatures) x = (__ldg(feat + r * kFeatures + c) - s.mu[c]) * s.inv_sd[c];
      v[h][q] = x;
    }
  }
  a0 = pack_bf16(v[0][0], v[0][1]);
  a1 = pack_bf16(v[1][0], v[1][1]);
  a2 = pack_bf16(v[0][2], v[0][3]);
  a3 = pack_bf16(v[1][2], v[1][3]);
  if (xs) {
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < 4; ++q) xs[h][q] = bf16r(v[h][q]);
  }
}

// ------------------------------------------------------------------ training

// Forward + backward over the batch; every block writes its partial gradient
// (and loss) to part[blockIdx.x], reduced in block order by k_mlp_adam.
// Gradients are of  L = mean_r (y_r - target_r)^2  over the n rows.
struct GradSmem {
  MlpSmem s;
  __nv_bfloat16 xT[kIn][64 + 8];   // [feature][sample]
  __nv_bfloat16 h1T[kH][64 + 8];   // [unit][sample]
  __nv_bfloat16 dz1T[kH][64 + 8];
  __nv_bfloat16 dz2T[kH][64 + 8];
  float red[4][3 * kH + 2];        // per warp: db1, db2, dw3, db3, loss
};

size_t mlp_grad_smem() { return sizeof(GradSmem); }

__global__ void __launch_bounds__(128) k_mlp_grad(MlpGradArgs a) {
  extern __shared__ __align__(16) unsigned char dsm[];
  GradSmem& G = *reinterpret_cast<GradSmem*>(dsm);
  MlpSmem& s = G.s;
  auto& xT = G.xT;
  auto& h1T = G.h1T;
  auto& dz1T = G.dz1T;
  auto& dz2T = G.dz2T;
  auto& red = G.red;
  load_weights(s, a.w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float acc_w2[8][4], acc_w1[2][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) acc_w2[nt][0] = acc_w2[nt][1] = acc_w2[nt][2] = acc_w2[nt][3] = 0.f;
#pragma unroll
  for (int q = 0; q < 2; ++q) acc_w1[q][0] = acc_w1[q][1] = acc_w1[q][2] = acc_w1[q][3] = 0.f;
  float acc_b3 = 0.f, acc_loss = 0.f;
  for (int k = threadIdx.x; k < 4 * (3 * kH + 2); k += blockDim.x) (&red[0][0])[k] = 0.f;
  __syncthreads();
  // column sums over the 16 rows of the tile (lanes with equal t), added to this warp's slots
  auto colsum = [&](float v0, float v1, int base, int nt) {
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) {
      v0 += __shfl_xor_sync(0xffffffffu, v0, o);
      v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    }
    if (g == 0) {
      red[warp][base + 8 * nt + 2 * t] += v0;
      red[warp][base + 8 * nt + 2 * t + 1] += v1;
    }
  };
  const float inv_n = 1.0f / float(a.n);

  for (long long base = (long long)blockIdx.x * 64; base < a.n; base += (long long)gridDim.x * 64) {
    const long long r0 = base + 16 * warp;
    uint32_t a0, a1, a2, a3;
    float xs[2][4];
    feature_frag(s, a.feat, r0, a.n, a0, a1, a2, a3, xs);
    Fwd f;
    forward(s, a0, a1, a2, a3, f);
    // loss gradient dy for rows g, g+8 (held by lane t == 0, broadcast to the quad)
    float dy[2] = {0.f, 0.f};
    if (t == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long r = r0 + g + 8 * h;
        if (r < a.n) {
          const float e = f.y[2 * h] - __ldg(a.target + r);
          acc_loss += e * e;
          dy[h] = 2.0f * e * inv_n;
        }
      }
    }
    dy[0] = __shfl_sync(0xffffffffu, dy[0], lane & ~3);
    dy[1] = __shfl_sync(0xffffffffu, dy[1], lane & ~3);
    if (t == 0) acc_b3 += dy[0] + dy[1];
    // layer 3: dW3 += h2^T dy ; dZ2 = (dy w3^T) * relu'(z2)
    float dz2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      const float w3a = __bfloat162float(s.w3f[0][c]), w3b = __bfloat162float(s.w3f[0][c + 1]);
      const float* z = f.z2[nt];
      colsum(bf16r(fmaxf(z[0], 0.f)) * dy[0] + bf16r(fmaxf(z[2], 0.f)) * dy[1],
             bf16r(fmaxf(z[1], 0.f)) * dy[0] + bf16r(fmaxf(z[3], 0.f)) * dy[1], 2 * kH, nt);
      dz2[nt][0] = z[0] > 0.f ? dy[0] * w3a : 0.f;
      dz2[nt][1] = z[1] > 0.f ? dy[0] * w3b : 0.f;
      dz2[nt][2] = z[2] > 0.f ? dy[1] * w3a : 0.f;
      dz2[nt][3] = z[3] > 0.f ? dy[1] * w3b : 0.f;
      colsum(dz2[nt][0] + dz2[nt][2], dz2[nt][1] + dz2[nt][3], kH, nt);
    }
    // layer 2 input gradient: dH1 = bf16(dZ2) W2^T ; dZ1 = dH1 * relu'(z1)
    uint32_t gz2[4][4];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      gz2[kt][0] = pack_bf16(dz2[2 * kt][0], dz2[2 * kt][1]);
      gz2[kt][1] = pack_bf16(dz2[2 * kt][2], dz2[2 * kt][3]);
      gz2[kt][2] = pack_bf16(dz2[2 * kt + 1][0], dz2[2 * kt + 1][1]);
      gz2[kt][3] = pack_bf16(dz2[2 * kt + 1][2], dz2[2 * kt + 1][3]);
    }
    float dz1[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kt = 0; kt < 4; ++kt)
        mma_bf16(d, gz2[kt][0], gz2[kt][1], gz2[kt][2], gz2[kt][3], lds32(&s.w2b[8 * nt + g][16 * kt + 2 * t]),
                 lds32(&s.w2b[8 * nt + g][16 * kt + 2 * t + 8]));
      const float* z = f.z1[nt];
      dz1[nt][0] = z[0] > 0.f ? d[0] : 0.f;
      dz1[nt][1] = z[1] > 0.f ? d[1] : 0.f;
      dz1[nt][2] = z[2] > 0.f ? d[2] : 0.f;
      dz1[nt][3] = z[3] > 0.f ? d[3] : 0.f;
      colsum(dz1[nt][0] + dz1[nt][2], dz1[nt][1] + dz1[nt][3], 0, nt);
    }
    // stage transposed bf16 operands of the weight-gradient products
    const int sr = 16 * warp + g;  // block-local sample rows sr, sr + 8
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      const float* z = f.z1[nt];
      h1T[c][sr] = __float2bfloat16_rn(fmaxf(z[0], 0.f));
      h1T[c + 1][sr] = __float2bfloat16_rn(fmaxf(z[1], 0.f));
      h1T[c][sr + 8] = __float2bfloat16_rn(fmaxf(z[2], 0.f));
      h1T[c + 1][sr + 8] = __float2bfloat16_rn(fmaxf(z[3], 0.f));
      dz2T[c][sr] = __float2bfloat16_rn(dz2[nt][0]);
      dz2T[c + 1][sr] = __float2bfloat16_rn(dz2[nt][1]);
      dz2T[c][sr + 8] = __float2bfloat16_rn(dz2[nt][2]);
      dz2T[c + 1][sr + 8] = __float2bfloat16_rn(dz2[nt][3]);
      dz1T[c][sr] = __float2bfloat16_rn(dz1[nt][0]);
      dz1T[c + 1][sr] = __float2bfloat16_rn(dz1[nt][1]);
      dz1T[c][sr + 8] = __float2bfloat16_rn(dz1[nt][2]);
      dz1T[c + 1][sr + 8] = __float2bfloat16_rn(dz1[nt][3]);
    }
    {
      const int cols[4] = {2 * t, 2 * t + 1, 2 * t + 8, 2 * t + 9};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        xT[cols[q]][sr] = __float2bfloat16_rn(xs[0][q]);
        xT[cols[q]][sr + 8] = __float2bfloat16_rn(xs[1][q]);
      }
    }
    __syncthreads();
    // dW2 rows [16w, 16w+16) = h1T[rows][samples] . dz2T[cols][samples]^T over the block's 64 samples
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      const int m = 16 * warp + g, k = 16 * kt + 2 * t;
      const uint32_t b_a0 = lds32(&h1T[m][k]), b_a1 = lds32(&h1T[m + 8][k]);
      const uint32_t b_a2 = lds32(&h1T[m][k + 8]), b_a3 = lds32(&h1T[m + 8][k + 8]);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt)
        mma_bf16(acc_w2[nt], b_a0, b_a1, b_a2, b_a3, lds32(&dz2T[8 * nt + g][k]), lds32(&dz2T[8 * nt + g][k + 8]));
    }
    // dW1 (16 x 64, rows = features): this warp's columns [16w, 16w+16)
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      const int k = 16 * kt + 2 * t;
      const uint32_t x0 = lds32(&xT[g][k]), x1 = lds32(&xT[g + 8][k]);
      const uint32_t x2 = lds32(&xT[g][k + 8]), x3 = lds32(&xT[g + 8][k + 8]);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int n = 16 * warp + 8 * q + g;
        mma_bf16(acc_w1[q], x0, x1, x2, x3, lds32(&dz1T[n][k]), lds32(&dz1T[n][k + 8]));
      }
    }
    __syncthreads();
  }

  // per-warp totals of the scalar gradients
#pragma unroll
  for (int o = 4; o < 32; o <<= 1) {
    acc_b3 += __shfl_xor_sync(0xffffffffu, acc_b3, o);
    acc_loss += __shfl_xor_sync(0xffffffffu, acc_loss, o);
  }
  if (lane == 0) {
    red[warp][3 * kH] = acc_b3;
    red[warp][3 * kH + 1] = acc_loss;
  }
  __syncthreads();
  float* out = a.part + (long long)blockIdx.x * kGradStride;
  for (int k = threadIdx.x; k < 3 * kH + 2; k += blockDim.x) {
    const float v = ((red[0][k] + red[1][k]) + red[2][k]) + red[3][k];
    if (k < kH) out[kOffB1 + k] = v;
    else if (k < 2 * kH) out[kOffB2 + k - kH] = v;
    else if (k < 3 * kH) out[kOffW3 + k - 2 * kH] = v;
    else if (k == 3 * kH) out[kOffB3] = v;
    else out[kOffLoss] = v * inv_n;
  }
  // dW2 tile of this warp (rows 16w+g, +8; cols 8nt+2t, +1), dW1 rows (features) g, g+8
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int r = 16 * warp + g, c = 8 * nt + 2 * t;
    out[kOffW2 + r * kH + c] = acc_w2[nt][0];
    out[kOffW2 + r * kH + c + 1] = acc_w2[nt][1];
    out[kOffW2 + (r + 8) * kH + c] = acc_w2[nt][2];
    out[kOffW2 + (r + 8) * kH + c + 1] = acc_w2[nt][3];
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int c = 16 * warp + 8 * q + 2 * t;
    if (g < kFeatures) {
      out[kOffW1 + g * kH + c] = acc_w1[q][0];
      out[kOffW1 + g * kH + c + 1] = acc_w1[q][1];
    }
    if (g + 8 < kFeatures) {
      out[kOffW1 + (g + 8) * kH + c] = acc_w1[q][2];
      out[kOffW1 + (g + 8) * kH + c + 1] = acc_w1[q][3];
    }
  }
}

// Sum the per-block partial gradients in block order; optionally export the
// gradient, and apply one Adam step to the FP32 master weights.
__global__ void k_mlp_reduce_adam(MlpAdamArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kGradStride) return;
  float gsum = 0.f;
  for (int b = 0; b < a.nblocks; ++b) gsum += a.part[(long long)b * kGradStride + k];
  if (a.grad_out) a.grad_out[k] = gsum;
  if (k == kOffLoss) {
    if (a.loss_out) *a.loss_out = gsum;
    return;
  }
  if (!a.master || k >= kNumParams) return;
  float* w = a.master + kBlobParams + k;
  const float m = a.beta1 * a.m[k] + (1.f - a.beta1) * gsum;
  const float v = a.beta2 * a.v[k] + (1.f - a.beta2) * gsum * gsum;
  a.m[k] = m;
  a.v[k] = v;
  const float mh = m / (1.f - a.beta1_t), vh = v / (1.f - a.beta2_t);
  *w -= a.lr * mh / (sqrtf(vh) + a.eps);
}

// FP32 blob -> packed bf16 device layout (zero padding included).
__global__ void k_mlp_pack(const float* __restrict__ blob, MlpPacked* out) {
  MlpSmem& p = *reinterpret_cast<MlpSmem*>(out);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  const float* W1 = blob + kBlobParams + kOffW1;
  const float* B1 = blob + kBlobParams + kOffB1;
  const float* W2 = blob + kBlobParams + kOffW2;
  const float* B2 = blob + kBlobParams + kOffB2;
  const float* W3 = blob + kBlobParams + kOffW3;
  for (int k = tid; k < kH * kW1Pitch; k += stride) {
    const int o = k / kW1Pitch, i = k % kW1Pitch;
    p.w1f[o][i] = __float2bfloat16_rn(i < kFeatures ? W1[i * kH + o] : 0.f);
  }
  for (int k = tid; k < kH * kWPitch; k += stride) {
    const int r = k / kWPitch, c = k % kWPitch;
    p.w2f[r][c] = __float2bfloat16_rn(c < kH ? W2[c * kH + r] : 0.f);  // [out][in]
    p.w2b[r][c] = __float2bfloat16_rn(c < kH ? W2[r * kH + c] : 0.f);  // [in][out]
  }
  for (int k = tid; k < 8 * kWPitch; k += stride) {
    const int r = k / kWPitch, c = k % kWPitch;
    p.w3f[r][c] = __float2bfloat16_rn((r == 0 && c < kH) ? W3[c] : 0.f);
  }
  for (int k = tid; k < kH; k += stride) {
    p.b1[k] = B1[k];
    p.b2[k] = B2[k];
  }
  for (int k = tid; k < kIn; k += stride) {
    p.mu[k] = k < kFeatures ? blob[kBlobMu + k] : 0.f;
    p.inv_sd[k] = k < kFeatures ? 1.0f / blob[kBlobSd + k] : 0.f;
  }
  if (tid == 0) {
    p.b3 = blob[kBlobParams + kOffB3];
    p.t_scale = blob[kBlobTScale];
  }
}

__global__ void k_gather_rows(long long n, const int* __restrict__ idx, const float* __restrict__ feat,
                              const float* __restrict__ target, float* __restrict__ feat_out,
                              float* __restrict__ target_out) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const long long src = idx[r];
#pragma unroll
  for (int c = 0; c < kFeatures; ++c) feat_out[r * kFeatures + c] = feat[src * kFeatures + c];
  target_out[r] = target[src];
}

cudaError_t launch_gather_rows(long long n, const int* idx, const float* feat, const float* target,
                               float* feat_out, float* target_out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_gather_rows<<<int((n + 255) / 256), 256, 0, s>>>(n, idx, feat, target, feat_out, target_out);
  return cudaGetLastError();
}

cudaError_t launch_mlp_pack(const float* blob, MlpPacked* out, cudaStream_t s) {
  k_mlp_pack<<<8, 256, 0, s>>>(blob, out);
  return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const MlpGradArgs& a, int nblocks, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const size_t smem = sizeof(GradSmem);
  cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  k_mlp_grad<<<nblocks, 128, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_reduce_adam(const MlpAdamArgs& a, cudaStream_t s) {
  k_mlp_reduce_adam<<<(kGradStride + 255) / 256, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace sph
