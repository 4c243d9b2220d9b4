// Warm-start inference on the 5th-generation tensor cores (tcgen05, sm_100a):
// the per-particle MLP 10 -> 64 -> 64 -> 1 over tiles of 128 particles.
//
// Per CTA (128 threads, one particle row per thread): the layer weights sit in
// shared memory once, in the canonical no-swizzle K-major operand layout
// (core matrices of 8 rows x 16 bytes: element (r, k) of an operand with K
// columns at ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// bytes, so the leading byte offset between K-adjacent core matrices is 128
// and the stride byte offset between 8-row groups is K * 16).  One thread
// issues the MMAs; the FP32 accumulators live in tensor memory (TMEM):
//   layer 1  D1[128 x 64] = X[128 x 16] . W1^T     one tcgen05.mma, K = 16
//   layer 2  D2[128 x 64] = H1[128 x 64] . W2^T    four tcgen05.mma, K = 16 each
// (D1 and D2 in the same 64 TMEM columns, one after the other)
// Each thread reads its row of D1 / D2 back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31), adds the bias, applies ReLU and rounds to BF16, exactly
// where the register (mma.sync) kernels round; layer 3 (64 -> 1) is a dot
// product on the CUDA cores.  Completion of the MMAs is signalled through an
// mbarrier (tcgen05.commit); every wait is bounded, and a CTA whose wait runs
// out sets SPH_F_TIMEOUT in the step flags and stops, releasing its TMEM.
#include <cuda_bf16.h>

#include "sph_internal.cuh"
#include "sph_mlp.cuh"

namespace sph {

namespace {

constexpr int kTile = 128;        // particles per MMA (M)
// D1 and D2 share the same 64 TMEM columns: every thread has read D1 (and
// waited for the read) before the barrier that precedes the layer-2 MMA.
// 64 columns per CTA lets 7 CTAs (the shared-memory and register limit) hold
// TMEM on one SM at once (448 of 512 columns).
constexpr uint32_t kTmemCols = 64;
constexpr int kCtasPerSm = 7;

struct __align__(1024) TcSmem {
  __nv_bfloat16 x[kTile * kIn];     // A of layer 1 (K = 16)
  __nv_bfloat16 h1[kTile * kH];     // A of layer 2 (K = 64)
  __nv_bfloat16 w1[kH * kIn];       // B of layer 1: rows n = output, K = input
  __nv_bfloat16 w2[kH * kH];        // B of layer 2
  float b1[kH], b2[kH], w3[kH];
  float mu[kIn], inv_sd[kIn];
  float b3, t_scale;
  unsigned long long mbar;
  uint32_t tmem_base;
};

// Byte offset of element (r, k) in a canonical no-swizzle K-major operand with K columns.
__device__ __forceinline__ uint32_t op_off(int r, int k, int K) {
  return uint32_t((((r >> 3) * (K >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05): start address, leading / stride
// byte offsets (all >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;  // version
  return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major, N, M.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4)                        // D format F32
         | (1u << 7)                      // A format BF16
         | (1u << 10)                     // B format BF16
         | (uint32_t(N >> 3) << 17)       // N / 8
         | (uint32_t(M >> 4) << 24);      // M / 16
}

__device__ __forceinline__ void mma_bf16_tc(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                            uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
        "r"(mask3));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Bounded wait for the mbarrier phase with parity `parity` to complete.  An
// MMA here completes in microseconds; 2^18 polls (each try_wait may suspend
// the thread for a few microseconds) give up after about a second.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 18); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// BF16 pair (lo in the low half) of relu(lo), relu(hi), rounded to nearest
// even in one conversion: for finite values relu commutes with the rounding
// (it keeps signs), so this equals rounding fmaxf(v, 0).
__device__ __forceinline__ uint32_t relu_pack2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// relu(z + b) of 8 consecutive columns, rounded to BF16, as one 16-byte store.
__device__ __forceinline__ void store_relu8(uint8_t* dst, const float* z, const float* b) {
  uint4 q;
  q.x = relu_pack2(z[0] + b[0], z[1] + b[1]);
  q.y = relu_pack2(z[2] + b[2], z[3] + b[3]);
  q.z = relu_pack2(z[4] + b[4], z[5] + b[5]);
  q.w = relu_pack2(z[6] + b[6], z[7] + b[7]);
  *reinterpret_cast<uint4*>(dst) = q;
}

__global__ void __launch_bounds__(kTile) k_mlp_infer_tc(MlpInferArgs a) {
  __shared__ TcSmem s;
  const int tid = threadIdx.x, warp = tid >> 5;
  const MlpPacked* w = a.w;

  // TMEM for both accumulators (warp 0 allocates and, at the end, frees it)
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // weights into the operand layouts
  uint8_t* w1b = reinterpret_cast<uint8_t*>(s.w1);
  uint8_t* w2b = reinterpret_cast<uint8_t*>(s.w2);
  for (int e = tid; e < kH * kIn; e += blockDim.x) {
    const int n = e / kIn, k = e % kIn;
    *reinterpret_cast<__nv_bfloat16*>(w1b + op_off(n, k, kIn)) = w->w1f[n][k];
  }
  for (int e = tid; e < kH * kH; e += blockDim.x) {
    const int n = e / kH, k = e % kH;
    *reinterpret_cast<__nv_bfloat16*>(w2b + op_off(n, k, kH)) = w->w2f[n][k];
  }
  for (int k = tid; k < kH; k += blockDim.x) {
    s.b1[k] = w->b1[k];
    s.b2[k] = w->b2[k];
    s.w3[k] = __bfloat162float(w->w3f[0][k]);
  }
  if (tid < kIn) {
    s.mu[tid] = w->mu[tid];
    s.inv_sd[tid] = w->inv_sd[tid];
  }
  if (tid == 0) {
    s.b3 = w->b3;
    s.t_scale = w->t_scale;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar)));
  }
  fence_async_smem();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();

  const uint32_t tmem = s.tmem_base;
  const uint32_t d1 = tmem, d2 = tmem;
  const uint32_t lane_row = uint32_t(warp * 32) << 16;  // this warp's TMEM lanes
  const uint32_t mbar = smem_u32(&s.mbar);
  constexpr uint32_t idesc = idesc_bf16(kTile, kH);
  const uint32_t x_addr = smem_u32(s.x), h1_addr = smem_u32(s.h1);
  const uint32_t w1_addr = smem_u32(s.w1), w2_addr = smem_u32(s.w2);
  uint8_t* xb = reinterpret_cast<uint8_t*>(s.x);
  uint8_t* hb = reinterpret_cast<uint8_t*>(s.h1);
  uint32_t phase = 0;

  const long long tiles = (a.n + kTile - 1) / kTile;
  // the raw features of this thread's row of the next tile are loaded one
  // tile ahead, so their latency overlaps the current tile's MMAs; in the
  // feature-major layout each of a warp's loads is one coalesced 128-byte row
  // (with the row's density and previous pressure, read by the epilogue)
  float fn[kFeatures], rho_n = 1.f, pprev_n = 0.f;
  const long long cs = a.feat_ld > 0 ? a.feat_ld : 1, rs = a.feat_ld > 0 ? 1 : kFeatures;
  auto load_row = [&](long long tile) {
    const long long r = tile * kTile + tid;
    const bool ok = tile < tiles && r < a.n;
#pragma unroll
    for (int c = 0; c < kFeatures; ++c) fn[c] = ok ? __ldg(a.feat + c * cs + r * rs) : 0.f;
    if (a.p0) rho_n = ok ? __ldg(a.rho + r) : 1.f;
    if (a.pprev) pprev_n = ok ? __ldg(a.pprev + r) : 0.f;
  };
  load_row(blockIdx.x);
  for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const long long row = tile * kTile + tid;
    const bool live = row < a.n;
    // the residual's base, unrounded: the larger of asinh(p_prev / (rho0 g h))
    // and asinh(depth / h), the hydrostatic pressure of the column above
    const float u_prev = fmaxf(fn[3], fn[10]);
    const float rho_row = rho_n, pprev_row = pprev_n;
    // 1. standardised features of this row, BF16, K padded to 16 with zeros
    {
      float f[kIn];
#pragma unroll
      for (int c = 0; c < kIn; ++c) f[c] = (live && c < kFeatures) ? (fn[c < kFeatures ? c : 0] - s.mu[c]) * s.inv_sd[c] : 0.f;
      load_row(tile + gridDim.x);
      uint4 lo, hi;
      lo.x = pack2(f[0], f[1]);
      lo.y = pack2(f[2], f[3]);
      lo.z = pack2(f[4], f[5]);
      lo.w = pack2(f[6], f[7]);
      hi.x = pack2(f[8], f[9]);
      hi.y = pack2(f[10], f[11]);
      hi.z = pack2(f[12], f[13]);
      hi.w = pack2(f[14], f[15]);
      *reinterpret_cast<uint4*>(xb + op_off(tid, 0, kIn)) = lo;
      *reinterpret_cast<uint4*>(xb + op_off(tid, 8, kIn)) = hi;
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    // 2. layer 1 on the tensor cores (the test hook withholds it: nothing is
    // then in flight when the bounded wait below runs out)
    if (tid == 0 && !a.withhold_mma) {
      mma_bf16_tc(d1, smem_desc(x_addr, 128, 16 * 16), smem_desc(w1_addr, 128, 16 * 16), idesc, 0);
      mma_commit(mbar);
    }
    bool ok = mbar_wait(mbar, phase);
    phase ^= 1u;
    tc_after_sync();
    if (!__syncthreads_and(ok)) {
      if (tid == 0 && a.flags) atomicOr(a.flags, SPH_F_TIMEOUT);
      break;
    }
    // 3. bias + ReLU -> BF16 H1 row
    {
      float z[32];
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        tmem_ld32(d1 + lane_row + uint32_t(32 * half), z);
#pragma unroll
        for (int g = 0; g < 4; ++g)
          store_relu8(hb + op_off(tid, 32 * half + 8 * g, kH), z + 8 * g, s.b1 + 32 * half + 8 * g);
      }
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    // 4. layer 2 on the tensor cores: four K = 16 steps (2 core matrices = 256 bytes each)
    if (tid == 0) {
#pragma unroll
      for (int ks = 0; ks < kH / 16; ++ks)
        mma_bf16_tc(d2, smem_desc(h1_addr + 256u * ks, 128, 64 * 16), smem_desc(w2_addr + 256u * ks, 128, 64 * 16),
                    idesc, ks > 0 ? 1u : 0u);
      mma_commit(mbar);
    }
    ok = mbar_wait(mbar, phase);
    phase ^= 1u;
    tc_after_sync();
    if (!__syncthreads_and(ok)) {
      if (tid == 0 && a.flags) atomicOr(a.flags, SPH_F_TIMEOUT);
      break;
    }
    // 5. bias + ReLU -> BF16, layer 3 as a dot product, outputs
    float y = 0.f;
    {
      float z[32];
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        tmem_ld32(d2 + lane_row + uint32_t(32 * half), z);
#pragma unroll
        for (int k = 0; k < 32; k += 2) {
          // relu + BF16 rounding of two columns at once, then back to FP32
          const uint32_t hp = relu_pack2(z[k] + s.b2[32 * half + k], z[k + 1] + s.b2[32 * half + k + 1]);
          y = fmaf(__uint_as_float(hp << 16), s.w3[32 * half + k], y);
          y = fmaf(__uint_as_float(hp & 0xffff0000u), s.w3[32 * half + k + 1], y);
        }
      }
    }
    y += s.b3;
    if (live) {
      if (a.p0) {
        const int sc = a.scenes ? find_scene(a.scenes->fluid_off, a.scenes->nscenes, int(row)) : 0;
        const float p = (a.restart && __ldg(a.restart + sc))
                            ? pprev_row
                            : sinhf(fmaxf(u_prev + fminf(y * s.t_scale, kMaxRise), 0.f)) * a.p_unit;
        a.p0[row] = p;
        reinterpret_cast<float*>(a.pos_q + row)[3] = p / (rho_row * rho_row);
      }
      if (a.pred) a.pred[row] = y;
    }
    // the next tile rewrites x / h1 and the accumulators
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

cudaError_t launch_mlp_infer_tc(const MlpInferArgs& a, int sm_count, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const long long tiles = (a.n + kTile - 1) / kTile;
  long long blocks = (long long)kCtasPerSm * sm_count;
  if (blocks > tiles) blocks = tiles;
  k_mlp_infer_tc<<<int(blocks), kTile, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace sph
