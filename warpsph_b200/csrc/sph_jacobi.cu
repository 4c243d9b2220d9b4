// Relaxed-Jacobi pressure solve as one persistent cooperative kernel, with the
// step's kick, drift and CFL update fused behind it.
//
// Reference loop (IISPH.py:1155-1296): compute_term_Ap_1/2 with p_0, then
//   while loop < 2 or avg_err > ETA:  (break once loop > 100)
//       update_p; compute_term_Ap_1; compute_term_Ap_2; update_rho_error; loop += 1
// with the error read on the host twice per iteration (IISPH.py:1489-1494).
//
// Here one iteration k is two grid-wide passes separated by barriers:
//   pass A  s_k  = sum_j d_ij p_j            = -m dt^2 sum_j gradW_ij p_j / rho_j^2
//           A1_k = m sum_j (d_ji p_i - d_jj p_j) . gradW_ij          (compute_term_Ap_1)
//   pass B  Ap_k = A1_k + m sum_j (s_i - s_j) . gradW_ij + s_i . B_i + a_ii p_i
//                                                                     (compute_term_Ap_2)
//           err_k from rho_adv + Ap_k (update_rho_error), reduced in FP64 with a
//           fixed order, and p_{k+1} = update_p(p_k, Ap_k) into the other buffer
// After the second barrier every block reduces the per-block partial sums in the
// same order, so all blocks take the same convergence decision; the loop exits
// with p_k and s_k exactly where the reference's does.  The zero warm start
// begins at k = 1 because p_0 = 0 gives Ap_0 = 0 and the build already wrote p_1.
//
// Epilogue: kick (IISPH.py:674-688), drift (IISPH.py:691-699) written straight
// into the next step's state arrays, max |v| by atomicMax, and the last block to
// finish computes the CFL dt (IISPH.py:1367-1371) on the device.
#include "sph_internal.cuh"

namespace sph {

constexpr int kJacobiThreads = 256;

// Neighbour loops are unrolled by kUnroll with every load of a group issued
// before any use, and the next group's indices are fetched while the current
// group's gathers are in flight, so each thread keeps up to 2*kUnroll
// independent loads outstanding (the passes are bound by gather latency).
// List entries are read once per pass with the streaming hint (ld.global.cs),
// which lets the L2 keep the gathered pos / P4 / s4 arrays resident instead of
// the list stream.  Positions and counts are read-only for the whole kernel and
// use the non-coherent path; P4 and s4 are rewritten between barriers and use
// plain coherent loads.
constexpr int kUnroll = 4;

template <typename Body>
__device__ __forceinline__ void for_neighbours(const int* nb, int cnt, const float4* pos, const float4* other,
                                               Body body) {
  int k = 0;
  int jn[kUnroll];
  if (cnt >= kUnroll) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) jn[u] = __ldcs(nb + u * kWarp);
  }
  for (; k + kUnroll <= cnt; k += kUnroll) {
    int j[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) j[u] = jn[u];
    if (k + 2 * kUnroll <= cnt) {
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) jn[u] = __ldcs(nb + (k + kUnroll + u) * kWarp);
    }
    float4 xj[kUnroll], oj[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      xj[u] = __ldg(pos + j[u]);
      oj[u] = other[j[u]];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) body(xj[u], oj[u]);
  }
  for (; k < cnt; ++k) {
    const int j = __ldcs(nb + k * kWarp);
    body(__ldg(pos + j), other[j]);
  }
}

template <class Tab>
__device__ inline void pass_a(int i, const JacobiArgs& a, const Tab& G, float t3) {
  const Consts& c = a.c;
  const float4 xi = __ldg(a.pos + i);
  const float4 qi = a.P4[i];
  const float ci = t3 * qi.w;  // d_ji p_i = gradW_ij * (m dt^2 p_i / rho_i^2)
  const int cnt = min(__ldg(a.cnt_ff + i), c.max_ff);
  const int* nb = a.nbr_ff + ell_index(i, 0, c.max_ff);
  float sx = 0.f, sy = 0.f, sz = 0.f, a1 = 0.f;
  for_neighbours(nb, cnt, a.pos, a.P4, [&](const float4 xj, const float4 qj) {
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    const float gs = grad_scalar(G, r, c);
    const float gx = gs * dx, gy = gs * dy, gz = gs * dz;
    sx += gx * qj.w;
    sy += gy * qj.w;
    sz += gz * qj.w;
    a1 += (ci * gx - qj.x) * gx + (ci * gy - qj.y) * gy + (ci * gz - qj.z) * gz;
  });
  a.s4[i] = make_float4(-t3 * sx, -t3 * sy, -t3 * sz, a1 * c.m);
}

template <class Tab>
__device__ inline void pass_b(int i, const JacobiArgs& a, const Tab& G, const float* pc, float* pn,
                              double& es, long long& ec) {
  const Consts& c = a.c;
  const float4 xi = __ldg(a.pos + i);
  const float4 si = a.s4[i];
  const int cnt = min(__ldg(a.cnt_ff + i), c.max_ff);
  const int* nb = a.nbr_ff + ell_index(i, 0, c.max_ff);
  float acc = 0.f;
  for_neighbours(nb, cnt, a.pos, a.s4, [&](const float4 xj, const float4 sj) {
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    const float gs = grad_scalar(G, r, c);
    acc += (si.x - sj.x) * (gs * dx) + (si.y - sj.y) * (gs * dy) + (si.z - sj.z) * (gs * dz);
  });
  const float4 bv = __ldg(a.bvec + i);
  const float4 da = __ldg(a.dii_aii + i);
  const float p = pc[i];
  const float Ap = si.w + ((acc * c.m + (si.x * bv.x + si.y * bv.y + si.z * bv.z)) + da.w * p);
  // update_p (IISPH.py:534-539)
  float aa = da.w;
  if (aa > -c.inv_small && aa < c.inv_small) aa = (aa < 0.f ? -1.f : 1.f) * c.inv_small;
  const float pnew = fmaxf(p + (c.rho0 - bv.w - Ap) * c.omega / aa, 0.f);
  // update_rho_error (IISPH.py:565-568)
  const float rp = bv.w + Ap;
  if (rp > c.rho0) {
    es += double(fabsf(rp / c.rho0 - 1.0f));
    ec += 1;
  }
  const float rho = __ldg(a.rho + i);
  pn[i] = pnew;
  a.P4[i] = make_float4(da.x * pnew, da.y * pnew, da.z * pnew, pnew / (rho * rho));
  a.Ap[i] = Ap;
}

template <class Tab>
__device__ __forceinline__ void jacobi_body(const JacobiArgs& a, const Tab& G);

template <bool SMEM>
__global__ void __launch_bounds__(kJacobiThreads) k_jacobi(JacobiArgs a) {
  extern __shared__ float2 s_pairs[];
  if (SMEM) {
    stage_pairs(s_pairs, a.g_table, a.c.sg);
    jacobi_body(a, PairTable{s_pairs});
  } else {
    jacobi_body(a, FlatTable{a.g_table});
  }
}

template <class Tab>
__device__ __forceinline__ void jacobi_body(const JacobiArgs& a, const Tab& G) {
  __shared__ double s_sum[kJacobiThreads / 32];
  __shared__ long long s_cnt[kJacobiThreads / 32];
  __shared__ double s_avg;
  __shared__ int s_stop, s_iters;
  __shared__ unsigned int s_vmax;

  // A capacity overflow in the build truncated some neighbour lists: leave the
  // state untouched so the host can grow the lists and redo the step.
  if (*(volatile const int*)&a.acc->flags & (SPH_F_FF_OVERFLOW | SPH_F_FB_OVERFLOW)) return;

  if (threadIdx.x == 0) s_vmax = 0u;
  __syncthreads();

  const Consts& c = a.c;
  const float dt = a.st->dt;
  const float inv_dt = a.st->inv_dt;
  const float t3 = c.m * (dt * dt);
  const int n = a.n;
  const int stride = gridDim.x * blockDim.x;
  const int tid0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  float* pc = a.p_a;
  float* pn = a.p_b;
  int k = a.start_iter;
  int iters = 0;
  double avg = 0.0;
  bool ok = true;
  bool converged = false;

  for (;;) {
    for (int i = tid0; i < n; i += stride) pass_a(i, a, G, t3);
    if (!grid_barrier(a.acc, gridDim.x, a.budget)) { ok = false; break; }

    double es = 0.0;
    long long ec = 0;
    for (int i = tid0; i < n; i += stride) pass_b(i, a, G, pc, pn, es, ec);
    es = warp_sum(es);
    ec = warp_sum(ec);
    if (lane == 0) {
      s_sum[warp] = es;
      s_cnt[warp] = ec;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double bs = 0.0;
      long long bc = 0;
      for (int w = 0; w < kJacobiThreads / 32; ++w) {
        bs += s_sum[w];
        bc += s_cnt[w];
      }
      a.partials[blockIdx.x].sum = bs;
      a.partials[blockIdx.x].cnt = bc;
    }
    if (!grid_barrier(a.acc, gridDim.x, a.budget)) { ok = false; break; }

    if (k >= 1) {
      // identical fixed-order reduction in every block -> identical decision
      if (warp == 0) {
        double ts = 0.0;
        long long tc = 0;
        for (int b = lane; b < (int)gridDim.x; b += 32) {
          ts += a.partials[b].sum;
          tc += a.partials[b].cnt;
        }
        ts = warp_sum(ts);
        tc = warp_sum(tc);
        if (lane == 0) {
          const double av = tc ? ts / double(tc) : 0.0;
          const bool conv = (k >= c.min_iter) && !(av > a.eta_d);
          const bool stop = (c.fixed_iters > 0) ? (k >= c.fixed_iters) : (conv || k > c.max_loop);
          s_avg = av;
          s_stop = stop ? (conv || c.fixed_iters > 0 ? 1 : 2) : 0;
          s_iters = k;
        }
      }
      __syncthreads();
      iters = s_iters;
      avg = s_avg;
      const int st = s_stop;
      __syncthreads();
      if (st) {
        converged = (st == 1);
        break;
      }
    }
    float* t = pc;
    pc = pn;
    pn = t;
    ++k;
  }

  // kick + drift -> next step's state (pc holds p_k, s4 holds s_k)
  float vmax = 0.f;
  bool finite = true;
  if (ok) {
    for (int i = tid0; i < n; i += stride) {
      const float4 va = a.vadv[i];
      const float4 da = a.dii_aii[i];
      const float4 s = a.s4[i];
      const float p = pc[i];
      const float vx = va.x + inv_dt * (da.x * p + s.x);
      const float vy = va.y + inv_dt * (da.y * p + s.y);
      const float vz = va.z + inv_dt * (da.z * p + s.z);
      const float4 x = a.pos[i];
      a.vel_out[i] = make_float4(vx, vy, vz, 0.f);
      a.pos_out[i] = make_float4(x.x + vx * dt, x.y + vy * dt, x.z + vz * dt, 0.f);
      a.orig_out[i] = a.orig_w[i];
      a.p_out[i] = p;
      const float vl = sqrtf(vx * vx + vy * vy + vz * vz);
      vmax = fmaxf(vmax, vl);
      finite = finite && isfinite(vl) && isfinite(p);
    }
  }
  // max over the block, then over the grid (non-negative floats order as uints)
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  const int nonfinite = __syncthreads_or(!finite);
  if (lane == 0) atomicMax(&s_vmax, __float_as_uint(vmax));
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&a.acc->vmax_bits, s_vmax);
    if (nonfinite) atomicOr(&a.acc->flags, SPH_F_NONFINITE);
    __threadfence();
    const unsigned int done = atomicAdd(&a.acc->done_blocks, 1u);
    if (done == gridDim.x - 1) {
      // last block: CFL (IISPH.py:1367-1371) and the step's statistics
      __threadfence();
      StepAcc* acc = a.acc;
      DevState* st = a.st;
      const float vm = __uint_as_float(*(volatile unsigned int*)&acc->vmax_bits);
      int flags = *(volatile int*)&acc->flags;
      if (!isfinite(vm)) flags |= SPH_F_NONFINITE;
      if (ok && !converged && c.fixed_iters <= 0) flags |= SPH_F_NOT_CONVERGED;
      double dt_next, inv_next;
      if (double(vm) >= double(float(a.inv_small_d))) {
        // numpy-2 float32 semantics of 0.4*DIAMETER / v_max (IISPH.py:1369)
        const float q = float(a.cfl_len) / vm;
        if (q < float(a.dt_max)) {
          dt_next = double(q);
          inv_next = double(1.0f / q);
        } else {
          dt_next = a.dt_max;
          inv_next = 1.0 / a.dt_max;
        }
      } else {
        dt_next = fmin(a.cfl_len / a.inv_small_d, a.dt_max);
        inv_next = 1.0 / dt_next;
      }
      const double dt_used = st->dt64;
      st->sim_time += dt_used;
      st->step_index += 1;
      acc->iterations = iters;
      acc->avg_err = avg;
      acc->flags = flags;
      SphStepStats r;
      r.iterations = iters;
      r.flags = flags;
      r.avg_err = avg;
      r.v_max = double(vm);
      r.dt = dt_used;
      r.dt_next = dt_next;
      r.sim_time = st->sim_time;
      r.n_ff_pairs = (long long)acc->pairs_ff;
      r.n_fb_pairs = (long long)acc->pairs_fb;
      r.max_ff_count = acc->max_ff;
      r.max_fb_count = acc->max_fb;
      r.step_index = st->step_index;
      a.ring[(st->step_index - 1) % kStatsRing] = r;
      *a.last = r;
      st->dt64 = dt_next;
      st->inv_dt64 = inv_next;
      st->dt = float(dt_next);
      st->inv_dt = float(inv_next);
    }
  }
}

static size_t jacobi_smem(int sg) { return (sg <= 8192) ? sizeof(float2) * size_t(sg) : 0; }

cudaError_t jacobi_config(int block, int sg, int* blocks_per_sm, size_t* smem_out) {
  const size_t smem = jacobi_smem(sg);
  int b = 0;
  cudaError_t e;
  if (smem > 0) {
    e = cudaFuncSetAttribute(k_jacobi<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_jacobi<true>, block, smem);
  } else {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_jacobi<false>, block, 0);
  }
  if (e != cudaSuccess) return e;
  *blocks_per_sm = b;
  if (smem_out) *smem_out = smem;
  return cudaSuccess;
}

cudaError_t launch_jacobi(const JacobiArgs& a, int grid, int block, size_t smem, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (smem > 0) return cudaLaunchKernelEx(&cfg, k_jacobi<true>, a);
  return cudaLaunchKernelEx(&cfg, k_jacobi<false>, a);
}

}  // namespace sph
