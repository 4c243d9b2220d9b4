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

// Neighbour loops are unrolled by U with every load of a group issued before
// any use, and the next group's indices are fetched while the current group's
// gathers are in flight, so each thread keeps up to 2U independent loads
// outstanding (the passes are bound by gather latency).
// List entries are read once per pass with the streaming hint (ld.global.cs),
// which lets the L2 keep the gathered pos / P4 / s4 arrays resident instead of
// the list stream.  Positions and counts are read-only for the whole kernel and
// use the non-coherent path; P4 and s4 are rewritten between barriers and use
// plain coherent loads.
template <int kUnroll, typename Body>
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

template <int U, class Tab>
__device__ inline void pass_a(int i, const JacobiArgs& a, const Tab& G, float t3) {
  const Consts& c = a.c;
  const float4 xi = __ldg(a.pos + i);
  const float4 qi = a.P4[i];
  const float ci = t3 * qi.w;  // d_ji p_i = gradW_ij * (m dt^2 p_i / rho_i^2)
  const int cnt = min(__ldg(a.cnt_ff + i), c.max_ff);
  const int* nb = a.nbr_ff + ell_index(i, 0, c.max_ff);
  float sx = 0.f, sy = 0.f, sz = 0.f, a1 = 0.f;
  for_neighbours<U>(nb, cnt, a.pos, a.P4, [&](const float4 xj, const float4 qj) {
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

template <int U, class Tab>
__device__ inline void pass_b(int i, const JacobiArgs& a, const Tab& G, const float* pc, float* pn,
                              double& es, long long& ec) {
  const Consts& c = a.c;
  const float4 xi = __ldg(a.pos + i);
  const float4 si = a.s4[i];
  const int cnt = min(__ldg(a.cnt_ff + i), c.max_ff);
  const int* nb = a.nbr_ff + ell_index(i, 0, c.max_ff);
  float acc = 0.f;
  for_neighbours<U>(nb, cnt, a.pos, a.s4, [&](const float4 xj, const float4 sj) {
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

template <int T, int PPT, int U, class Tab>
__device__ __forceinline__ void jacobi_body(const JacobiArgs& a, const Tab& G);

// T threads per block, PPT particles per thread (chunks of T * PPT particles),
// neighbour-loop unroll U: the knobs the autotuner chooses among.
template <bool SMEM, int T, int PPT, int U>
__global__ void __launch_bounds__(T) k_jacobi(JacobiArgs a) {
  extern __shared__ float2 s_pairs[];
  if (SMEM) {
    stage_pairs(s_pairs, a.g_table, a.c.sg);
    jacobi_body<T, PPT, U>(a, PairTable{s_pairs});
  } else {
    jacobi_body<T, PPT, U>(a, FlatTable{a.g_table});
  }
}

// Block-wide sum of (double, long long) in a fixed order; result valid in thread 0.
template <int T>
__device__ __forceinline__ void block_sum2(double& v, long long& c, double* sv, long long* sc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  c = warp_sum(c);
  if (lane == 0) {
    sv[warp] = v;
    sc[warp] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = 0.0;
    long long bc = 0;
    for (int w = 0; w < T / 32; ++w) {
      bv += sv[w];
      bc += sc[w];
    }
    v = bv;
    c = bc;
  }
  __syncthreads();
}

template <int T, int PPT, int U, class Tab>
__device__ __forceinline__ void jacobi_body(const JacobiArgs& a, const Tab& G) {
  __shared__ double s_sum[T / 32];
  __shared__ long long s_cnt[T / 32];
  __shared__ int s_stop;

  // A capacity overflow in the build truncated some neighbour lists: leave the
  // state untouched so the host can grow the lists and redo the step.
  if (*(volatile const int*)&a.acc->flags & (SPH_F_FF_OVERFLOW | SPH_F_FB_OVERFLOW)) return;
  if (threadIdx.x == 0) s_stop = 0;
  __syncthreads();

  const Consts& c = a.c;
  StepAcc* acc = a.acc;
  float* pc = a.p_a;
  float* pn = a.p_b;
  int k = a.start_iter;
  bool ok = true;
  int stop_code = 0;  // single scene: how the solve stopped (1 converged, 2 capped)

  for (;;) {
    // pass A over the chunks of unconverged scenes
    for (int ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
      const int s = __ldg(a.chunk_scene + ch);
      if (ld_volatile_int(&acc->done[s])) continue;
      const int2 r = __ldg(a.chunks + ch);
      const float dt = a.st->dt[s];
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        const int i = r.x + q * T + threadIdx.x;
        if (i < r.y) pass_a<U>(i, a, G, c.m * (dt * dt));
      }
    }
    if (!grid_barrier(acc, gridDim.x, a.budget)) { ok = false; break; }

    // pass B: Ap, p_{k+1} and the density error.  A block's chunks visit the
    // scenes in non-decreasing order, so each scene is one contiguous run of
    // them; the run's error sum goes to partials[block][scene] (fixed order).
    for (int q = threadIdx.x; q < a.nscenes; q += blockDim.x) {
      a.partials[blockIdx.x * a.nscenes + q].sum = 0.0;
      a.partials[blockIdx.x * a.nscenes + q].cnt = 0;
    }
    __syncthreads();
    {
      int run = -1;
      double es = 0.0;
      long long ec = 0;
      auto flush = [&]() {
        block_sum2<T>(es, ec, s_sum, s_cnt);
        if (threadIdx.x == 0) {
          a.partials[blockIdx.x * a.nscenes + run].sum = es;
          a.partials[blockIdx.x * a.nscenes + run].cnt = ec;
        }
        es = 0.0;
        ec = 0;
      };
      for (int ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
        const int s = __ldg(a.chunk_scene + ch);
        if (s != run) {
          if (run >= 0) flush();
          run = s;
        }
        if (ld_volatile_int(&acc->done[s])) continue;
        const int2 r = __ldg(a.chunks + ch);
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          const int i = r.x + q * T + threadIdx.x;
          if (i < r.y) pass_b<U>(i, a, G, pc, pn, es, ec);
        }
      }
      if (run >= 0) flush();
    }
    if (!grid_barrier(acc, gridDim.x, a.budget)) { ok = false; break; }

    if (k >= 1) {
      // Scene s's error is the block partials summed in block order.
      if (a.nscenes == 1) {
        // one scene: every block does this sum itself and takes the same
        // decision from shared memory; no flag is written inside the loop,
        // so no thread ever reads a value another block is changing
        double ts = 0.0;
        long long tc = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
          ts += a.partials[b].sum;
          tc += a.partials[b].cnt;
        }
        block_sum2<T>(ts, tc, s_sum, s_cnt);
        if (threadIdx.x == 0) {
          const double av = tc ? ts / double(tc) : 0.0;
          const bool conv = (k >= c.min_iter) && !(av > a.eta_d);
          const bool stop = (c.fixed_iters > 0) ? (k >= c.fixed_iters) : (conv || k > c.max_loop);
          s_stop = stop ? ((conv || c.fixed_iters > 0) ? 1 : 2) : 0;
          if (blockIdx.x == 0) {
            acc->iterations[0] = k;
            acc->avg_err[0] = av;
          }
        }
        __syncthreads();
        const int st = s_stop;
        __syncthreads();
        if (st) {
          stop_code = st;
          break;
        }
      } else {
        // several scenes: scene s is decided by block s mod G alone (the only
        // reader and writer of its flag here); a third barrier publishes it
        for (int s = blockIdx.x; s < a.nscenes; s += gridDim.x) {
          if (ld_volatile_int(&acc->done[s])) continue;
          double ts = 0.0;
          long long tc = 0;
          for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
            ts += a.partials[b * a.nscenes + s].sum;
            tc += a.partials[b * a.nscenes + s].cnt;
          }
          block_sum2<T>(ts, tc, s_sum, s_cnt);
          if (threadIdx.x == 0) {
            const double av = tc ? ts / double(tc) : 0.0;
            const bool conv = (k >= c.min_iter) && !(av > a.eta_d);
            const bool stop = (c.fixed_iters > 0) ? (k >= c.fixed_iters) : (conv || k > c.max_loop);
            acc->iterations[s] = k;
            acc->avg_err[s] = av;
            if (stop) {
              acc->final_buf[s] = (pc == a.p_a) ? 0 : 1;
              acc->done[s] = (conv || c.fixed_iters > 0) ? 1 : 2;
            }
          }
          __syncthreads();
        }
        if (!grid_barrier(acc, gridDim.x, a.budget)) { ok = false; break; }
        bool mine = false;  // scenes may outnumber the block's threads
        for (int s = threadIdx.x; s < a.nscenes; s += blockDim.x) mine = mine || !ld_volatile_int(&acc->done[s]);
        if (!__syncthreads_or(mine)) break;
      }
    }
    float* t = pc;
    pc = pn;
    pn = t;
    ++k;
  }

  if (a.nscenes == 1 && blockIdx.x == 0 && threadIdx.x == 0) {
    acc->done[0] = stop_code;  // read only by the last block, after every block finished
    acc->final_buf[0] = (pc == a.p_a) ? 0 : 1;
  }

  // kick + drift -> next step's state, with each scene's final p and s.  With
  // one scene every block knows the final buffer (pc); with several it is in
  // acc->final_buf, published by the last barrier.
  bool finite = true;
  if (ok) {
    int run = -1;
    float vrun = 0.f;
    auto flush = [&]() {
      float v = vrun;
      for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
      if ((threadIdx.x & 31) == 0) atomicMax(&acc->vmax_bits[run], __float_as_uint(v));
      vrun = 0.f;
    };
    for (int ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
      const int s = __ldg(a.chunk_scene + ch);
      if (s != run) {
        if (run >= 0) flush();
        run = s;
      }
      const int2 r = __ldg(a.chunks + ch);
      const float* pf = (a.nscenes == 1) ? pc : (ld_volatile_int(&acc->final_buf[s]) ? a.p_b : a.p_a);
      const float dt = a.st->dt[s], inv_dt = a.st->inv_dt[s];
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        const int i = r.x + q * T + threadIdx.x;
        if (i >= r.y) continue;
        const float4 va = a.vadv[i];
        const float4 da = a.dii_aii[i];
        const float4 sv = a.s4[i];
        const float p = pf[i];
        const float vx = va.x + inv_dt * (da.x * p + sv.x);
        const float vy = va.y + inv_dt * (da.y * p + sv.y);
        const float vz = va.z + inv_dt * (da.z * p + sv.z);
        const float4 x = a.pos[i];
        a.vel_out[i] = make_float4(vx, vy, vz, 0.f);
        a.pos_out[i] = make_float4(x.x + vx * dt, x.y + vy * dt, x.z + vz * dt, 0.f);
        a.orig_out[i] = a.orig_w[i];
        a.p_out[i] = p;
        const float vl = sqrtf(vx * vx + vy * vy + vz * vz);
        vrun = fmaxf(vrun, vl);  // non-negative floats order as uints; NaN sorts high
        finite = finite && isfinite(vl) && isfinite(p);
      }
    }
    if (run >= 0) flush();
    if (a.move_boundary) {
      // update_rigid_x (IISPH.py:651-671): x_b += v_b dt with the step's dt
      // (the last block replaces dt only after every block has finished here)
      for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < a.nb; b += gridDim.x * blockDim.x) {
        const int s = (a.nscenes == 1) ? 0 : find_scene(a.scenes->bound_off, a.nscenes, b);
        const float dt = a.st->dt[s];
        float4 xb = a.bpos[b];
        const float4 vb = __ldg(a.bvel + b);
        xb.x = __fadd_rn(xb.x, __fmul_rn(vb.x, dt));
        xb.y = __fadd_rn(xb.y, __fmul_rn(vb.y, dt));
        xb.z = __fadd_rn(xb.z, __fmul_rn(vb.z, dt));
        a.bpos[b] = xb;
      }
    }
  }
  const int nonfinite = __syncthreads_or(!finite);
  if (threadIdx.x == 0) {
    if (nonfinite) atomicOr(&acc->flags, SPH_F_NONFINITE);
    __threadfence();
    const unsigned int done = atomicAdd(&acc->done_blocks, 1u);
    if (done == gridDim.x - 1) {
      // last block: per-scene CFL (IISPH.py:1367-1371) and the step's statistics
      __threadfence();
      DevState* st = a.st;
      int flags = *(volatile int*)&acc->flags;
      int iters = 0;
      double avg = 0.0, vmax_all = 0.0;
      const double dt_used0 = st->dt64[0];
      for (int s = 0; s < a.nscenes; ++s) {
        const float vm = __uint_as_float(*(volatile unsigned int*)&acc->vmax_bits[s]);
        if (!isfinite(vm)) flags |= SPH_F_NONFINITE;
        if (ok && acc->done[s] == 2 && c.fixed_iters <= 0) flags |= SPH_F_NOT_CONVERGED;
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
        st->sim_time[s] += st->dt64[s];
        st->dt64[s] = dt_next;
        st->inv_dt64[s] = inv_next;
        st->dt[s] = float(dt_next);
        st->inv_dt[s] = float(inv_next);
        iters = max(iters, acc->iterations[s]);
        avg = fmax(avg, acc->avg_err[s]);
        vmax_all = fmax(vmax_all, double(vm));
      }
      st->step_index += 1;
      acc->flags = flags;
      SphStepStats r;
      r.iterations = iters;
      r.flags = flags;
      r.avg_err = avg;
      r.v_max = vmax_all;
      r.dt = dt_used0;
      r.dt_next = st->dt64[0];
      r.sim_time = st->sim_time[0];
      r.n_ff_pairs = (long long)acc->pairs_ff;
      r.n_fb_pairs = (long long)acc->pairs_fb;
      r.max_ff_count = acc->max_ff;
      r.max_fb_count = acc->max_fb;
      r.step_index = st->step_index;
      a.ring[(st->step_index - 1) % kStatsRing] = r;
      *a.last = r;
    }
  }
}

static size_t jacobi_smem(int sg) { return (sg <= 8192) ? sizeof(float2) * size_t(sg) : 0; }

using JacobiKernel = void (*)(JacobiArgs);

template <bool SMEM>
static JacobiKernel pick_jacobi(int T, int ppt, int unroll) {
#define SPH_JACOBI_CASE(T_, P_, U_) \
  if (T == T_ && ppt == P_ && unroll == U_) return k_jacobi<SMEM, T_, P_, U_>;
  SPH_JACOBI_CASE(128, 1, 2)
  SPH_JACOBI_CASE(128, 1, 4)
  SPH_JACOBI_CASE(128, 1, 8)
  SPH_JACOBI_CASE(128, 2, 2)
  SPH_JACOBI_CASE(128, 2, 4)
  SPH_JACOBI_CASE(128, 2, 8)
  SPH_JACOBI_CASE(256, 1, 2)
  SPH_JACOBI_CASE(256, 1, 4)
  SPH_JACOBI_CASE(256, 1, 8)
  SPH_JACOBI_CASE(256, 2, 2)
  SPH_JACOBI_CASE(256, 2, 4)
  SPH_JACOBI_CASE(256, 2, 8)
#undef SPH_JACOBI_CASE
  return nullptr;
}

static JacobiKernel jacobi_kernel(int sg, int T, int ppt, int unroll) {
  return jacobi_smem(sg) > 0 ? pick_jacobi<true>(T, ppt, unroll) : pick_jacobi<false>(T, ppt, unroll);
}

bool jacobi_variant_ok(int block, int ppt, int unroll) { return pick_jacobi<true>(block, ppt, unroll) != nullptr; }

cudaError_t jacobi_config(int block, int ppt, int unroll, int sg, int* blocks_per_sm, size_t* smem_out) {
  JacobiKernel k = jacobi_kernel(sg, block, ppt, unroll);
  if (!k) return cudaErrorInvalidValue;
  const size_t smem = jacobi_smem(sg);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
  }
  int b = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, block, smem);
  if (e != cudaSuccess) return e;
  *blocks_per_sm = b;
  if (smem_out) *smem_out = smem;
  return cudaSuccess;
}

cudaError_t launch_jacobi(const JacobiArgs& a, int grid, int block, int ppt, int unroll, size_t smem,
                          cudaStream_t s) {
  JacobiKernel k = jacobi_kernel(a.c.sg, block, ppt, unroll);
  if (!k) return cudaErrorInvalidValue;
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
  return cudaLaunchKernelEx(&cfg, k, a);
}

}  // namespace sph
