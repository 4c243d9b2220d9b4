// Relaxed-Jacobi pressure solve as one persistent cooperative kernel, with the
// step's kick, drift and CFL update fused behind it.
//
// Reference loop (IISPH.py:1155-1296): compute_term_Ap_1/2 with p_0, then
//   while loop < 2 or avg_err > ETA:  (break once loop > 100)
//       update_p; compute_term_Ap_1; compute_term_Ap_2; update_rho_error; loop += 1
// with the error read on the host twice per iteration (IISPH.py:1489-1494).
//
// The reference evaluates, with d_ij = -m dt^2 gradW_ij / rho_j^2 and
// d_ji = m dt^2 gradW_ij / rho_i^2 (compute_term_d, IISPH.py:332-382),
//   s_i  = sum_j d_ij p_j                                   (compute_term_Ap_1)
//   Ap_i = m sum_j (d_ji p_i - d_jj p_j) . gradW_ij
//        + m sum_j (s_i - s_j) . gradW_ij + s_i . B_i + a_ii p_i   (compute_term_Ap_2)
// with B_i = sum_b psi_b gradW_ib.  Substituting a_ii (IISPH.py:385-428) and
// d_ii (IISPH.py:382) and collecting terms gives the same value as
//   a_i  = d_ii p_i + s_i
//   Ap_i = m sum_j (a_i - a_j) . gradW_ij + a_i . B_i
// (a_i is dt^2 times the pressure acceleration, the quantity the kick adds,
// IISPH.py:684).  The pairwise differences a_i - a_j cancel the common part of
// the field exactly, as s_i - s_j does in the reference.  Pass A needs only the
// neighbours' positions and q_j = p_j / rho_j^2, which sit together in one
// 16-byte record (pos.w); pass B needs their positions and a_j.  That is three
// 16-byte gathers per neighbour per iteration instead of the four a direct
// transcription needs (x and (d_jj p_j, q_j) in the first pass, x and s_j in
// the second), and the gathers bound the passes.
//
// One iteration k is two grid-wide passes separated by barriers:
//   pass A  s_k = -m dt^2 sum_j q_j gradW_ij,  a_k = d_ii p_k + s_k
//   pass B  Ap_k, err_k from rho_adv + Ap_k (update_rho_error), reduced in FP64
//           with a fixed order, and p_{k+1} = update_p(p_k, Ap_k) into the other
//           buffer (and q_{k+1} into pos.w)
// After the second barrier every block reduces the per-block partial sums in the
// same order, so all blocks take the same convergence decision; the loop exits
// with p_k and a_k exactly where the reference's does.  The zero warm start
// begins at k = 1 because p_0 = 0 gives Ap_0 = 0 and the build already wrote p_1.
//
// Epilogue: kick (IISPH.py:674-688), drift (IISPH.py:691-699) written straight
// into the next step's state arrays, max |v| by atomicMax, and the last block to
// finish computes the CFL dt (IISPH.py:1367-1371) on the device.
#include "sph_internal.cuh"

namespace sph {

// Neighbour loops run the same trip count on every lane of a warp (the
// warp's largest neighbour count, rounded up to the unroll U) with no
// divergent tail: a lane past its own count takes its own index, whose
// gradient term is exactly zero (x_j = x_i).  Every load of a group is issued
// before any use, and the next group's indices are fetched while the current
// group's gathers are in flight, so each thread keeps up to 2U independent
// loads outstanding.  List entries are read once per pass with the streaming
// hint (ld.global.cs), which lets the L2 keep the gathered pos / a4 arrays
// resident instead of the list stream.  pos (its .w) and a4 are rewritten
// between barriers, so they are read with plain coherent loads.  NG = 1
// gathers pos only, NG = 2 also the second array.
// NG = 3 is pass B's compact form: the second array is a4, whose .w holds the
// neighbour's x (pass A stores it there), and (y_j, z_j) come as an 8-byte
// record through the texture path from a texture object over a (y, z) copy of
// the positions, written by the cell sort's gather before the solve (the solve
// never changes positions, so the texture path sees no stale data).  Pass B
// then moves 24 bytes per neighbour instead of 32, and the 8-byte records put
// a warp's gathers on fewer lines.
template <int kUnroll, int NG, typename Body>
__device__ __forceinline__ void for_neighbours(const int* __restrict__ nb, int cnt, int self,
                                               const float4* pos, const float4* other, Body body,
                                               unsigned long long yztex = 0) {
  const int wmax = __reduce_max_sync(0xffffffffu, cnt);
  int jn[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; ++u) jn[u] = (u < cnt) ? __ldcs(nb + u * kWarp) : self;
  for (int k = 0; k < wmax; k += kUnroll) {
    int j[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      j[u] = jn[u];
      const int kn = k + kUnroll + u;
      jn[u] = (kn < cnt) ? __ldcs(nb + kn * kWarp) : self;
    }
    float4 xj[kUnroll], oj[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (NG == 3) {
        oj[u] = other[j[u]];
        const float2 yz = tex1Dfetch<float2>(cudaTextureObject_t(yztex), j[u]);
        xj[u].y = yz.x;
        xj[u].z = yz.y;
      } else {
        xj[u] = pos[j[u]];
        if (NG == 2) oj[u] = other[j[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (NG == 3) xj[u].x = oj[u].w;
      body(xj[u], oj[u]);
    }
  }
}

// pass A for particle i: s = sum_j d_ij p_j (IISPH.py:458-464) and a = d_ii p + s.
// Every lane of the warp calls it (live = false past the chunk's end, with i
// a valid slot of the chunk), because the neighbour loop is warp-synchronous.
template <int U, class Tab>
__device__ inline void pass_a(int i, bool live, const JacobiArgs& a, const Tab& G, float t3, const float* pc) {
  const Consts& c = a.c;
  const float4 xi = a.pos[i];
  const int cnt = live ? min(__ldg(a.cnt_ff + i), c.max_ff) : 0;
  const int* nb = a.nbr_ff + ell_index(i, 0, c.max_ff);
  float sx = 0.f, sy = 0.f, sz = 0.f;
  // one gather per neighbour here against two in pass B: unroll twice as deep
  // so both passes keep the same number of loads in flight
  for_neighbours<(2 * U > 8 ? 8 : 2 * U), 1>(nb, cnt, i, a.pos, nullptr, [&](const float4 xj, const float4) {
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float gq = G(c, dx * dx + dy * dy + dz * dz) * xj.w;
    sx = fmaf(gq, dx, sx);
    sy = fmaf(gq, dy, sy);
    sz = fmaf(gq, dz, sz);
  });
  if (!live) return;
  const float4 da = __ldg(a.dii_aii + i);
  const float p = pc[i];
  a.a4[i] = make_float4(da.x * p + (-t3 * sx), da.y * p + (-t3 * sy), da.z * p + (-t3 * sz), xi.x);
}

// pass B for particle i: Ap (compute_term_Ap_2, IISPH.py:469-518), the density
// error (update_rho_error, IISPH.py:542-567) and p_{k+1} (update_p, IISPH.py:521-539)
template <int U, bool XT, class Tab>
__device__ inline void pass_b(int i, bool live, const JacobiArgs& a, const Tab& G, const float* pc, float* pn,
                              double& es, long long& ec) {
  const Consts& c = a.c;
  const float4 xi = a.pos[i];
  const float4 ai = a.a4[i];
  const int cnt = live ? min(__ldg(a.cnt_ff + i), c.max_ff) : 0;
  const int* nb = a.nbr_ff + ell_index(i, 0, c.max_ff);
  float acc = 0.f;
  for_neighbours<U, XT ? 3 : 2>(nb, cnt, i, a.pos, a.a4, [&](const float4 xj, const float4 aj) {
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float gs = G(c, dx * dx + dy * dy + dz * dz);
    acc = fmaf(gs, (ai.x - aj.x) * dx + (ai.y - aj.y) * dy + (ai.z - aj.z) * dz, acc);
  }, a.yztex);
  if (!live) return;
  const float4 bv = __ldg(a.bvec + i);
  const float4 da = __ldg(a.dii_aii + i);
  const float p = pc[i];
  const float Ap = acc * c.m + (ai.x * bv.x + ai.y * bv.y + ai.z * bv.z);
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
  reinterpret_cast<float*>(a.pos + i)[3] = pnew / (rho * rho);
  a.Ap[i] = Ap;
}

template <int T, int PPT, int U, bool XT, class Tab>
__device__ __forceinline__ void jacobi_body(const JacobiArgs& a, const Tab& G);

// How the passes get the kernel gradient: the table staged in shared memory,
// the table in global memory (too large to stage), or the closed form; the
// last also with pass B's position gathers through the texture path.
constexpr int kGradSmem = 0, kGradFlat = 1, kGradSpline = 2, kGradSplineTex = 3;

// GM gradient mode, T threads per block, PPT particles per thread (chunks of
// T * PPT particles), neighbour-loop unroll U: the knobs the autotuner chooses among.
template <int GM, int T, int PPT, int U>
__global__ void __launch_bounds__(T) k_jacobi(JacobiArgs a) {
  extern __shared__ float2 s_pairs[];
  if (GM == kGradSmem) {
    stage_slopes(s_pairs, a.g_table, a.c.sg);
    jacobi_body<T, PPT, U, false>(a, TableGrad<SlopeTable>{SlopeTable{s_pairs}});
  } else if (GM == kGradFlat) {
    jacobi_body<T, PPT, U, false>(a, TableGrad<FlatSlopeTable>{FlatSlopeTable{a.g_table}});
  } else {
    jacobi_body<T, PPT, U, GM == kGradSplineTex>(a, SplineGrad{});
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

template <int T, int PPT, int U, bool XT, class Tab>
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
  // One scene: each block walks one contiguous run of chunks (run lengths
  // differ by at most one), so consecutive chunks of a block are neighbours
  // in the sorted order and the next chunk's neighbour rows are partly in the
  // SM's L1 (133.6 against 139.1 us per iteration at 1M with chunks dealt
  // round-robin).  Several scenes: round-robin, so that the chunks of the
  // scenes still iterating stay spread over all blocks when others converge.
  const bool runs = (a.nscenes == 1);
  const int c_lo = runs ? int((long long)blockIdx.x * a.nchunks / gridDim.x) : int(blockIdx.x);
  const int c_hi = runs ? int((long long)(blockIdx.x + 1) * a.nchunks / gridDim.x) : a.nchunks;
  const int c_step = runs ? 1 : int(gridDim.x);
  float* pc = a.p_a;
  float* pn = a.p_b;
  int k = a.start_iter;
  bool ok = true;
  int stop_code = 0;  // single scene: how the solve stopped (1 converged, 2 capped)

  for (;;) {
    // pass A over the chunks of unconverged scenes
    for (int ch = c_lo; ch < c_hi; ch += c_step) {
      const int s = __ldg(a.chunk_scene + ch);
      if (ld_volatile_int(&acc->done[s])) continue;
      const int2 r = __ldg(a.chunks + ch);
      const float dt = a.st->dt[s];
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        const int i = r.x + q * T + threadIdx.x;
        pass_a<U>(i < r.y ? i : r.x, i < r.y, a, G, c.m * (dt * dt), pc);
      }
    }
    if (!grid_barrier(acc, gridDim.x, a.budget, int(blockIdx.x) != a.stall_block)) {
      ok = false;
      break;
    }

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
      // with runs, pass B walks its run backwards: it starts on the chunk
      // pass A just finished (its lists and records still cached), and the
      // next pass A starts on the chunk pass B finished last
      const int nb_ch = (c_hi - c_lo + c_step - 1) / c_step;
      for (int t = 0; t < nb_ch; ++t) {
        const int ch = runs ? c_hi - 1 - t : c_lo + t * c_step;
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
          pass_b<U, XT>(i < r.y ? i : r.x, i < r.y, a, G, pc, pn, es, ec);
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

  // kick + drift -> next step's state, with each scene's final p and a.  With
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
    for (int ch = c_lo; ch < c_hi; ch += c_step) {
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
        const float4 ak = a.a4[i];  // d_ii p + s of the final iterate
        const float p = pf[i];
        const float vx = va.x + inv_dt * ak.x;
        const float vy = va.y + inv_dt * ak.y;
        const float vz = va.z + inv_dt * ak.z;
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
      // a wait ran out: no block ran the epilogue, so the state is still the
      // step's input; time, dt and the statistics stay as they were and the
      // host reports SPH_E_TIMEOUT (the step can be taken again)
      if (flags & SPH_F_TIMEOUT) return;
      int iters = 0;
      double avg = 0.0, vmax_all = 0.0;
      const double dt_used0 = st->dt64[0];
      for (int s = 0; s < a.nscenes; ++s) {
        const float vm = __uint_as_float(*(volatile unsigned int*)&acc->vmax_bits[s]);
        if (!isfinite(vm)) flags |= SPH_F_NONFINITE;
        const bool capped = ok && acc->done[s] == 2 && c.fixed_iters <= 0;
        if (capped) flags |= SPH_F_NOT_CONVERGED;
        st->capped[s] = capped ? 1 : 0;
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

static int grad_mode(int sg, bool spline, bool tex = false) {
  return spline ? (tex ? kGradSplineTex : kGradSpline) : (sg <= 8192 ? kGradSmem : kGradFlat);
}
static size_t jacobi_smem(int mode, int sg) { return mode == kGradSmem ? sizeof(float2) * size_t(sg) : 0; }

using JacobiKernel = void (*)(JacobiArgs);

template <int GM>
static JacobiKernel pick_jacobi(int T, int ppt, int unroll) {
#define SPH_JACOBI_CASE(T_, P_, U_) \
  if (T == T_ && ppt == P_ && unroll == U_) return k_jacobi<GM, T_, P_, U_>;
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
  SPH_JACOBI_CASE(512, 1, 4)
  SPH_JACOBI_CASE(1024, 1, 4)
#undef SPH_JACOBI_CASE
  return nullptr;
}

static JacobiKernel jacobi_kernel(int mode, int T, int ppt, int unroll) {
  switch (mode) {
    case kGradSmem: return pick_jacobi<kGradSmem>(T, ppt, unroll);
    case kGradFlat: return pick_jacobi<kGradFlat>(T, ppt, unroll);
    case kGradSplineTex: return pick_jacobi<kGradSplineTex>(T, ppt, unroll);
    default: return pick_jacobi<kGradSpline>(T, ppt, unroll);
  }
}

bool jacobi_variant_ok(int block, int ppt, int unroll) {
  return pick_jacobi<kGradSpline>(block, ppt, unroll) != nullptr;
}

cudaError_t jacobi_config(int block, int ppt, int unroll, int sg, bool spline, int* blocks_per_sm, size_t* smem_out,
                          bool tex) {
  const int mode = grad_mode(sg, spline, tex);
  JacobiKernel k = jacobi_kernel(mode, block, ppt, unroll);
  if (!k) return cudaErrorInvalidValue;
  const size_t smem = jacobi_smem(mode, sg);
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
  JacobiKernel k = jacobi_kernel(grad_mode(a.c.sg, a.grad_spline != 0, a.yztex != 0), block, ppt, unroll);
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
