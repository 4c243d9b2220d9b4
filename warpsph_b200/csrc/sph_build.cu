// Neighbour build fused with everything of the step that depends only on
// positions and velocities.  One thread per sorted fluid particle scans the
// 3x3 rows of 5 x-adjacent half cells (9 contiguous particle ranges) of the fluid
// grid and of the boundary grid once, and produces:
//
//   ELL list of fluid neighbours    count_same/store_same_neighbor (IISPH.py:52-104)
//   fluid-boundary counts (+lists)  count_diff/store_diff_neighbor (IISPH.py:107-163)
//   rho                             compute_density (IISPH.py:177-214)
//   v_adv                           predict_v_adv (IISPH.py:217-278)
//   rho_adv                         predict_rho_adv (IISPH.py:281-329)
//   d_ii                            compute_term_d (IISPH.py:332-382)
//   a_ii                            compute_term_a (IISPH.py:385-428)
//   p for the first Jacobi pass     init_pressure + update_p (IISPH.py:166-174, 521-539),
//                                   and q = p / rho^2 in the position record's .w
//   B_i = sum_b psi_b gradW_ib      the boundary sum reused by every Jacobi pass
//
// With VIS_MU = 0 (the reference's default, main.py:61) v_adv = v - g dt y is
// local and everything above is one kernel (kBuildFull).  With viscosity,
// v_adv needs the neighbours' densities and rho_adv the neighbours' v_adv, so
// the step runs three list passes: kBuildLists (lists and rho), k_visc
// (v_adv with the laplacian), kBuildAdvect (the rest, reading v_adv).
//
// Membership uses the reference's float32 test |x_i - x_j| < h (IISPH.py:71-72)
// evaluated without contraction: r2 < r2_limit is exactly sqrt_rn(r2) < h.
//
// The per-pair vectors d_ij / d_ji the reference stores (IISPH.py:372-373,
// 24 B per pair) are not stored: the Jacobi passes recompute gradW from
// positions.  a_ii uses sum_j (d_ii - d_ji).gradW_ij
//   = d_ii . sum_j gradW_ij - (m dt^2 / rho_i^2) sum_j |gradW_ij|^2,
// both terms of which have the same sign, so the regrouping loses no accuracy.
#include "sph_internal.cuh"

namespace sph {

// Phase 1 of the build for one particle: filter the candidates of the 3x3
// rows of 5 x-adjacent half cells with the exact float32 test and write the hits
// into the particle's ELL list.  Only a compare and a predicated store run per
// candidate, so the warp stays converged; loads are issued four at a time.
// A record of a read-only float4 array, through the texture path when the
// array has a texture object (tex != 0), else with a read-only global load.
__device__ __forceinline__ float4 ro_load(const float4* __restrict__ p, unsigned long long tex, int j) {
  return tex ? tex1Dfetch<float4>(cudaTextureObject_t(tex), j) : __ldg(p + j);
}

__device__ inline int filter_rows(const Grid& g, int base, int3 ci, const int* __restrict__ cell_start,
                                  const float4* __restrict__ pts, float4 xi, float r2_limit, int self, int* out,
                                  int K, unsigned long long tex = 0) {
  int cnt = 0;
  const int x0 = max(ci.x - kXReach, 0), x1 = min(ci.x + kXReach, g.nx - 1);
  for (int cz = max(ci.z - 1, 0); cz <= min(ci.z + 1, g.nz - 1); ++cz) {
    for (int cy = max(ci.y - 1, 0); cy <= min(ci.y + 1, g.ny - 1); ++cy) {
      const int row = base + (cz * g.ny + cy) * g.nx;
      const int jb = __ldg(cell_start + row + x0), je = __ldg(cell_start + row + x1 + 1);
      int j = jb;
      for (; j + 4 <= je; j += 4) {
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = ro_load(pts, tex, j + u);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float r2 = dist2_rn(xi.x, xi.y, xi.z, q[u].x, q[u].y, q[u].z);
          if (r2 < r2_limit && j + u != self) {
            if (cnt < K) out[(long long)cnt * kWarp] = j + u;
            ++cnt;
          }
        }
      }
      for (; j < je; ++j) {
        const float4 q = ro_load(pts, tex, j);
        const float r2 = dist2_rn(xi.x, xi.y, xi.z, q.x, q.y, q.z);
        if (r2 < r2_limit && j != self) {
          if (cnt < K) out[(long long)cnt * kWarp] = j;
          ++cnt;
        }
      }
    }
  }
  return cnt;
}

// W and the gradient scalar of a listed neighbour (r < h; r2 = r^2) for the
// build's sums.  W always comes from the table (the densities follow the
// reference's interpolation); the gradient from its table, or in closed form
// when the gradient table is the cubic spline's own samples (one
// shared-memory load less per neighbour on the L1 data pipe; within 1.2e-6 of
// the table's interpolation, as in the solve).
template <class Tab>
struct TableKernel {
  Tab W, G;
  __device__ __forceinline__ float w(const Consts& c, float r, float) const { return table_lerp(W, r, c.w_scale, c.sw); }
  __device__ __forceinline__ float g(const Consts& c, float r, float) const { return grad_scalar(G, r, c); }
};
template <class Tab>
struct SplineKernel {
  Tab W;
  __device__ __forceinline__ float w(const Consts& c, float r, float) const { return table_lerp(W, r, c.w_scale, c.sw); }
  __device__ __forceinline__ float g(const Consts& c, float, float r2) const { return grad_spline(c, r2); }
};

template <int MODE, class Ker>
__device__ __forceinline__ void build_body(const BuildArgs& a, const Ker& ker);

// SMEM: the tables staged in shared memory; SPL: the gradient in closed form
// (only the W table is staged)
template <bool SMEM, int MODE, bool SPL>
__global__ void __launch_bounds__(256) k_build(BuildArgs a) {
  extern __shared__ float2 s_pairs[];
  if (SPL) {
    if (SMEM) {
      stage_pairs(s_pairs, a.w_table, a.c.sw);
      __syncthreads();
      build_body<MODE>(a, SplineKernel<PairTable>{PairTable{s_pairs}});
    } else {
      build_body<MODE>(a, SplineKernel<FlatTable>{FlatTable{a.w_table}});
    }
  } else if (SMEM) {
    stage_pairs(s_pairs, a.w_table, a.c.sw);
    stage_pairs(s_pairs + a.c.sw, a.g_table, a.c.sg);
    __syncthreads();
    build_body<MODE>(a, TableKernel<PairTable>{PairTable{s_pairs}, PairTable{s_pairs + a.c.sw}});
  } else {
    build_body<MODE>(a, TableKernel<FlatTable>{FlatTable{a.w_table}, FlatTable{a.g_table}});
  }
}

template <int MODE, class Ker>
__device__ __forceinline__ void build_body(const BuildArgs& a, const Ker& ker) {
  constexpr bool kLists = (MODE != kBuildAdvect);  // this pass builds the neighbour lists
  constexpr bool kTerms = (MODE != kBuildLists);   // this pass writes the advection terms
  const Consts c = a.c;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < a.n;
  int cnt = 0, cntb = 0;
  if (live) {
    const CellFrame fr = frame_of(a.scenes, a.grid, false, i);
    const Grid& g = fr.g;
    const float dt = a.st->dt[fr.scene];
    // v_adv of particle i and the term added to a neighbour's v to get its
    // v_adv: v - g dt y without viscosity, read back from k_visc with it
    const float gdt = (MODE == kBuildAdvect) ? 0.f : (-c.gravity) * dt;
    const float4 xi = a.pos[i];
    const float4 vi = (MODE == kBuildAdvect) ? a.vadv[i] : a.vel[i];
    const float4* vsrc = (MODE == kBuildAdvect) ? a.vadv : a.vel;
    const float vax = vi.x, vay = (MODE == kBuildAdvect) ? vi.y : vi.y + gdt, vaz = vi.z;
    const int3 ci = cell_coord(g, xi.x, xi.y, xi.z);
    const int K = c.max_ff, KB = c.max_fb;
    int* nbr = a.nbr_ff + ell_index(i, 0, K);
    int* nbrb = a.nbr_fb + ell_index(i, 0, KB);

    // phase 1: neighbour lists (the advect pass reads the lists built before)
    if (kLists) {
      cnt = filter_rows(g, fr.base, ci, a.cell_start, a.pos, xi, c.r2_limit, i, nbr, K, a.cand_tex);
      if (a.nb > 0) cntb = filter_rows(g, fr.base, ci, a.bcell_start, a.bpos, xi, c.r2_limit, -1, nbrb, KB);
    } else {
      cnt = a.cnt_ff[i];
      cntb = (a.nb > 0) ? a.cnt_fb[i] : 0;
    }

    // phase 2: everything summed over the neighbours, in list (= ascending j) order
    float sW = 0.f, sGx = 0.f, sGy = 0.f, sGz = 0.f, sG2 = 0.f, div = 0.f;
    auto fluid = [&](float4 xj, float4 vj) {
      const float r2 = dist2_rn(xi.x, xi.y, xi.z, xj.x, xj.y, xj.z);
      const float r = __fsqrt_rn(r2);
      sW += ker.w(c, r, r2);
      const float gs = ker.g(c, r, r2);
      const float gx = gs * (xj.x - xi.x), gy = gs * (xj.y - xi.y), gz = gs * (xj.z - xi.z);
      sGx += gx;
      sGy += gy;
      sGz += gz;
      sG2 += gx * gx + gy * gy + gz * gz;
      div += (vax - vj.x) * gx + (vay - (vj.y + gdt)) * gy + (vaz - vj.z) * gz;
    };
    const int nf = min(cnt, K);
    // the neighbours' velocities through the texture path only when they
    // are the step's velocities (not the v_adv the viscosity pass wrote)
    const unsigned long long vtex = (MODE == kBuildAdvect) ? 0ull : a.vel_tex;
    // compact form: (v_j, x_j) from the velocity record and (y_j, z_j) from
    // the 8-byte copy, 24 bytes per neighbour instead of two 16-byte records
    const unsigned long long yztex = (MODE == kBuildAdvect) ? 0ull : a.yz_tex;
    auto load = [&](int j, float4& xj, float4& vj) {
      if (yztex) {
        vj = tex1Dfetch<float4>(cudaTextureObject_t(vtex), j);
        const float2 yz = tex1Dfetch<float2>(cudaTextureObject_t(yztex), j);
        xj = make_float4(vj.w, yz.x, yz.y, 0.f);
      } else {
        xj = ro_load(a.pos, a.pos_tex, j);
        vj = ro_load(vsrc, vtex, j);
      }
    };
    int k = 0;
    for (; k + 4 <= nf; k += 4) {
      int j[4];
      float4 xj[4], vj[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) j[u] = nbr[(k + u) * kWarp];
#pragma unroll
      for (int u = 0; u < 4; ++u) load(j[u], xj[u], vj[u]);
#pragma unroll
      for (int u = 0; u < 4; ++u) fluid(xj[u], vj[u]);
    }
    for (; k < nf; ++k) {
      float4 xj, vj;
      load(nbr[k * kWarp], xj, vj);
      fluid(xj, vj);
    }

    float sWb = 0.f, Bx = 0.f, By = 0.f, Bz = 0.f, divb = 0.f;
    const int nbh = min(cntb, KB);
    for (int t = 0; t < nbh; ++t) {
      const int b = nbrb[t * kWarp];
      const float4 xb = __ldg(a.bpos + b);
      const float r2 = dist2_rn(xi.x, xi.y, xi.z, xb.x, xb.y, xb.z);
      const float r = __fsqrt_rn(r2);
      sWb += ker.w(c, r, r2) * xb.w;
      const float gs = ker.g(c, r, r2);
      const float gx = gs * (xb.x - xi.x), gy = gs * (xb.y - xi.y), gz = gs * (xb.z - xi.z);
      Bx += gx * xb.w;
      By += gy * xb.w;
      Bz += gz * xb.w;
      float wx = vax, wy = vay, wz = vaz;
      if (a.bvel) {
        const float4 vb = __ldg(a.bvel + b);
        wx -= vb.x;
        wy -= vb.y;
        wz -= vb.z;
      }
      divb += (wx * gx + wy * gy + wz * gz) * xb.w;
    }

    // compute_density (IISPH.py:214)
    const float rho = sW * c.m + sWb + c.w0 * c.m;
    // predict_rho_adv (IISPH.py:329)
    const float rho_adv = rho + (div * c.m + divb) * dt;
    // compute_term_d (IISPH.py:382): term_1 = -sum gradW_ij, term_2 = -sum psi gradW_ib
    const float dt2 = dt * dt;
    const float rr = rho * rho;
    const float dix = ((-sGx) * c.m + (-Bx)) * dt2 / rr;
    const float diy = ((-sGy) * c.m + (-By)) * dt2 / rr;
    const float diz = ((-sGz) * c.m + (-Bz)) * dt2 / rr;
    // compute_term_a (IISPH.py:428)
    const float t3 = c.m * dt2;
    const float aii = ((dix * sGx + diy * sGy + diz * sGz) - (t3 / rr) * sG2) * c.m + (dix * Bx + diy * By + diz * Bz);

    // initial pressure of the solve
    float p;
    if (c.warm_start == SPH_WARM_ZERO) {
      // p_0 = 0 gives Ap_0 = 0, so the first update_p (IISPH.py:534-539) is local
      float aa = aii;
      if (aa > -c.inv_small && aa < c.inv_small) aa = (aa < 0.f ? -1.f : 1.f) * c.inv_small;
      p = fmaxf(0.f + (c.rho0 - rho_adv - 0.f) * c.omega / aa, 0.f);
    } else if (c.warm_start == SPH_WARM_HALF) {
      p = a.pprev[i] / 2.0f;
    } else {
      p = 0.f;  // the learned warm start writes p_0 and q_0 after the build
    }

    a.rho[i] = rho;
    if (kLists) {
      a.cnt_ff[i] = cnt;
      if (a.cnt_fb) a.cnt_fb[i] = cntb;
    }
    if (kTerms) {
      a.bvec[i] = make_float4(Bx, By, Bz, rho_adv);
      a.dii_aii[i] = make_float4(dix, diy, diz, aii);
      if (MODE == kBuildFull) a.vadv[i] = make_float4(vax, vay, vaz, 0.f);
      if (c.warm_start != SPH_WARM_MLP) {
        a.p0[i] = p;
        // q = p / rho^2 for the solve's first pass; only .w of the record is
        // written, and other threads read only its .xyz in this kernel
        reinterpret_cast<float*>(a.pos_q + i)[3] = p / rr;
      }
    }

    if (kTerms && a.feat) {
      // Learned warm-start inputs (kFeatures per particle, dimensionless; the
      // network standardises them with its own mean / std).  Pressures span
      // orders of magnitude, so they enter as asinh(p / (rho0 g h)).
      // feature-major: feature c of sorted particle i at feat[c * feat_ld + i],
      // so each of a warp's stores (and the network's loads) is one 128-byte row
      float* f0 = a.feat + i;
      auto f = [&](int c) -> float& { return f0[(long long)c * a.feat_ld]; };
      const float inv_rho0 = 1.0f / c.rho0;
      const float p_ref = 1.0f / (c.rho0 * c.gravity * c.h);  // 1 / (rho0 g h)
      const float h2 = c.h * c.h, h4 = h2 * h2;
      float aa = aii;
      if (aa > -c.inv_small && aa < c.inv_small) aa = (aa < 0.f ? -1.f : 1.f) * c.inv_small;
      const float p1 = fmaxf((c.rho0 - rho_adv) * c.omega / aa, 0.f);  // first Jacobi iterate from p = 0
      const float gx = sGx * c.m + Bx, gy = sGy * c.m + By, gz = sGz * c.m + Bz;  // grad rho
      f(0) = rho_adv * inv_rho0 - 1.0f;                        // predicted density deviation
      f(1) = (rho_adv - rho) * inv_rho0;                       // velocity divergence over the step
      f(2) = aii * rr / (dt2 * c.m * c.m) * h4 * h4;           // a_ii in lattice units
      f(3) = asinhf((a.pprev ? a.pprev[i] : 0.f) * p_ref);     // previous-step pressure
      f(4) = float(cnt);                                       // fluid neighbour count
      f(5) = sWb * inv_rho0;                                   // boundary psi sum (density share)
      f(6) = sqrtf(gx * gx + gy * gy + gz * gz) * c.h * inv_rho0;  // |grad rho|
      f(7) = asinhf(p1 * p_ref);                               // Jacobi source term
      f(8) = gy * c.h * inv_rho0;                              // grad rho along gravity
      f(9) = float(cntb);                                      // boundary neighbour count
      // hydrostatic pressure of the fluid column above: depth below the
      // highest fluid particle of this grid column (x, z), in units of h
      const int3 top = make_int3(ci.x, 0, ci.z);
      const float depth = key_float(__ldg(a.coltop + fr.base + cell_index(g, top))) - xi.y;
      f(10) = asinhf(fmaxf(depth, 0.f) / c.h);
    }
  }
  // bookkeeping: overflow flags, pair totals, max counts (once per step)
  if (!kLists) return;
  const unsigned int full = 0xffffffffu;
  int over = live ? ((cnt > c.max_ff ? SPH_F_FF_OVERFLOW : 0) | (cntb > c.max_fb ? SPH_F_FB_OVERFLOW : 0)) : 0;
  unsigned long long pf = warp_sum((unsigned long long)cnt);
  unsigned long long pb = warp_sum((unsigned long long)cntb);
  int mf = warp_max(cnt), mb = warp_max(cntb);
  over = __reduce_or_sync(full, over);
  if ((threadIdx.x & 31) == 0) {
    if (pf) atomicAdd(&a.acc->pairs_ff, pf);
    if (pb) atomicAdd(&a.acc->pairs_fb, pb);
    atomicMax(&a.acc->max_ff, mf);
    atomicMax(&a.acc->max_fb, mb);
    if (over) atomicOr(&a.acc->flags, over);
  }
}

// Highest fluid y of each grid column (x, z): every sorted fluid particle
// raises the key of its column's bottom cell (cy = 0).
// Sorted neighbours usually share a column, so the lanes of a warp that do
// combine their keys first and one of them updates the column.
__global__ void k_column_top(BuildArgs a, unsigned int* coltop) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const CellFrame fr = frame_of(a.scenes, a.grid, false, i);
  const float4 xi = a.pos[i];
  int3 c = cell_coord(fr.g, xi.x, xi.y, xi.z);
  c.y = 0;
  const int col = fr.base + cell_index(fr.g, c);
  const unsigned int same = __match_any_sync(__activemask(), col);
  const unsigned int key = __reduce_max_sync(same, float_key(xi.y));
  if ((threadIdx.x & 31) == unsigned(__ffs(same) - 1)) atomicMax(coltop + col, key);
}

cudaError_t launch_column_top(const BuildArgs& a, unsigned int* coltop, int total_cells, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(coltop, 0, sizeof(unsigned int) * size_t(total_cells), s);
  if (e != cudaSuccess || a.n <= 0) return e;
  k_column_top<<<(a.n + 255) / 256, 256, 0, s>>>(a, coltop);
  return cudaGetLastError();
}

// predict_v_adv with viscosity (IISPH.py:217-278), after kBuildLists wrote
// the lists and every density:
//   term_1 = -sum_j gradW_ij ((v_i - v_j) . x_ij) / rho_j / r_ij^2
//   term_2 = -sum_b gradW_ib psi_b (v_i . x_ib) / r_ib^2
//   v_adv  = v + (10 (m term_1 + term_2 / rho0) mu / rho_i - g y) dt
// with x_ij = x_j - x_i and r the float32 length the list test used; the
// operations keep the reference's order (vector * scalar, then each division).
template <class Tab>
__device__ __forceinline__ void visc_body(const BuildArgs& a, const Tab& G) {
  const Consts c = a.c;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const CellFrame fr = frame_of(a.scenes, a.grid, false, i);
  const float dt = a.st->dt[fr.scene];
  const float4 xi = a.pos[i];
  const float4 vi = a.vel[i];
  const int K = c.max_ff, KB = c.max_fb;
  const int* nbr = a.nbr_ff + ell_index(i, 0, K);
  const int nf = min(a.cnt_ff[i], K);
  float t1x = 0.f, t1y = 0.f, t1z = 0.f;
  for (int k = 0; k < nf; ++k) {
    const int j = nbr[k * kWarp];
    const float4 xj = __ldg(a.pos + j);
    const float4 vj = __ldg(a.vel + j);
    const float rj = __ldg(a.rho + j);
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float r = __fsqrt_rn(dist2_rn(xi.x, xi.y, xi.z, xj.x, xj.y, xj.z));
    const float gs = grad_scalar(G, r, c);
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(vi.x - vj.x, dx), __fmul_rn(vi.y - vj.y, dy)),
                                __fmul_rn(vi.z - vj.z, dz));
    const float r2 = __fmul_rn(r, r);
    t1x -= __fdiv_rn(__fdiv_rn(__fmul_rn(__fmul_rn(gs, dx), dot), rj), r2);
    t1y -= __fdiv_rn(__fdiv_rn(__fmul_rn(__fmul_rn(gs, dy), dot), rj), r2);
    t1z -= __fdiv_rn(__fdiv_rn(__fmul_rn(__fmul_rn(gs, dz), dot), rj), r2);
  }
  float t2x = 0.f, t2y = 0.f, t2z = 0.f;
  if (a.nb > 0) {
    const int* nbrb = a.nbr_fb + ell_index(i, 0, KB);
    const int nbh = min(a.cnt_fb[i], KB);
    for (int t = 0; t < nbh; ++t) {
      const int b = nbrb[t * kWarp];
      const float4 xb = __ldg(a.bpos + b);
      const float dx = xb.x - xi.x, dy = xb.y - xi.y, dz = xb.z - xi.z;
      const float r = __fsqrt_rn(dist2_rn(xi.x, xi.y, xi.z, xb.x, xb.y, xb.z));
      const float gs = grad_scalar(G, r, c);
      const float dot = __fadd_rn(__fadd_rn(__fmul_rn(vi.x, dx), __fmul_rn(vi.y, dy)), __fmul_rn(vi.z, dz));
      const float r2 = __fmul_rn(r, r);
      t2x -= __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(gs, dx), xb.w), dot), r2);
      t2y -= __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(gs, dy), xb.w), dot), r2);
      t2z -= __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(gs, dz), xb.w), dot), r2);
    }
  }
  const float ri = a.rho[i];
  const float lx = 10.f * __fadd_rn(__fmul_rn(t1x, c.m), __fdiv_rn(t2x, c.rho0));
  const float ly = 10.f * __fadd_rn(__fmul_rn(t1y, c.m), __fdiv_rn(t2y, c.rho0));
  const float lz = 10.f * __fadd_rn(__fmul_rn(t1z, c.m), __fdiv_rn(t2z, c.rho0));
  const float ax = __fdiv_rn(__fmul_rn(lx, c.mu), ri);
  const float ay = __fadd_rn(__fdiv_rn(__fmul_rn(ly, c.mu), ri), -c.gravity);
  const float az = __fdiv_rn(__fmul_rn(lz, c.mu), ri);
  a.vadv[i] = make_float4(__fadd_rn(vi.x, __fmul_rn(ax, dt)), __fadd_rn(vi.y, __fmul_rn(ay, dt)),
                          __fadd_rn(vi.z, __fmul_rn(az, dt)), 0.f);
}

template <bool SMEM>
__global__ void __launch_bounds__(256) k_visc(BuildArgs a) {
  extern __shared__ float2 s_pairs[];
  if (SMEM) {
    stage_pairs(s_pairs, a.g_table, a.c.sg);
    __syncthreads();
    visc_body(a, PairTable{s_pairs});
  } else {
    visc_body(a, FlatTable{a.g_table});
  }
}

// compute_boundary_density (IISPH.py:23-49): psi_b = rho0 / (W(0) + sum_{b' != b} W(r)).
__global__ void __launch_bounds__(256) k_psi(PsiArgs a, float* psi) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nb) return;
  const Consts c = a.c;
  const CellFrame fr = frame_of(a.scenes, a.grid, true, b);
  const Grid& g = fr.g;
  const float4 xb = a.bpos[b];
  const int3 ci = cell_coord(g, xb.x, xb.y, xb.z);
  float rho = a.w0_from_table ? __ldg(a.w_table) : c.w0;
  const int x0 = max(ci.x - kXReach, 0), x1 = min(ci.x + kXReach, g.nx - 1);
  for (int cz = max(ci.z - 1, 0); cz <= min(ci.z + 1, g.nz - 1); ++cz)
    for (int cy = max(ci.y - 1, 0); cy <= min(ci.y + 1, g.ny - 1); ++cy) {
      const int row = fr.base + (cz * g.ny + cy) * g.nx;
      for (int j = a.bcell_start[row + x0]; j < a.bcell_start[row + x1 + 1]; ++j) {
        if (j == b) continue;
        const float4 xj = a.bpos[j];
        const float r2 = dist2_rn(xb.x, xb.y, xb.z, xj.x, xj.y, xj.z);
        if (r2 < c.r2_limit) rho += table_lerp(a.w_table, __fsqrt_rn(r2), c.w_scale, c.sw);
      }
    }
  psi[b] = c.rho0 / rho;
}

__global__ void k_pack_psi(int nb, const float* __restrict__ psi, float4* bpos) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) bpos[b].w = psi[b];
}

static size_t table_bytes(const Consts& c) { return sizeof(float2) * (size_t(c.sw) + size_t(c.sg)); }
static bool tables_fit_smem(const Consts& c) { return table_bytes(c) <= 96 * 1024; }

template <int MODE>
static cudaError_t launch_build_mode(const BuildArgs& a, int grid, int block, cudaStream_t s) {
  if (a.spline) {
    const size_t smem = sizeof(float2) * size_t(a.c.sw);
    if (smem <= 96 * 1024) {
      if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(k_build<true, MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
      }
      prefer_l1(k_build<true, MODE, true>, block, smem);
      k_build<true, MODE, true><<<grid, block, smem, s>>>(a);
    } else {
      k_build<false, MODE, true><<<grid, block, 0, s>>>(a);
    }
  } else if (tables_fit_smem(a.c)) {
    const size_t smem = table_bytes(a.c);
    if (smem > 48 * 1024) {
      cudaError_t e =
          cudaFuncSetAttribute(k_build<true, MODE, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) return e;
    }
    prefer_l1(k_build<true, MODE, false>, block, smem);
    k_build<true, MODE, false><<<grid, block, smem, s>>>(a);
  } else {
    k_build<false, MODE, false><<<grid, block, 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_build(const BuildArgs& a, int block, int mode, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const int grid = (a.n + block - 1) / block;
  switch (mode) {
    case kBuildFull: return launch_build_mode<kBuildFull>(a, grid, block, s);
    case kBuildLists: return launch_build_mode<kBuildLists>(a, grid, block, s);
    case kBuildAdvect: return launch_build_mode<kBuildAdvect>(a, grid, block, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_visc(const BuildArgs& a, int block, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const int grid = (a.n + block - 1) / block;
  const size_t smem = sizeof(float2) * size_t(a.c.sg);
  if (smem <= 96 * 1024) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_visc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) return e;
    }
    k_visc<true><<<grid, block, smem, s>>>(a);
  } else {
    k_visc<false><<<grid, block, 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_psi(const PsiArgs& a, int block, cudaStream_t s) {
  if (a.nb <= 0) return cudaSuccess;
  float* psi = nullptr;
  cudaError_t e = cudaMallocAsync(&psi, sizeof(float) * a.nb, s);
  if (e != cudaSuccess) return e;
  const int grid = (a.nb + block - 1) / block;
  k_psi<<<grid, block, 0, s>>>(a, psi);
  k_pack_psi<<<grid, block, 0, s>>>(a.nb, psi, a.bpos);
  e = cudaGetLastError();
  cudaError_t f = cudaFreeAsync(psi, s);
  return e != cudaSuccess ? e : f;
}

// psi in sorted boundary order into a caller-provided buffer, with no
// allocation (used by the no-allocation entry point).
cudaError_t launch_psi_sorted(const PsiArgs& a, float* psi_sorted, int block, cudaStream_t s) {
  if (a.nb <= 0) return cudaSuccess;
  k_psi<<<(a.nb + block - 1) / block, block, 0, s>>>(a, psi_sorted);
  return cudaGetLastError();
}

}  // namespace sph
