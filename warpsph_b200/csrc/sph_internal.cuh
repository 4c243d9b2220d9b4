// Internal structures and device helpers of libwpsph (sm_100a).
//
// Data layout (HBM), all in the cell-sorted particle order of the current step:
//   pos  float4 (x, y, z, q)          vel  float4 (vx, vy, vz, 0)
//        q = p / rho^2 of the current pressure iterate in the solve's work
//        array (first written by the build or the warm-start network, then by
//        every Jacobi update); the step's state arrays carry 0 there.  With
//        the texture path on, the work copy of vel carries x in .w and a
//        float2 (y, z) copy of pos sits beside it: the build's second phase
//        and the solve's pass B gather a position as (x from a 16-byte record
//        they read anyway) + 8 bytes
//   a4   float4 (a, x)                a = d_ii p + s of the current iterate
//   bpos float4 (x, y, z, psi)        boundary, sorted once
//   nbr  int32, tile-major ELL: element k of particle i sits at
//        (i/32)*32*K + k*32 + i%32, so a warp reading its k-th neighbours
//        issues one coalesced 128-byte load.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wpsph.h"

namespace sph {

constexpr int kWarp = 32;
constexpr int kFeatures = 11;  // learned warm-start inputs per particle

// Uniform neighbour grid.  Cell size is slightly above h (cell = 1.01 h or
// coarser) in y and z; along x, the direction in which sorted rows run, cells
// are cut in half (kXSplit), so a particle's neighbours within h lie in the
// 5 half cells x-2..x+2 of the 3 x 3 rows around it: 2.5 cells wide instead
// of 3, with the same 0.01 h margin for float32 rounding of the coordinate.
// Coordinates outside the grid are clamped to the edge cells: clamping is
// monotone and 1-Lipschitz in cell space, so the search stays complete for
// particles that leave the domain.
constexpr int kXSplit = 2;  // half cells along x
constexpr int kXReach = 2;  // half cells searched on each side
struct Grid {
  float ox, oy, oz;  // origin
  float inv_cell;    // 1 / cell (y, z)
  float inv_cell_x;  // kXSplit / cell
  int nx, ny, nz;    // nx counts half cells
  int ncells;
};

__host__ __device__ inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ inline int3 cell_coord(const Grid& g, float x, float y, float z) {
  int cx = __float2int_rd((x - g.ox) * g.inv_cell_x);
  int cy = __float2int_rd((y - g.oy) * g.inv_cell);
  int cz = __float2int_rd((z - g.oz) * g.inv_cell);
  return make_int3(clampi(cx, 0, g.nx - 1), clampi(cy, 0, g.ny - 1), clampi(cz, 0, g.nz - 1));
}
__device__ inline int cell_index(const Grid& g, int3 c) { return (c.z * g.ny + c.y) * g.nx + c.x; }

// Constants of the physics, as the float32 values the reference kernels see.
struct Consts {
  float h;          // fp32(SMOOTHING_LENGTH)
  float r2_limit;   // neighbour iff r2 < r2_limit  <=>  sqrt_rn(r2) < h (exact)
  float w_scale;    // fp32(W_SIZE-1) * fp32(1/h), as sph_funcs.py:97 evaluates it
  float g_scale;    // fp32(GRAD_W_SIZE-1) * fp32(1/h) (sph_funcs.py:112)
  int sw, sg;       // table sizes
  float rho0, gravity, omega, inv_small, mu, m;
  float w0;         // spline_W(0) = W_table[0]
  float eta;
  int min_iter, max_loop, fixed_iters, warm_start;
  int max_ff, max_fb, keep_fb;
  // the cubic spline's gradient scalar -(dW/dr)/r in closed form:
  // gi0 - gi1 r for r^2 <= h2q = h^2/4, go (h - r)^2 / r above
  float gi0, gi1, go, h2q;
};

// Independent scenes solved together (batching).  Scene s owns fluid slots
// [fluid_off[s], fluid_off[s+1]), boundary slots [bound_off[s], ...), its own
// grid, and global cell ids [cell_base[s], cell_base[s+1]): keys of different
// scenes never mix, so the cell sort keeps every scene in its slot range and
// neighbour searches never cross scenes.  Jacobi work is cut into warp-aligned
// chunks of at most one solve block's worth of particles ((threads per block)
// x (particles per thread)) that never straddle scenes, as many as the
// persistent grid takes in whole rounds: chunks [chunk_off[s], chunk_off[s+1])
// belong to scene s.  A single scene is the case nscenes = 1.
constexpr int kMaxScenes = 256;

struct SceneTable {
  int nscenes;
  int cell_base[kMaxScenes + 1];
  int fluid_off[kMaxScenes + 1];
  int bound_off[kMaxScenes + 1];
  int chunk_off[kMaxScenes + 1];
  Grid grid[kMaxScenes];
};

__device__ __forceinline__ int find_scene(const int* __restrict__ off, int nscenes, int i) {
  int lo = 0, hi = nscenes;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Grid and cell-id base of slot i of a fluid (or boundary) array; without a
// scene table the single grid passed by value applies.
struct CellFrame {
  Grid g;
  int base;
  int scene;
};
__device__ __forceinline__ CellFrame frame_of(const SceneTable* T, const Grid& g0, bool boundary, int i) {
  CellFrame f;
  if (!T) {
    f.g = g0;
    f.base = 0;
    f.scene = 0;
    return f;
  }
  const int S = T->nscenes;
  f.scene = (S == 1) ? 0 : find_scene(boundary ? T->bound_off : T->fluid_off, S, i);
  f.g = T->grid[f.scene];
  f.base = T->cell_base[f.scene];
  return f;
}

// Scalars carried across steps, per scene (device resident: no host sync per step).
struct DevState {
  double dt64[kMaxScenes], inv_dt64[kMaxScenes];  // dt, 1/dt as the reference holds them
  double sim_time[kMaxScenes];
  float dt[kMaxScenes], inv_dt[kMaxScenes];       // what the kernels use (float32 arguments)
  int capped[kMaxScenes];                         // 1: the last solve stopped at the iteration cap
  long long step_index;
};

// Per-step accumulators, zeroed at the start of every step.
struct StepAcc {
  int flags;
  int max_ff, max_fb;
  unsigned int bar_count, bar_gen, done_blocks;
  int all_done;
  int pad0;
  unsigned long long pairs_ff, pairs_fb;
  int iterations[kMaxScenes];
  int done[kMaxScenes];       // 0 running, 1 converged, 2 stopped at the iteration cap
  int final_buf[kMaxScenes];  // which pressure buffer holds the scene's final p
  unsigned int vmax_bits[kMaxScenes];
  double avg_err[kMaxScenes];
};

struct Partial {
  double sum;
  long long cnt;
};

constexpr int kStatsRing = 4096;

// ------------------------------------------------------------------ math

__device__ inline float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }

// Kernel tables.  A lookup needs the two samples bracketing r; the shared-memory
// copy stores them as float2 pairs (T[k], T[k+1]) so one 8-byte load serves a
// lookup (half the shared-memory wavefronts of two 4-byte loads).  Large tables
// (the reference's 65536-sample gradient table) stay in global memory.
struct FlatTable {
  const float* T;
  __device__ __forceinline__ float2 pair(int lo) const { return make_float2(__ldg(T + lo), __ldg(T + lo + 1)); }
};
struct PairTable {
  const float2* P;
  __device__ __forceinline__ float2 pair(int lo) const { return P[lo]; }
};

// Linear interpolation of sph_funcs.py:97-102 / 112-117, for r < h.
template <class Tab>
__device__ __forceinline__ float table_lerp(const Tab& t, float r, float scale, int S) {
  const float f = r * scale;
  const int lo = min(__float2int_rz(f), S - 2);
  const float a = f - float(lo);
  const float2 p = t.pair(lo);
  return (1.0f - a) * p.x + a * p.y;
}
__device__ __forceinline__ float table_lerp(const float* T, float r, float scale, int S) {
  return table_lerp(FlatTable{T}, r, scale, S);
}

// spline_W (sph_funcs.py:92-102)
template <class Tab>
__device__ __forceinline__ float spline_W(const Tab& T, float r, const Consts& c) {
  if (r >= c.h) return 0.0f;
  return table_lerp(T, r, c.w_scale, c.sw);
}

// Scalar part of grad_spline_W (sph_funcs.py:105-118): 0 outside (1e-10, h).
template <class Tab>
__device__ __forceinline__ float grad_scalar(const Tab& T, float r, const Consts& c) {
  if (r >= c.h || r < 1e-10f) return 0.0f;
  return table_lerp(T, r, c.g_scale, c.sg);
}

// Gradient scalar of the cubic spline (the function the gradient table
// samples, sph_funcs.py:79-82) evaluated in closed form for a listed
// neighbour, from r^2.  At r = 0 it returns the inner branch's finite value,
// and the direction vector (zero) makes the term vanish.
__device__ __forceinline__ float grad_spline(const Consts& c, float r2) {
  const float ir = rsqrtf(fmaxf(r2, 1e-30f));
  const float r = r2 * ir;
  const float t = c.h - r;
  return (r2 <= c.h2q) ? fmaf(-c.gi1, r, c.gi0) : c.go * t * t * ir;
}

// Stage a table into shared memory as (T[k], T[k+1]) pairs, k < S-1.
__device__ __forceinline__ void stage_pairs(float2* dst, const float* __restrict__ T, int S) {
  for (int k = threadIdx.x; k < S - 1; k += blockDim.x) dst[k] = make_float2(T[k], T[k + 1]);
}

// The gradient table as the Jacobi passes read it: (T[k], T[k+1] - T[k])
// pairs in shared memory, so an interpolation is one FMA, T[k] + a (T[k+1] -
// T[k]); it differs from the reference's (1 - a) T[k] + a T[k+1] by rounding
// only.  FlatSlopeTable is the same lookup on a table in global memory.
struct SlopeTable {
  const float2* P;
  __device__ __forceinline__ float lerp(int lo, float a) const {
    const float2 p = P[lo];
    return fmaf(a, p.y, p.x);
  }
};
struct FlatSlopeTable {
  const float* T;
  __device__ __forceinline__ float lerp(int lo, float a) const {
    const float t0 = __ldg(T + lo);
    return fmaf(a, __ldg(T + lo + 1) - t0, t0);
  }
};
__device__ __forceinline__ void stage_slopes(float2* dst, const float* __restrict__ T, int S) {
  for (int k = threadIdx.x; k < S - 1; k += blockDim.x) {
    const float t0 = T[k];
    dst[k] = make_float2(t0, T[k + 1] - t0);
  }
}

// Scalar part of gradW for a listed neighbour (r < h by the list's exact
// test) inside the Jacobi passes.  The reference's guards are not needed here:
// at r = 0 the gradient's direction vector is zero, so the product is zero
// whatever the table returns; an r that the approximate root rounds up to h
// clamps to the last segment, whose end sample is 0; NaN converts to index 0.
template <class Tab>
__device__ __forceinline__ float grad_listed(const Tab& t, float r, float scale, int S) {
  const float f = r * scale;
  const int lo = min(__float2int_rz(f), S - 2);
  return t.lerp(lo, f - float(lo));
}

// Square root for the kernel-table argument inside the Jacobi passes, where
// the neighbour sets are already fixed.  The approximate instruction differs
// from the rounded root by a few ulp, which moves a table lookup by ~1e-7
// relative; the parity tests bound the effect on p.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The gradient scalar of a listed neighbour as the Jacobi passes evaluate it,
// from r^2: in closed form when the gradient table is the cubic spline's own
// (SplineGrad; it differs from the table's interpolation by at most 1.2e-6 of
// the table's largest value at 1024 samples, and it needs no shared-memory
// load, which the L1 data pipe bounding the passes would otherwise serve), else
// from the table (TableGrad).
struct SplineGrad {
  __device__ __forceinline__ float operator()(const Consts& c, float r2) const { return grad_spline(c, r2); }
};
template <class Tab>
struct TableGrad {
  Tab t;
  __device__ __forceinline__ float operator()(const Consts& c, float r2) const {
    return grad_listed(t, sqrt_approx(r2), c.g_scale, c.sg);
  }
};

// Exact float32 |a-b|^2 as wp.length(a - b) squares it: no contraction,
// x*x + y*y + z*z left to right.
__device__ inline float dist2_rn(float ax, float ay, float az, float bx, float by, float bz) {
  float dx = __fsub_rn(ax, bx), dy = __fsub_rn(ay, by), dz = __fsub_rn(az, bz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ inline long long ell_index(long long i, int k, int K) {
  return (i >> 5) * (long long)(kWarp * K) + (long long)k * kWarp + (i & 31);
}

// ------------------------------------------------------------------ reductions

template <typename T>
__device__ inline T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ------------------------------------------------------------------ grid barrier

__device__ inline unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ inline int ld_volatile_int(const int* p) { return *(volatile const int*)p; }

// Grid-wide barrier for a cooperative (co-resident) launch.  Every wait is
// bounded by `budget` SM cycles; on expiry it sets SPH_F_TIMEOUT and returns
// false, and every later barrier returns false at once, so the kernel always
// terminates and the host reads SPH_E_TIMEOUT.  arrive = false (a test hook,
// sph_test_stall_barrier) makes this block wait without arriving, so that
// every block's wait runs out.
__device__ inline bool grid_barrier(StepAcc* acc, unsigned int nblocks, long long budget, bool arrive = true) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = (ld_volatile_int(&acc->flags) & SPH_F_TIMEOUT) ? 0 : 1;
    if (ok) {
      unsigned int gen = ld_acquire(&acc->bar_gen);
      __threadfence();
      unsigned int arrived = arrive ? atomicAdd(&acc->bar_count, 1u) : 0u;
      if (arrive && arrived == nblocks - 1) {
        atomicExch(&acc->bar_count, 0u);
        __threadfence();
        atomicAdd(&acc->bar_gen, 1u);
      } else {
        long long t0 = clock64();
        while (ld_acquire(&acc->bar_gen) == gen) {
          if (ld_volatile_int(&acc->flags) & SPH_F_TIMEOUT) { ok = 0; break; }
          if (clock64() - t0 > budget) {
            atomicOr(&acc->flags, SPH_F_TIMEOUT);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ------------------------------------------------------------------ kernel args

struct SortArgs {
  int n;
  Grid grid;                 // used when scenes == nullptr
  const SceneTable* scenes;  // per-scene grids (nullable)
  int boundary;              // 1: slots are boundary particles
  const float4* pos;   // unsorted (current state order)
  const int* orig;     // original id per particle of that order
  int* key;
  int* rank;
  int* cell_count;     // ncells, zeroed
  int* cell_start;     // ncells + 1
  int* scan_part;      // partial sums per scan block (two-kernel scan)
  // single-pass scan (used when scan_status != nullptr): per tile of cells a
  // 64-bit status word (flag << 32 | sum), zeroed by k_cell_keys, the tile
  // ticket, and where a look-back that waited too long sets SPH_F_TIMEOUT
  unsigned long long* scan_status;
  unsigned int* scan_ticket;
  int* err;
  int* sort_src;       // new index -> old index
  int* sort_orig;      // new index -> original id
};

struct BuildArgs {
  int n, nb;
  int spline;              // 1: the gradient table is the cubic spline's own (closed form in the build)
  Grid grid;
  const SceneTable* scenes;
  Consts c;
  const float* w_table;
  const float* g_table;
  const float4* pos;       // sorted fluid
  const float4* vel;
  const float* pprev;      // previous-step pressure, sorted (warm start)
  const float* pmlp;       // MLP warm-start prediction, sorted (SPH_WARM_MLP)
  const int* cell_start;   // fluid
  const float4* bpos;      // sorted boundary (x, y, z, psi)
  const float4* bvel;
  const int* bcell_start;
  const DevState* st;
  StepAcc* acc;
  int* nbr_ff;
  int* cnt_ff;
  int* nbr_fb;             // optional
  int* cnt_fb;
  float* rho;
  float4* bvec;            // (sum_b psi_b gradW_ib, rho_adv)
  float4* dii_aii;         // (d_ii, a_ii)
  float4* vadv;
  float* p0;               // initial pressure of the solve (p_1 for the zero warm start)
  float4* pos_q;           // the array `pos` points to: p0 / rho^2 goes into .w
  float* feat;             // optional MLP inputs, feature-major (kFeatures x feat_ld), NULL to skip
  long long feat_ld;       // feature c of sorted particle i at feat[c * feat_ld + i]
  const unsigned int* coltop;  // with feat: per grid column (x, z), the highest fluid y (ordered key)
  // texture objects over pos and vel (0: plain read-only loads): the second
  // phase's neighbour gathers, and (cand_tex) the first phase's candidates
  unsigned long long pos_tex, vel_tex, cand_tex;
  // texture object over the (y, z) copy of pos (0: none); when set, vel's .w
  // holds x and the second phase gathers (v, x) and (y, z) instead of pos and v
  unsigned long long yz_tex;
};

// Order-preserving uint key of a float (atomicMax on keys = max on floats);
// key 0 is below every float's key.
__device__ __forceinline__ unsigned int float_key(float y) {
  const unsigned int u = __float_as_uint(y);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct JacobiArgs {
  int n;
  int nscenes, nchunks;
  const int2* chunks;        // [start, end) particle slots of each chunk
  const int* chunk_scene;
  const SceneTable* scenes;
  Consts c;
  const float* g_table;
  float4* pos;             // (x, y, z, q = p / rho^2): .w is rewritten by every update
  const int* nbr_ff;
  const int* cnt_ff;
  const float* rho;
  const float4* bvec;
  const float4* dii_aii;
  const float4* vadv;
  const int* orig_w;
  float* p_a;              // ping
  float* p_b;              // pong
  float4* a4;              // (d_ii p + s, x): dt^2 times the pressure acceleration, and x of the position
  float* Ap;
  Partial* partials;       // one per chunk
  DevState* st;
  StepAcc* acc;
  SphStepStats* ring;      // per-step stats ring buffer
  SphStepStats* last;      // stats of the last completed step
  float4* bpos;            // sorted boundary (x, y, z, psi), moved by v dt after the drift
  const float4* bvel;
  int nb, move_boundary;
  // outputs of the kick/drift epilogue (next step's state)
  float4* pos_out;
  float4* vel_out;
  int* orig_out;
  float* p_out;
  int start_iter;          // 1: p_1 came from the build; 0: warm start, run pass 0
  int grad_spline;         // 1: the gradient table is the cubic spline's (closed form in the passes)
  unsigned long long yztex; // texture object over (y, z) of pos (0: none): pass B then takes x_j from a4's .w
                            // and fetches (y_j, z_j) through the texture path
  long long budget;        // barrier spin budget in SM cycles
  int stall_block;         // test hook: this block skips its first barrier arrival (-1: none)
  double dt_max, cfl_len, inv_small_d, eta_d;
};

struct PsiArgs {
  int nb;
  Grid grid;
  const SceneTable* scenes;
  Consts c;
  const float* w_table;
  float4* bpos;            // in: x,y,z; out: w = psi
  const int* bcell_start;
  int w0_from_table;       // 1: W(0) is read from w_table[0] on the device instead of c.w0
};

// Shared-memory carveout hint for a kernel that reads its neighbours through
// the L1: the smallest share of the SM's unified L1 / shared storage that
// still holds every block the registers and threads allow, so the rest stays
// L1.  Left to itself the driver gave the build's 8 blocks of 9 KB a 132 KB
// carveout (about 120 KB of L1); with the hint it takes 100 KB.  The solve
// does not use it: for its 4 blocks of 1.2 KB the driver answered the hint
// with 64 KB where it picks 16 KB by itself.  A hint only: errors are
// cleared and ignored.
template <class Kernel>
inline void prefer_l1(Kernel* k, int block, size_t dyn_smem) {
  int dev = 0, per_sm = 0, reserved = 0, nb = 0;
  cudaFuncAttributes fa{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaFuncGetAttributes(&fa, k) != cudaSuccess ||
      cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, block, dyn_smem) != cudaSuccess || per_sm <= 0) {
    cudaGetLastError();
    return;
  }
  const size_t need = size_t(nb) * (fa.sharedSizeBytes + dyn_smem + size_t(reserved));
  size_t pct = (100 * need + size_t(per_sm) - 1) / size_t(per_sm);
  if (pct > 100) pct = 100;
  if (cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, int(pct)) != cudaSuccess)
    cudaGetLastError();
}

// launchers (host)
cudaError_t launch_sort(const SortArgs& a, int ncells, cudaStream_t s);
// neighbour-build passes: one fused pass without viscosity, or lists + rho,
// then launch_visc (v_adv), then the advection terms
constexpr int kBuildFull = 0, kBuildLists = 1, kBuildAdvect = 2;
cudaError_t launch_build(const BuildArgs& a, int block, int mode, cudaStream_t s);
cudaError_t launch_visc(const BuildArgs& a, int block, cudaStream_t s);
// highest fluid y of every grid column (x, z) into a.coltop (zeroed first)
cudaError_t launch_column_top(const BuildArgs& a, unsigned int* coltop, int total_cells, cudaStream_t s);
cudaError_t launch_psi(const PsiArgs& a, int block, cudaStream_t s);
cudaError_t launch_psi_sorted(const PsiArgs& a, float* psi_sorted, int block, cudaStream_t s);
cudaError_t launch_gather(int n, const int* sort_src, const int* sort_orig, const float4* pos_in,
                          const float4* vel_in, const float* p_in, float4* pos_out, float4* vel_out,
                          int* orig_out, float* p_out, cudaStream_t s, float2* yz_out = nullptr);
bool jacobi_variant_ok(int block, int ppt, int unroll);
cudaError_t jacobi_config(int block, int ppt, int unroll, int sg, bool spline, int* blocks_per_sm, size_t* smem,
                          bool tex = false);
cudaError_t launch_jacobi(const JacobiArgs& a, int grid, int block, int ppt, int unroll, size_t smem,
                          cudaStream_t s);
cudaError_t launch_pack_fluid(int n, int base, const float* x3, const float* v3, float4* pos, float4* vel,
                              int* orig, float* p, cudaStream_t s, const float* p_in = nullptr);
cudaError_t launch_unsort4(int n, const int* orig, const float4* src, int component, float* out, cudaStream_t s);
cudaError_t launch_unsort1(int n, const int* orig, const float* src, float* out, cudaStream_t s);
cudaError_t launch_sort1(int n, const int* orig, const float* src, float* out, cudaStream_t s);

}  // namespace sph
