// C ABI of libwpsph (include/wpsph.h): context, device memory, the per-step
// launch sequence and its CUDA graph, and host readback in original order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sph_internal.cuh"
#include "sph_mlp.cuh"

using sph::Consts;
using sph::DevState;
using sph::Grid;
using sph::StepAcc;

struct SphCtx {
  SphParams P{};
  std::string err;
  int dev = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  int clock_khz = 0;
  Consts c{};
  bool grid_valid = false;
  int ncells_cap = 0;

  // scenes (a single scene is nscenes = 1)
  int S = 1;
  std::vector<int64_t> f_off{0, 0}, b_off{0, 0};  // host prefix offsets of fluid / boundary slots
  std::vector<Grid> grids;                        // per scene
  std::vector<int> cell_base;                     // prefix of per-scene cell counts
  std::vector<double> domains;                    // 6 per scene (min xyz, max xyz); zero extent = fit
  int total_cells = 0;
  sph::SceneTable* d_scenes = nullptr;
  int2* d_chunks = nullptr;
  int* d_chunk_scene = nullptr;
  int nchunks = 0;

  std::vector<float> w_host, g_host;
  float* d_w = nullptr;
  float* d_g = nullptr;
  // the gradient table is the cubic spline's own (sampled as build_tables
  // does): the solve may then evaluate the gradient in closed form
  bool g_spline = true;

  // boundary (host copy in original order, to re-sort when the grid changes)
  int64_t nb = 0;
  std::vector<float> bx_host, bv_host;
  bool b_moving = false;
  float4* bpos = nullptr;
  float4* bvel = nullptr;
  int* borig = nullptr;
  // per-step re-sort of a moving boundary (move_boundary): keys and temporaries
  float4 *bpos_t = nullptr, *bvel_t = nullptr;
  int *borig_t = nullptr, *bkey = nullptr, *brank = nullptr, *bsrc = nullptr;
  int* bcell_start = nullptr;

  // fluid
  int64_t n = 0, n_cap = 0;
  int K_ff = 0, K_fb = 0;
  float4 *pos_s = nullptr, *vel_s = nullptr, *pos_w = nullptr, *vel_w = nullptr;
  float2* yz_w = nullptr;  // (y, z) of pos_w: pass B's compact position gathers
  int *orig_s = nullptr, *orig_w = nullptr;
  float *p_s = nullptr, *pprev_w = nullptr;
  int *key = nullptr, *rank = nullptr, *sort_src = nullptr, *sort_orig = nullptr;
  int *cell_count = nullptr, *cell_start = nullptr, *scan_part = nullptr;
  unsigned long long* scan_status = nullptr;  // single-pass scan: tile states, then the ticket
  int scan_tiles_cap = 0;
  unsigned int* coltop = nullptr;  // per grid column, the highest fluid y (warm-start input 10)
  int *nbr_ff = nullptr, *cnt_ff = nullptr, *nbr_fb = nullptr, *cnt_fb = nullptr;
  float* rho = nullptr;
  float4 *bvec = nullptr, *dii_aii = nullptr, *vadv = nullptr, *a4 = nullptr;
  float *p_a = nullptr, *p_b = nullptr, *Ap = nullptr;
  float* pmlp = nullptr;
  float* feat = nullptr;             // learned warm-start inputs, kFeatures per particle
  float* p_start = nullptr;          // the solve's starting iterate, kept while recording features
  sph::MlpPacked* mlp = nullptr;     // packed network weights
  bool have_mlp = false;
  bool record_feat = false;
  float* stage = nullptr;  // 7 floats per particle: host<->device exchange

  sph::Partial* partials = nullptr;  // [cooperative block][scene]
  int64_t partials_cap = 0;
  int coop_grid = 0;
  int blocks_per_sm = 0;
  size_t jac_smem = 0;
  int jac_block = 1024, jac_ppt = 1, jac_unroll = 4;  // autotuner knobs of the solve
  bool jac_tex = false;                               // pass B reads x_j through the texture path
  cudaTextureObject_t pos_tex = 0;                    // over pos_w, when jac_tex
  cudaTextureObject_t vel_tex = 0;                    // over vel_w, when jac_tex
  cudaTextureObject_t yz_tex = 0;                     // over yz_w, when jac_tex
  int stall_block = -1;                               // sph_test_stall_barrier
  int withhold_mma = 0;                               // sph_test_withhold_mma
  int chunk = 256;                                    // particles per solve chunk

  DevState* st = nullptr;
  StepAcc* acc = nullptr;
  SphStepStats* ring = nullptr;
  SphStepStats* last = nullptr;
  SphStepStats* h_last = nullptr;  // pinned
  DevState* h_state = nullptr;     // pinned

  cudaGraphExec_t gexec = nullptr;
  bool graph_dirty = true;
  bool graph_ok = true;
};

namespace {

int fail(SphCtx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(expr)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (expr);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? SPH_E_NOMEM : SPH_E_CUDA,                 \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                             \
  } while (0)

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <typename T>
cudaError_t dalloc(T*& p, size_t count) {
  dfree(p);
  if (count == 0) count = 1;
  return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
}

// Kernel tables exactly as sph_funcs.py:47-86 builds them: numpy linspace
// (i * step, last = h), FP64 evaluation with libm pow, then a float32 cast.
void build_tables(const SphParams& P, std::vector<float>& w, std::vector<float>& g) {
  const double h = P.h, sigma = P.sigma;
  const double h_inv = 1.0 / h, h_inv2 = 1.0 / (h * h);
  auto lin = [&](int S, int i) { return (i == S - 1) ? h : double(i) * (h / double(S - 1)); };
  w.assign(P.w_table_size, 0.f);
  g.assign(P.g_table_size, 0.f);
  for (int i = 0; i < P.w_table_size; ++i) {
    const double r = lin(P.w_table_size, i), q = r * h_inv;
    double v = 0.0;
    if (q <= 0.5) v = (6.0 * (std::pow(q, 3.0) - q * q) + 1.0) * sigma;
    else if (q < 1.0) v = 2.0 * std::pow(1.0 - q, 3.0) * sigma;
    w[i] = float(v);
  }
  for (int i = 0; i < P.g_table_size; ++i) {
    const double r = lin(P.g_table_size, i), q = r * h_inv;
    double v = 0.0;
    if (r > 1e-10) {
      if (q <= 0.5) v = (12.0 - 18.0 * q) * sigma * h_inv2;
      else if (q < 1.0) v = 6.0 * ((1.0 - q) * (1.0 - q)) * sigma * h_inv / r;
    }
    g[i] = float(v);
  }
}

// Smallest float r2 with sqrtf(r2) >= h: then sqrt_rn(r2) < h  <=>  r2 < limit.
float r2_limit_for(float h) {
  float t = h * h;
  while (std::sqrt(t) >= h) t = std::nextafter(t, 0.0f);
  while (std::sqrt(t) < h) t = std::nextafter(t, INFINITY);
  return t;
}

void make_consts(SphCtx* ctx) {
  const SphParams& P = ctx->P;
  Consts& c = ctx->c;
  c.h = float(P.h);
  c.r2_limit = r2_limit_for(c.h);
  const float h_inv = float(1.0 / P.h);
  c.sw = int(ctx->w_host.size());
  c.sg = int(ctx->g_host.size());
  c.w_scale = float(c.sw - 1) * h_inv;
  c.g_scale = float(c.sg - 1) * h_inv;
  c.rho0 = float(P.rho0);
  c.gravity = float(P.gravity);
  c.omega = float(P.omega);
  c.inv_small = float(P.inv_small);
  c.mu = float(P.vis_mu);
  c.m = float(P.fluid_mass);
  c.w0 = ctx->w_host.empty() ? 0.f : ctx->w_host[0];
  c.eta = float(P.eta);
  c.min_iter = P.min_iter;
  c.max_loop = P.max_loop;
  c.fixed_iters = P.fixed_iters;
  c.warm_start = P.warm_start;
  c.max_ff = ctx->K_ff;
  c.max_fb = ctx->K_fb;
  c.keep_fb = P.keep_fb_lists;
  const double sigma = P.sigma, h = P.h;
  c.gi0 = float(12.0 * sigma / (h * h));
  c.gi1 = float(18.0 * sigma / (h * h * h));
  c.go = float(6.0 * sigma / (h * h * h));
  c.h2q = float(h * h / 4.0);
}

int upload_tables(SphCtx* ctx) {
  CK(dalloc(ctx->d_w, ctx->w_host.size()));
  CK(dalloc(ctx->d_g, ctx->g_host.size()));
  CK(cudaMemcpy(ctx->d_w, ctx->w_host.data(), sizeof(float) * ctx->w_host.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_g, ctx->g_host.data(), sizeof(float) * ctx->g_host.size(), cudaMemcpyHostToDevice));
  make_consts(ctx);
  ctx->graph_dirty = true;
  return SPH_OK;
}

// One grid per scene over the union of its boundary and fluid bounding boxes
// (or its domain), padded by 2h, cell size 1.01 h (grown if a scene's cell count
// would exceed 2^26).  Scenes get consecutive global cell-id ranges.  Returns 1
// when any grid changed, 0 when none did, < 0 on error.
Grid fit_grid(const SphParams& P, const double* lo, const double* hi) {
  double cell = double(float(P.h)) * 1.01;
  const double pad = 2.0 * P.h;
  long long dims[3];
  for (;;) {
    long long tot = 1;
    for (int a = 0; a < 3; ++a) {
      const double w = a == 0 ? cell / sph::kXSplit : cell;
      dims[a] = std::max<long long>(1, (long long)std::ceil((hi[a] - lo[a] + 2 * pad) / w) + 1);
      tot *= dims[a];
    }
    if (tot <= (1ll << 26)) break;
    cell *= 1.25;
  }
  Grid g{};
  g.ox = float(lo[0] - pad);
  g.oy = float(lo[1] - pad);
  g.oz = float(lo[2] - pad);
  g.inv_cell = float(1.0 / cell);
  g.inv_cell_x = float(sph::kXSplit / cell);
  g.nx = int(dims[0]);
  g.ny = int(dims[1]);
  g.nz = int(dims[2]);
  g.ncells = int(dims[0] * dims[1] * dims[2]);
  return g;
}

int upload_scene_table(SphCtx* ctx) {
  const int S = ctx->S;
  // Scene-aligned chunks of at most ctx->chunk fluid slots, warp-aligned, and
  // as many of them as the persistent grid takes in whole rounds: the blocks
  // take chunks round-robin, so with ceil(n / chunk) full chunks the blocks
  // holding one chunk more set every pass's length.  Each scene's warps are
  // spread evenly over its share of rounds * grid chunks instead (chunks of
  // w or w + 1 warps), so every block ends a pass with the same work.
  std::vector<int2> chunks;
  std::vector<int> cscene;
  sph::SceneTable T{};
  T.nscenes = S;
  const int64_t wchunk = std::max<int64_t>(1, ctx->chunk / 32);
  std::vector<int64_t> ws(S), ms(S, 0);
  int64_t warps_tot = 0;
  for (int sc = 0; sc < S; ++sc) warps_tot += ws[sc] = (ctx->f_off[sc + 1] - ctx->f_off[sc] + 31) / 32;
  const int64_t grid = std::max(1, ctx->coop_grid);
  const int64_t target = grid * std::max<int64_t>(1, ((warps_tot + wchunk - 1) / wchunk + grid - 1) / grid);
  // each scene's share of the target chunk count (largest remainders round
  // up), at least enough for chunks of at most wchunk warps, at most one
  // chunk per warp
  std::vector<std::pair<int64_t, int>> rem;
  int64_t left = target;
  for (int sc = 0; sc < S; ++sc) {
    if (ws[sc] == 0) continue;
    ms[sc] = std::min(ws[sc], std::max(ws[sc] * target / warps_tot, (ws[sc] + wchunk - 1) / wchunk));
    left -= ms[sc];
    rem.emplace_back(ws[sc] * target % warps_tot, -sc);
  }
  std::sort(rem.rbegin(), rem.rend());
  for (const auto& r : rem) {
    if (left <= 0) break;
    const int sc = -r.second;
    if (ms[sc] < ws[sc]) {
      ++ms[sc];
      --left;
    }
  }
  for (int sc = 0; sc < S; ++sc) {
    T.chunk_off[sc] = int(chunks.size());
    const int64_t a0 = ctx->f_off[sc], a1 = ctx->f_off[sc + 1];
    const int64_t w = ws[sc], m = ms[sc];
    for (int64_t k = 0; k < m; ++k) {
      const int64_t b = a0 + 32 * (k * w / m), e = std::min(a1, a0 + 32 * ((k + 1) * w / m));
      chunks.push_back(make_int2(int(b), int(e)));
      cscene.push_back(sc);
    }
  }
  T.chunk_off[S] = int(chunks.size());
  for (int sc = 0; sc <= S; ++sc) {
    T.cell_base[sc] = ctx->cell_base[sc];
    T.fluid_off[sc] = int(ctx->f_off[sc]);
    T.bound_off[sc] = int(ctx->b_off[sc]);
  }
  for (int sc = 0; sc < S; ++sc) T.grid[sc] = ctx->grids[sc];
  if (!ctx->d_scenes) CK(cudaMalloc(&ctx->d_scenes, sizeof(sph::SceneTable)));
  CK(cudaMemcpy(ctx->d_scenes, &T, sizeof(T), cudaMemcpyHostToDevice));
  if (int(chunks.size()) != ctx->nchunks || !ctx->d_chunks) {
    ctx->nchunks = int(chunks.size());
    CK(dalloc(ctx->d_chunks, chunks.size()));
    CK(dalloc(ctx->d_chunk_scene, chunks.size()));
  }
  if (!chunks.empty()) {
    CK(cudaMemcpy(ctx->d_chunks, chunks.data(), sizeof(int2) * chunks.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_chunk_scene, cscene.data(), sizeof(int) * cscene.size(), cudaMemcpyHostToDevice));
  }
  ctx->graph_dirty = true;
  return SPH_OK;
}

int set_grid(SphCtx* ctx, const float* xf, int64_t n) {
  const SphParams& P = ctx->P;
  const int S = ctx->S;
  std::vector<Grid> grids(S);
  for (int sc = 0; sc < S; ++sc) {
    double lo[3], hi[3];
    const double* dom = ctx->domains.empty() ? nullptr : &ctx->domains[6 * size_t(sc)];
    bool have_domain = false;
    for (int a = 0; a < 3; ++a) {
      const double dmin = dom ? dom[a] : P.domain_min[a], dmax = dom ? dom[3 + a] : P.domain_max[a];
      have_domain = have_domain || (dmax > dmin);
    }
    if (have_domain) {
      for (int a = 0; a < 3; ++a) {
        lo[a] = dom ? dom[a] : P.domain_min[a];
        hi[a] = dom ? dom[3 + a] : P.domain_max[a];
      }
    } else {
      for (int a = 0; a < 3; ++a) {
        lo[a] = 1e300;
        hi[a] = -1e300;
      }
      auto fold = [&](const float* x, int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i)
          for (int a = 0; a < 3; ++a) {
            const double v = x[3 * i + a];
            if (std::isfinite(v)) {
              lo[a] = std::min(lo[a], v);
              hi[a] = std::max(hi[a], v);
            }
          }
      };
      if (ctx->nb) fold(ctx->bx_host.data(), ctx->b_off[sc], ctx->b_off[sc + 1]);
      if (xf && n == ctx->f_off[S]) fold(xf, ctx->f_off[sc], ctx->f_off[sc + 1]);
      for (int a = 0; a < 3; ++a)
        if (lo[a] > hi[a]) lo[a] = hi[a] = 0.0;
    }
    grids[sc] = fit_grid(P, lo, hi);
  }
  std::vector<int> base(S + 1, 0);
  long long total = 0;
  for (int sc = 0; sc < S; ++sc) {
    base[sc] = int(total);
    total += grids[sc].ncells;
  }
  if (total > (1ll << 28)) return fail(ctx, SPH_E_INVALID, "too many grid cells in total");
  base[S] = int(total);
  bool changed = !ctx->grid_valid || int(ctx->grids.size()) != S;
  if (!changed)
    for (int sc = 0; sc < S; ++sc) changed = changed || std::memcmp(&grids[sc], &ctx->grids[sc], sizeof(Grid)) != 0;
  ctx->grids = grids;
  ctx->cell_base = base;
  ctx->total_cells = int(total);
  ctx->grid_valid = true;
  if (ctx->total_cells > ctx->ncells_cap) {
    CK(dalloc(ctx->cell_count, ctx->total_cells));
    CK(dalloc(ctx->cell_start, ctx->total_cells + 1));
    CK(dalloc(ctx->bcell_start, ctx->total_cells + 1));
    CK(dalloc(ctx->scan_part, ctx->total_cells / 4096 + 2));
    ctx->scan_tiles_cap = ctx->total_cells / 4096 + 2;
    CK(dalloc(ctx->scan_status, size_t(ctx->scan_tiles_cap) + 1));
    CK(dalloc(ctx->coltop, ctx->total_cells));
    ctx->ncells_cap = ctx->total_cells;
  }
  int rc = upload_scene_table(ctx);
  if (rc) return rc;
  if (changed) ctx->graph_dirty = true;
  return changed ? 1 : 0;
}

// Sort the boundary into the grid and compute psi (compute_boundary_density).
// The boundary moves every step: requested, and some boundary velocity is nonzero.
bool boundary_moves(const SphCtx* ctx) { return ctx->P.move_boundary && ctx->b_moving && ctx->nb > 0; }

// Re-sort the (moved) boundary into the grid on the device, carrying psi in
// bpos.w: the per-step boundary_grid.build of a dynamic scene (IISPH.py:1415-1416).
int enqueue_boundary_resort(SphCtx* ctx) {
  const int64_t nb = ctx->nb;
  sph::SortArgs s{};
  s.n = int(nb);
  s.grid = ctx->grids[0];
  s.scenes = ctx->d_scenes;
  s.boundary = 1;
  s.pos = ctx->bpos;
  s.orig = ctx->borig;
  s.key = ctx->bkey;
  s.rank = ctx->brank;
  s.cell_count = ctx->cell_count;
  s.cell_start = ctx->bcell_start;
  s.scan_part = ctx->scan_part;
  s.sort_src = ctx->bsrc;
  s.sort_orig = ctx->borig_t;
  CK(sph::launch_sort(s, ctx->total_cells, ctx->stream));
  CK(sph::launch_gather(int(nb), ctx->bsrc, ctx->borig_t, ctx->bpos, ctx->bvel, nullptr, ctx->bpos_t, ctx->bvel_t,
                        ctx->borig, nullptr, ctx->stream));
  CK(cudaMemcpyAsync(ctx->bpos, ctx->bpos_t, sizeof(float4) * nb, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->bvel, ctx->bvel_t, sizeof(float4) * nb, cudaMemcpyDeviceToDevice, ctx->stream));
  return SPH_OK;
}

int sort_boundary(SphCtx* ctx) {
  const int64_t nb = ctx->nb;
  const int nc = ctx->total_cells;
  if (nb == 0) {
    CK(cudaMemsetAsync(ctx->bcell_start, 0, sizeof(int) * (nc + 1), ctx->stream));
    return SPH_OK;
  }
  std::vector<float4> hx(nb), hv(nb);
  std::vector<int> ho(nb);
  for (int64_t i = 0; i < nb; ++i) {
    hx[i] = make_float4(ctx->bx_host[3 * i], ctx->bx_host[3 * i + 1], ctx->bx_host[3 * i + 2], 0.f);
    hv[i] = make_float4(ctx->bv_host[3 * i], ctx->bv_host[3 * i + 1], ctx->bv_host[3 * i + 2], 0.f);
    ho[i] = int(i);
  }
  float4 *tx = nullptr, *tv = nullptr;
  int *to = nullptr, *key = nullptr, *rank = nullptr, *src = nullptr, *cnt = nullptr, *part = nullptr;
  CK(dalloc(tx, nb));
  CK(dalloc(tv, nb));
  CK(dalloc(to, nb));
  CK(dalloc(key, nb));
  CK(dalloc(rank, nb));
  CK(dalloc(src, nb));
  CK(dalloc(cnt, nc));
  CK(dalloc(part, nc / 4096 + 2));
  CK(cudaMemcpy(tx, hx.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(tv, hv.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(to, ho.data(), sizeof(int) * nb, cudaMemcpyHostToDevice));
  CK(dalloc(ctx->bpos, nb));
  CK(dalloc(ctx->borig, nb));
  if (ctx->b_moving) CK(dalloc(ctx->bvel, nb));
  else dfree(ctx->bvel);
  if (boundary_moves(ctx)) {
    CK(dalloc(ctx->bpos_t, nb));
    CK(dalloc(ctx->bvel_t, nb));
    CK(dalloc(ctx->borig_t, nb));
    CK(dalloc(ctx->bkey, nb));
    CK(dalloc(ctx->brank, nb));
    CK(dalloc(ctx->bsrc, nb));
  }
  sph::SortArgs s{};
  s.n = int(nb);
  s.grid = ctx->grids[0];
  s.scenes = ctx->d_scenes;
  s.boundary = 1;
  s.pos = tx;
  s.orig = to;
  s.key = key;
  s.rank = rank;
  s.cell_count = cnt;
  s.cell_start = ctx->bcell_start;
  s.scan_part = part;
  s.sort_src = src;
  s.sort_orig = ctx->borig;
  CK(sph::launch_sort(s, nc, ctx->stream));
  int* dummy = nullptr;
  CK(dalloc(dummy, nb));
  CK(sph::launch_gather(int(nb), src, ctx->borig, tx, tv, nullptr, ctx->bpos, ctx->bvel, dummy, nullptr,
                        ctx->stream));
  sph::PsiArgs pa{};
  pa.nb = int(nb);
  pa.grid = ctx->grids[0];
  pa.scenes = ctx->d_scenes;
  pa.c = ctx->c;
  pa.w_table = ctx->d_w;
  pa.bpos = ctx->bpos;
  pa.bcell_start = ctx->bcell_start;
  CK(sph::launch_psi(pa, 256, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (void* p : {(void*)tx, (void*)tv, (void*)to, (void*)key, (void*)rank, (void*)src, (void*)cnt, (void*)part,
                  (void*)dummy})
    cudaFree(p);
  ctx->graph_dirty = true;
  return SPH_OK;
}

int alloc_neighbors(SphCtx* ctx) {
  const int64_t tiles = (ctx->n_cap + 31) / 32;
  CK(dalloc(ctx->nbr_ff, tiles * 32 * int64_t(ctx->K_ff)));
  CK(dalloc(ctx->nbr_fb, tiles * 32 * int64_t(ctx->K_fb)));
  make_consts(ctx);
  ctx->graph_dirty = true;
  return SPH_OK;
}

// Whether the build's first phase reads its fluid candidates through the
// texture path as well as the second phase's neighbour gathers.
constexpr bool kBuildTexCandidates = false;

// 1-D texture objects over the work arrays of positions and velocities
// (float4 per slot): read-only gathers that then use the texture path.
int make_textures(SphCtx* ctx) {
  for (cudaTextureObject_t* t : {&ctx->pos_tex, &ctx->vel_tex, &ctx->yz_tex})
    if (*t) {
      cudaDestroyTextureObject(*t);
      *t = 0;
    }
  if (!ctx->jac_tex) return SPH_OK;
  for (int k = 0; k < 2; ++k) {
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = k == 0 ? static_cast<void*>(ctx->pos_w) : static_cast<void*>(ctx->vel_w);
    rd.res.linear.desc = cudaCreateChannelDesc<float4>();
    rd.res.linear.sizeInBytes = sizeof(float4) * size_t(ctx->n_cap);
    cudaTextureDesc td{};
    td.readMode = cudaReadModeElementType;
    CK(cudaCreateTextureObject(k == 0 ? &ctx->pos_tex : &ctx->vel_tex, &rd, &td, nullptr));
  }
  cudaResourceDesc rd{};
  rd.resType = cudaResourceTypeLinear;
  rd.res.linear.devPtr = ctx->yz_w;
  rd.res.linear.desc = cudaCreateChannelDesc<float2>();
  rd.res.linear.sizeInBytes = sizeof(float2) * size_t(ctx->n_cap);
  cudaTextureDesc td{};
  td.readMode = cudaReadModeElementType;
  CK(cudaCreateTextureObject(&ctx->yz_tex, &rd, &td, nullptr));
  return SPH_OK;
}

int alloc_fluid(SphCtx* ctx, int64_t n) {
  if (n <= ctx->n_cap && ctx->pos_s) return SPH_OK;
  const int64_t m = std::max<int64_t>(n, 1);
  ctx->n_cap = m;
  CK(dalloc(ctx->pos_s, m));
  CK(dalloc(ctx->vel_s, m));
  CK(dalloc(ctx->pos_w, m));
  CK(dalloc(ctx->vel_w, m));
  CK(dalloc(ctx->yz_w, m));
  {
    const int rc = make_textures(ctx);
    if (rc) return rc;
  }
  CK(dalloc(ctx->orig_s, m));
  CK(dalloc(ctx->orig_w, m));
  CK(dalloc(ctx->p_s, m));
  CK(dalloc(ctx->pprev_w, m));
  CK(dalloc(ctx->key, m));
  CK(dalloc(ctx->rank, m));
  CK(dalloc(ctx->sort_src, m));
  CK(dalloc(ctx->sort_orig, m));
  CK(dalloc(ctx->cnt_ff, m));
  CK(dalloc(ctx->cnt_fb, m));
  CK(dalloc(ctx->rho, m));
  CK(dalloc(ctx->bvec, m));
  CK(dalloc(ctx->dii_aii, m));
  CK(dalloc(ctx->vadv, m));
  CK(dalloc(ctx->a4, m));
  CK(dalloc(ctx->p_a, m));
  CK(dalloc(ctx->p_b, m));
  CK(dalloc(ctx->Ap, m));
  CK(dalloc(ctx->pmlp, m));
  CK(dalloc(ctx->stage, 7 * m));
  CK(dalloc(ctx->feat, size_t(sph::kFeatures) * m));
  CK(dalloc(ctx->p_start, m));
  CK(cudaMemset(ctx->rho, 0, sizeof(float) * m));
  CK(cudaMemset(ctx->bvec, 0, sizeof(float4) * m));
  CK(cudaMemset(ctx->dii_aii, 0, sizeof(float4) * m));
  CK(cudaMemset(ctx->vadv, 0, sizeof(float4) * m));
  CK(cudaMemset(ctx->a4, 0, sizeof(float4) * m));
  CK(cudaMemset(ctx->Ap, 0, sizeof(float) * m));
  CK(cudaMemset(ctx->pmlp, 0, sizeof(float) * m));
  CK(cudaMemset(ctx->cnt_ff, 0, sizeof(int) * m));
  CK(cudaMemset(ctx->cnt_fb, 0, sizeof(int) * m));
  return alloc_neighbors(ctx);
}

sph::SortArgs fluid_sort_args(SphCtx* ctx) {
  sph::SortArgs s{};
  s.n = int(ctx->n);
  s.grid = ctx->grids[0];
  s.scenes = ctx->d_scenes;
  s.pos = ctx->pos_s;
  s.orig = ctx->orig_s;
  s.key = ctx->key;
  s.rank = ctx->rank;
  s.cell_count = ctx->cell_count;
  s.cell_start = ctx->cell_start;
  s.scan_part = ctx->scan_part;
  s.scan_status = ctx->scan_status;
  s.scan_ticket = reinterpret_cast<unsigned int*>(ctx->scan_status + ctx->scan_tiles_cap);
  s.err = &ctx->acc->flags;
  s.sort_src = ctx->sort_src;
  s.sort_orig = ctx->sort_orig;
  return s;
}

sph::BuildArgs build_args(SphCtx* ctx) {
  sph::BuildArgs b{};
  b.n = int(ctx->n);
  b.nb = int(ctx->nb);
  b.grid = ctx->grids[0];
  b.scenes = ctx->d_scenes;
  b.c = ctx->c;
  b.w_table = ctx->d_w;
  b.g_table = ctx->d_g;
  b.spline = ctx->g_spline ? 1 : 0;
  b.pos = ctx->pos_w;
  b.vel = ctx->vel_w;
  b.pprev = ctx->pprev_w;
  b.pmlp = ctx->pmlp;
  b.cell_start = ctx->cell_start;
  b.bpos = ctx->bpos;
  b.bvel = ctx->bvel;
  b.bcell_start = ctx->bcell_start;
  b.st = ctx->st;
  b.acc = ctx->acc;
  b.nbr_ff = ctx->nbr_ff;
  b.cnt_ff = ctx->cnt_ff;
  b.nbr_fb = ctx->nbr_fb;
  b.cnt_fb = ctx->cnt_fb;
  b.rho = ctx->rho;
  b.bvec = ctx->bvec;
  b.dii_aii = ctx->dii_aii;
  b.vadv = ctx->vadv;
  b.p0 = ctx->p_a;
  b.pos_q = ctx->pos_w;
  b.feat = (ctx->record_feat || ctx->P.warm_start == SPH_WARM_MLP) ? ctx->feat : nullptr;
  b.feat_ld = ctx->n_cap;
  b.coltop = ctx->coltop;
  b.pos_tex = ctx->jac_tex ? (unsigned long long)ctx->pos_tex : 0ull;
  b.vel_tex = ctx->jac_tex ? (unsigned long long)ctx->vel_tex : 0ull;
  b.cand_tex = kBuildTexCandidates ? b.pos_tex : 0ull;
  b.yz_tex = ctx->jac_tex ? (unsigned long long)ctx->yz_tex : 0ull;
  return b;
}

// sort + gather + build: everything up to the pressure solve
int enqueue_front(SphCtx* ctx) {
  CK(cudaMemsetAsync(ctx->acc, 0, sizeof(StepAcc), ctx->stream));
  if (boundary_moves(ctx)) {
    const int rc = enqueue_boundary_resort(ctx);
    if (rc) return rc;
  }
  CK(sph::launch_sort(fluid_sort_args(ctx), ctx->total_cells, ctx->stream));
  CK(sph::launch_gather(int(ctx->n), ctx->sort_src, ctx->sort_orig, ctx->pos_s, ctx->vel_s, ctx->p_s, ctx->pos_w,
                        ctx->vel_w, ctx->orig_w, ctx->pprev_w, ctx->stream, ctx->jac_tex ? ctx->yz_w : nullptr));
  int block = ctx->P.block_size > 0 ? ctx->P.block_size : 128;
  const sph::BuildArgs b = build_args(ctx);
  if (b.feat) CK(sph::launch_column_top(b, ctx->coltop, ctx->total_cells, ctx->stream));
  if (ctx->P.vis_mu == 0.0) {
    CK(sph::launch_build(b, block, sph::kBuildFull, ctx->stream));
  } else {
    // viscosity: v_adv needs every density, rho_adv every v_adv (three passes)
    CK(sph::launch_build(b, block, sph::kBuildLists, ctx->stream));
    CK(sph::launch_visc(b, block, ctx->stream));
    CK(sph::launch_build(b, block, sph::kBuildAdvect, ctx->stream));
  }
  return SPH_OK;
}

// learned warm start: the network's prediction becomes the first iterate
int enqueue_warm(SphCtx* ctx) {
  if (ctx->P.warm_start == SPH_WARM_MLP) {
    sph::MlpInferArgs m{};
    m.n = ctx->n;
    m.w = ctx->mlp;
    m.feat = ctx->feat;
    m.feat_ld = ctx->n_cap;  // feature-major, as the build writes them
    m.rho = ctx->rho;
    m.p_unit = float(ctx->P.rho0 * ctx->P.gravity * ctx->P.h);
    m.p0 = ctx->p_a;
    m.pos_q = ctx->pos_w;
    m.flags = &ctx->acc->flags;
    m.withhold_mma = ctx->withhold_mma;
    if (ctx->P.warm_continue) {
      // a scene whose last solve stopped at the cap continues from that solve
      m.pprev = ctx->pprev_w;
      m.restart = ctx->st->capped;
      m.scenes = ctx->S > 1 ? ctx->d_scenes : nullptr;
    }
    CK(sph::launch_mlp_infer_tc(m, ctx->sm_count, ctx->stream));
  }
  // while features are recorded, keep the iterate the solve starts from
  // (sph_get_solve_start): p_1 from the build or the network, or 0.5 p_prev
  if (ctx->record_feat && ctx->n > 0)
    CK(cudaMemcpyAsync(ctx->p_start, ctx->p_a, sizeof(float) * size_t(ctx->n), cudaMemcpyDeviceToDevice,
                       ctx->stream));
  return SPH_OK;
}

// the persistent pressure solve with the fused kick, drift and CFL update
int enqueue_jacobi(SphCtx* ctx) {
  sph::JacobiArgs j{};
  j.n = int(ctx->n);
  j.nscenes = ctx->S;
  j.nchunks = ctx->nchunks;
  j.chunks = ctx->d_chunks;
  j.chunk_scene = ctx->d_chunk_scene;
  j.scenes = ctx->d_scenes;
  j.c = ctx->c;
  j.g_table = ctx->d_g;
  j.pos = ctx->pos_w;
  j.nbr_ff = ctx->nbr_ff;
  j.cnt_ff = ctx->cnt_ff;
  j.rho = ctx->rho;
  j.bvec = ctx->bvec;
  j.dii_aii = ctx->dii_aii;
  j.vadv = ctx->vadv;
  j.orig_w = ctx->orig_w;
  j.p_a = ctx->p_a;
  j.p_b = ctx->p_b;
  j.a4 = ctx->a4;
  j.Ap = ctx->Ap;
  j.partials = ctx->partials;
  j.st = ctx->st;
  j.acc = ctx->acc;
  j.ring = ctx->ring;
  j.last = ctx->last;
  j.bpos = ctx->bpos;
  j.bvel = ctx->bvel;
  j.nb = int(ctx->nb);
  j.move_boundary = boundary_moves(ctx) ? 1 : 0;
  j.pos_out = ctx->pos_s;
  j.vel_out = ctx->vel_s;
  j.orig_out = ctx->orig_s;
  j.p_out = ctx->p_s;
  // p_1 comes from the build (zero start: p_0 = 0 makes the first update local)
  // or from the network (its prediction is used as the first iterate); the
  // 0.5 p_prev start runs the reference's extra Ap_0 evaluation (pass 0).
  j.start_iter = (ctx->P.warm_start == SPH_WARM_HALF) ? 0 : 1;
  j.grad_spline = ctx->g_spline ? 1 : 0;
  j.yztex = (ctx->jac_tex && ctx->g_spline) ? (unsigned long long)ctx->yz_tex : 0ull;
  j.budget = (long long)ctx->P.timeout_ms * (long long)ctx->clock_khz;
  j.stall_block = ctx->stall_block;
  j.dt_max = ctx->P.dt_max;
  j.cfl_len = ctx->P.cfl_len;
  j.inv_small_d = ctx->P.inv_small;
  j.eta_d = ctx->P.eta;
  CK(sph::launch_jacobi(j, ctx->coop_grid, ctx->jac_block, ctx->jac_ppt, ctx->jac_unroll, ctx->jac_smem,
                        ctx->stream));
  return SPH_OK;
}

int enqueue_solve(SphCtx* ctx) {
  int rc = enqueue_warm(ctx);
  if (rc) return rc;
  return enqueue_jacobi(ctx);
}

int enqueue_step(SphCtx* ctx) {
  int rc = enqueue_front(ctx);
  if (rc) return rc;
  return enqueue_solve(ctx);
}

int ensure_ready(SphCtx* ctx) {
  if (ctx->P.warm_start == SPH_WARM_MLP && !ctx->have_mlp)
    return fail(ctx, SPH_E_INVALID, "SPH_WARM_MLP needs a network: call sph_set_mlp first");
  if (!ctx->grid_valid) {
    int rc = set_grid(ctx, nullptr, 0);
    if (rc < 0) return rc;
    rc = sort_boundary(ctx);
    if (rc) return rc;
  }
  if (!ctx->pos_s) {
    int rc = alloc_fluid(ctx, 1);
    if (rc) return rc;
  }
  const int64_t need = int64_t(ctx->coop_grid) * ctx->S;
  if (need > ctx->partials_cap) {
    CK(dalloc(ctx->partials, need));
    ctx->partials_cap = need;
    ctx->graph_dirty = true;
  }
  return SPH_OK;
}

// Capture the step into a CUDA graph (once per configuration).  Falls back to
// plain launches of the same kernels if this runtime cannot capture them.
int ensure_graph(SphCtx* ctx) {
  if (!ctx->P.use_graph || !ctx->graph_ok) return SPH_OK;
  if (!ctx->graph_dirty && ctx->gexec) return SPH_OK;
  if (ctx->gexec) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int erc = enqueue_step(ctx);
  cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
  if (erc == SPH_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&ctx->gexec, g, 0);
  if (g) cudaGraphDestroy(g);
  if (erc != SPH_OK || ce != cudaSuccess) {
    cudaGetLastError();
    ctx->graph_ok = false;
    ctx->gexec = nullptr;
    return SPH_OK;
  }
  ctx->graph_dirty = false;
  return SPH_OK;
}

int launch_step(SphCtx* ctx) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  rc = ensure_graph(ctx);
  if (rc) return rc;
  if (ctx->gexec) {
    CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    return SPH_OK;
  }
  return enqueue_step(ctx);
}

int flags_to_rc(SphCtx* ctx, int flags) {
  if (flags & SPH_F_TIMEOUT) return fail(ctx, SPH_E_TIMEOUT, "a grid-wide wait expired (SPH_F_TIMEOUT)");
  if (flags & (SPH_F_FF_OVERFLOW | SPH_F_FB_OVERFLOW))
    return fail(ctx, SPH_E_CAPACITY, "neighbour capacity exceeded");
  if (flags & SPH_F_NONFINITE) return fail(ctx, SPH_E_NONFINITE, "non-finite pressure or velocity");
  return SPH_OK;
}

// Grow the ELL capacities to the observed maxima (+25%) after an overflow.
int grow_capacity(SphCtx* ctx, int max_ff, int max_fb) {
  bool grow = false;
  if (max_ff > ctx->K_ff) {
    ctx->K_ff = ((max_ff + max_ff / 4 + 7) / 8) * 8;
    grow = true;
  }
  if (max_fb > ctx->K_fb) {
    ctx->K_fb = ((max_fb + max_fb / 4 + 7) / 8) * 8;
    grow = true;
  }
  if (!grow) return SPH_OK;
  return alloc_neighbors(ctx);
}

template <typename T>
void unsort(const std::vector<T>& sorted, const std::vector<int>& orig, T* out, int width) {
  for (size_t k = 0; k < orig.size(); ++k)
    for (int a = 0; a < width; ++a) out[size_t(orig[k]) * width + a] = sorted[k * width + a];
}

}  // namespace

extern "C" {

int sph_params_default(SphParams* p) {
  if (!p) return SPH_E_INVALID;
  std::memset(p, 0, sizeof(*p));
  const double d = 0.05;  // DIAMETER (main.py:26)
  p->spacing = d;
  p->h = 2 * d;
  p->rho0 = 1.0e3;
  p->gravity = 9.8;
  p->omega = 0.5;
  p->eta = 1.0e-3;
  p->inv_small = 1.0e-6;
  p->vis_mu = 0.0 * p->rho0;
  p->fluid_mass = p->rho0 * std::pow(d, 3.0);
  p->sigma = 8.0 / (M_PI * std::pow(p->h, 3.0));
  p->dt_max = 5e-2 * d;
  p->cfl_len = 0.4 * d;
  p->dt0 = p->dt_max;
  p->w_table_size = 8192;
  p->g_table_size = 65536;
  p->min_iter = 2;
  p->max_loop = 100;
  p->fixed_iters = -1;
  p->warm_start = SPH_WARM_ZERO;
  p->max_ff = 48;
  p->max_fb = 48;
  p->keep_fb_lists = 0;
  p->use_graph = 1;
  p->device = 0;
  p->block_size = 0;
  p->timeout_ms = 2000;
  return SPH_OK;
}

int sph_create(const SphParams* params, SphCtx** out) {
  if (!params || !out) return SPH_E_INVALID;
  *out = nullptr;
  const SphParams& P = *params;
  if (!(P.h > 0) || !(P.rho0 > 0) || P.w_table_size < 2 || P.g_table_size < 2 || P.max_ff < 1 || P.max_fb < 1 ||
      !(P.dt0 > 0) || !(P.dt_max > 0))
    return SPH_E_INVALID;
  if (!(P.vis_mu >= 0.0)) return SPH_E_INVALID;
  if (P.warm_continue != 0 && P.warm_continue != 1) return SPH_E_INVALID;
  SphCtx* ctx = new SphCtx();
  ctx->P = P;
  if (ctx->P.timeout_ms <= 0) ctx->P.timeout_ms = 2000;
  ctx->K_ff = P.max_ff;
  ctx->K_fb = P.max_fb;
  ctx->dev = P.device;
  auto bail = [&](int rc) {
    sph_destroy(ctx);
    return rc;
  };
  cudaError_t e = cudaSetDevice(ctx->dev);
  if (e != cudaSuccess) return bail(SPH_E_CUDA);
  if (cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&ctx->clock_khz, cudaDevAttrClockRate, ctx->dev) != cudaSuccess)
    return bail(SPH_E_CUDA);
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->dev);
  if (!coop) return bail(SPH_E_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(SPH_E_CUDA);
  build_tables(ctx->P, ctx->w_host, ctx->g_host);
  if (upload_tables(ctx)) return bail(SPH_E_CUDA);
  if (cudaMalloc(&ctx->st, sizeof(DevState)) != cudaSuccess || cudaMalloc(&ctx->acc, sizeof(StepAcc)) != cudaSuccess ||
      cudaMalloc(&ctx->ring, sizeof(SphStepStats) * sph::kStatsRing) != cudaSuccess ||
      cudaMalloc(&ctx->last, sizeof(SphStepStats)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_last, sizeof(SphStepStats)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_state, sizeof(DevState)) != cudaSuccess)
    return bail(SPH_E_NOMEM);
  cudaMemset(ctx->acc, 0, sizeof(StepAcc));
  cudaMemset(ctx->ring, 0, sizeof(SphStepStats) * sph::kStatsRing);
  cudaMemset(ctx->last, 0, sizeof(SphStepStats));
  DevState s{};
  for (int sc = 0; sc < sph::kMaxScenes; ++sc) {
    s.dt64[sc] = P.dt0;
    s.inv_dt64[sc] = 1.0 / P.dt0;
    s.dt[sc] = float(s.dt64[sc]);
    s.inv_dt[sc] = float(s.inv_dt64[sc]);
  }
  if (cudaMemcpy(ctx->st, &s, sizeof(s), cudaMemcpyHostToDevice) != cudaSuccess) return bail(SPH_E_CUDA);
  // 1024 threads: one block per SM (64 registers), 148 barrier arrivals per
  // pass instead of 592 with 256 threads (138.5 against 143.2 us per
  // iteration at 1M)
  ctx->jac_block = P.jacobi_block ? P.jacobi_block : 1024;
  ctx->jac_ppt = P.jacobi_ppt ? P.jacobi_ppt : 1;
  ctx->jac_unroll = P.jacobi_unroll ? P.jacobi_unroll : 4;
  if (!sph::jacobi_variant_ok(ctx->jac_block, ctx->jac_ppt, ctx->jac_unroll)) return bail(SPH_E_INVALID);
  ctx->chunk = ctx->jac_block * ctx->jac_ppt;
  ctx->jac_tex = (P.plain_loads == 0);
  if (sph::jacobi_config(ctx->jac_block, ctx->jac_ppt, ctx->jac_unroll, ctx->c.sg, ctx->g_spline, &ctx->blocks_per_sm,
                         &ctx->jac_smem, ctx->jac_tex) != cudaSuccess ||
      ctx->blocks_per_sm < 1)
    return bail(SPH_E_CUDA);
  ctx->coop_grid = ctx->blocks_per_sm * ctx->sm_count;
  *out = ctx;
  return SPH_OK;
}

void sph_destroy(SphCtx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->dev);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->pos_tex) cudaDestroyTextureObject(ctx->pos_tex);
  if (ctx->vel_tex) cudaDestroyTextureObject(ctx->vel_tex);
  if (ctx->yz_tex) cudaDestroyTextureObject(ctx->yz_tex);
  void* ptrs[] = {ctx->d_w, ctx->d_g, ctx->bpos, ctx->bvel, ctx->borig, ctx->bpos_t, ctx->bvel_t, ctx->borig_t,
                  ctx->bkey, ctx->brank, ctx->bsrc, ctx->bcell_start, ctx->pos_s, ctx->vel_s,
                  ctx->pos_w, ctx->vel_w, ctx->yz_w, ctx->orig_s, ctx->orig_w, ctx->p_s, ctx->pprev_w, ctx->key, ctx->rank,
                  ctx->sort_src, ctx->sort_orig, ctx->cell_count, ctx->cell_start, ctx->scan_part, ctx->scan_status, ctx->coltop, ctx->nbr_ff,
                  ctx->cnt_ff, ctx->nbr_fb, ctx->cnt_fb, ctx->rho, ctx->bvec, ctx->dii_aii, ctx->vadv, ctx->a4,
                  ctx->p_a, ctx->p_b, ctx->Ap, ctx->pmlp, ctx->feat, ctx->p_start, ctx->mlp, ctx->stage, ctx->partials, ctx->st, ctx->acc, ctx->ring,
                  ctx->d_scenes, ctx->d_chunks, ctx->d_chunk_scene,
                  ctx->last};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ctx->h_last) cudaFreeHost(ctx->h_last);
  if (ctx->h_state) cudaFreeHost(ctx->h_state);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* sph_last_error(const SphCtx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int sph_set_tables(SphCtx* ctx, const float* w, int32_t nw, const float* g, int32_t ng) {
  if (!ctx || !w || !g || nw < 2 || ng < 2) return fail(ctx, SPH_E_INVALID, "bad tables");
  CK(cudaSetDevice(ctx->dev));
  ctx->w_host.assign(w, w + nw);
  ctx->g_host.assign(g, g + ng);
  {
    // the closed-form gradient stands in for the table only if the table is
    // exactly the cubic spline's, sampled as this library samples it
    SphParams P2 = ctx->P;
    P2.w_table_size = nw;
    P2.g_table_size = ng;
    std::vector<float> w2, g2;
    build_tables(P2, w2, g2);
    ctx->g_spline = g2.size() == size_t(ng) && std::memcmp(g2.data(), g, sizeof(float) * size_t(ng)) == 0;
  }
  int rc = upload_tables(ctx);
  if (rc) return rc;
  int b = 0;
  CK(sph::jacobi_config(ctx->jac_block, ctx->jac_ppt, ctx->jac_unroll, ctx->c.sg, ctx->g_spline, &b,
                        &ctx->jac_smem, ctx->jac_tex));
  if (b < 1) return fail(ctx, SPH_E_CUDA, "jacobi kernel does not fit");
  if (b != ctx->blocks_per_sm) {
    ctx->blocks_per_sm = b;
    ctx->coop_grid = b * ctx->sm_count;
    if (ctx->grid_valid) {
      rc = upload_scene_table(ctx);  // chunks are cut for the grid size
      if (rc) return rc;
    }
  }
  if (ctx->nb) return sort_boundary(ctx);  // psi depends on W
  return SPH_OK;
}

int sph_set_boundary(SphCtx* ctx, const float* xb3, const float* vb3, int64_t nb) {
  if (!ctx || nb < 0 || (nb > 0 && !xb3)) return fail(ctx, SPH_E_INVALID, "bad boundary arguments");
  if (nb > INT32_MAX / 2) return fail(ctx, SPH_E_INVALID, "too many boundary particles");
  CK(cudaSetDevice(ctx->dev));
  if (ctx->S == 1) ctx->b_off = {0, nb};
  else if (nb != ctx->b_off[ctx->S])
    return fail(ctx, SPH_E_INVALID, "a batch takes all scenes' boundary particles, concatenated in scene order");
  ctx->nb = nb;
  ctx->bx_host.assign(xb3, xb3 + 3 * nb);
  ctx->bv_host.assign(3 * nb, 0.f);
  ctx->b_moving = false;
  if (vb3) {
    ctx->bv_host.assign(vb3, vb3 + 3 * nb);
    for (float v : ctx->bv_host) ctx->b_moving = ctx->b_moving || (v != 0.f);
  }
  // fluid positions, if any, take part in the grid extent
  std::vector<float> xf;
  if (ctx->n > 0) {
    std::vector<float4> h(ctx->n);
    CK(cudaMemcpy(h.data(), ctx->pos_s, sizeof(float4) * ctx->n, cudaMemcpyDeviceToHost));
    xf.resize(3 * ctx->n);
    for (int64_t i = 0; i < ctx->n; ++i) {
      xf[3 * i] = h[i].x;
      xf[3 * i + 1] = h[i].y;
      xf[3 * i + 2] = h[i].z;
    }
  }
  int rc = set_grid(ctx, xf.empty() ? nullptr : xf.data(), ctx->n);
  if (rc < 0) return rc;
  ctx->graph_dirty = true;
  return sort_boundary(ctx);
}

int sph_set_fluid(SphCtx* ctx, const float* x3, const float* v3, int64_t n) {
  if (!ctx || n < 0 || (n > 0 && !x3)) return fail(ctx, SPH_E_INVALID, "bad fluid arguments");
  if (n > INT32_MAX / 64) return fail(ctx, SPH_E_INVALID, "too many fluid particles");
  CK(cudaSetDevice(ctx->dev));
  if (ctx->S == 1) {
    if (ctx->f_off[1] != n) ctx->grid_valid = false;
    ctx->f_off = {0, n};
  } else if (n != ctx->f_off[ctx->S]) {
    return fail(ctx, SPH_E_INVALID, "a batch takes all scenes' fluid particles, concatenated in scene order");
  }
  int rc = alloc_fluid(ctx, n);
  if (rc) return rc;
  const bool resized = (n != ctx->n);
  if (resized) ctx->graph_dirty = true;
  ctx->n = n;
  if (!ctx->grid_valid || resized) {
    // the grid covers the particles given here; later states that leave it stay
    // correct (edge cells absorb them), so it is not refitted on every call
    rc = set_grid(ctx, x3, n);
    if (rc < 0) return rc;
    if (rc == 1) {
      rc = sort_boundary(ctx);
      if (rc) return rc;
    }
  }
  // a new state: no solve of it has stopped at the cap yet (warm_continue)
  CK(cudaMemsetAsync(ctx->st->capped, 0, sizeof(ctx->st->capped), ctx->stream));
  if (n > 0) {
    float* sx = ctx->stage;
    float* sv = ctx->stage + 3 * n;
    CK(cudaMemcpyAsync(sx, x3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
    if (v3) CK(cudaMemcpyAsync(sv, v3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(sph::launch_pack_fluid(int(n), 0, sx, v3 ? sv : nullptr, ctx->pos_s, ctx->vel_s, ctx->orig_s, ctx->p_s,
                              ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return SPH_OK;
}

int sph_update_fluid(SphCtx* ctx, const float* x3, const float* v3, const float* p, int64_t n) {
  if (!ctx || n != ctx->n || (n > 0 && (!x3 || !v3)))
    return fail(ctx, SPH_E_INVALID, "sph_update_fluid replaces x, v (and p) of the current particles (n = fluid count)");
  CK(cudaSetDevice(ctx->dev));
  if (n == 0) return SPH_OK;
  // the grid, dt, simulated time and the per-scene cap flags stay as they are
  float* sx = ctx->stage;
  float* sv = ctx->stage + 3 * n;
  float* sp = ctx->stage + 6 * n;
  CK(cudaMemcpyAsync(sx, x3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(sv, v3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
  if (p) CK(cudaMemcpyAsync(sp, p, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  // p = NULL keeps each particle's pressure on the device: into original
  // order before the pack below resets the state order
  else CK(sph::launch_unsort1(int(n), ctx->orig_s, ctx->p_s, sp, ctx->stream));
  CK(sph::launch_pack_fluid(int(n), 0, sx, sv, ctx->pos_s, ctx->vel_s, ctx->orig_s, ctx->p_s, ctx->stream, sp));
  CK(cudaStreamSynchronize(ctx->stream));
  return SPH_OK;
}

int sph_add_fluid(SphCtx* ctx, const float* x3, const float* v3, int64_t count) {
  if (!ctx || count < 0 || (count > 0 && !x3)) return fail(ctx, SPH_E_INVALID, "bad fluid arguments");
  if (ctx->S != 1) return fail(ctx, SPH_E_INVALID, "sph_add_fluid takes single-scene contexts");
  const int64_t n0 = ctx->n, n1 = n0 + count;
  if (n1 > INT32_MAX / 64) return fail(ctx, SPH_E_INVALID, "too many fluid particles");
  if (count == 0) return SPH_OK;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  if (n1 > ctx->n_cap || !ctx->pos_s) {
    // grow by half at least, carrying the state (x, v, original ids, p) over
    const int64_t cap = std::max<int64_t>(n1, ctx->n_cap + ctx->n_cap / 2);
    float4 *tx = nullptr, *tv = nullptr;
    int* to = nullptr;
    float* tp = nullptr;
    if (n0 > 0) {
      CK(dalloc(tx, n0));
      CK(dalloc(tv, n0));
      CK(dalloc(to, n0));
      CK(dalloc(tp, n0));
      CK(cudaMemcpyAsync(tx, ctx->pos_s, sizeof(float4) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(tv, ctx->vel_s, sizeof(float4) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(to, ctx->orig_s, sizeof(int) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(tp, ctx->p_s, sizeof(float) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
    }
    int rc = alloc_fluid(ctx, cap);
    if (rc) return rc;
    if (n0 > 0) {
      CK(cudaMemcpyAsync(ctx->pos_s, tx, sizeof(float4) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(ctx->vel_s, tv, sizeof(float4) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(ctx->orig_s, to, sizeof(int) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(ctx->p_s, tp, sizeof(float) * n0, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      dfree(tx);
      dfree(tv);
      dfree(to);
      dfree(tp);
    }
  }
  float* sx = ctx->stage;
  float* sv = ctx->stage + 3 * count;  // stage holds 7 floats per particle of capacity
  CK(cudaMemcpyAsync(sx, x3, sizeof(float) * 3 * count, cudaMemcpyHostToDevice, ctx->stream));
  if (v3) CK(cudaMemcpyAsync(sv, v3, sizeof(float) * 3 * count, cudaMemcpyHostToDevice, ctx->stream));
  CK(sph::launch_pack_fluid(int(count), int(n0), sx, v3 ? sv : nullptr, ctx->pos_s, ctx->vel_s, ctx->orig_s,
                            ctx->p_s, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->n = n1;
  ctx->f_off = {0, n1};
  ctx->graph_dirty = true;
  if (!ctx->grid_valid) {
    const int rc = set_grid(ctx, nullptr, 0);
    if (rc < 0) return rc;
    if (rc == 1) return sort_boundary(ctx);
    return SPH_OK;
  }
  return upload_scene_table(ctx);  // the solve's chunks cover the new count
}

int sph_set_pressure(SphCtx* ctx, const float* p, int64_t n) {
  if (!ctx || !p || n != ctx->n) return fail(ctx, SPH_E_INVALID, "pressure length must equal the fluid count");
  CK(cudaSetDevice(ctx->dev));
  if (n == 0) return SPH_OK;
  // one copy in original order, then a gather into the state's sorted order
  CK(cudaMemcpyAsync(ctx->stage, p, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  CK(sph::launch_sort1(int(n), ctx->orig_s, ctx->stage, ctx->p_s, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SPH_OK;
}

static int run_and_check(SphCtx* ctx, int nsteps, SphStepStats* out) {
  for (int attempt = 0; attempt < 4; ++attempt) {
    CK(cudaMemcpyAsync(ctx->h_state, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const long long start = ctx->h_state->step_index;
    int flags = 0, max_ff = 0, max_fb = 0;
    for (int s = 0; s < nsteps; ++s) {
      int rc = launch_step(ctx);
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(ctx->h_last, ctx->last, sizeof(SphStepStats), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_state, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    StepAcc acc{};
    CK(cudaMemcpyAsync(&acc, ctx->acc, sizeof(StepAcc), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    flags = acc.flags;
    max_ff = acc.max_ff;
    max_fb = acc.max_fb;
    const long long done = ctx->h_state->step_index - start;
    if (flags & (SPH_F_FF_OVERFLOW | SPH_F_FB_OVERFLOW)) {
      // the overflowing step left the state untouched: grow and redo the rest
      int rc = grow_capacity(ctx, max_ff, max_fb);
      if (rc) return rc;
      nsteps -= int(done);
      if (nsteps <= 0) break;
      continue;
    }
    if (out) *out = *ctx->h_last;
    return flags_to_rc(ctx, ctx->h_last->flags | (flags & (SPH_F_TIMEOUT | SPH_F_NONFINITE)));
  }
  if (out) *out = *ctx->h_last;
  return fail(ctx, SPH_E_CAPACITY, "neighbour capacity kept overflowing");
}

int sph_step(SphCtx* ctx, SphStepStats* out) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  return run_and_check(ctx, 1, out);
}

int sph_steps(SphCtx* ctx, int32_t nsteps, SphStepStats* last) {
  if (!ctx || nsteps < 0) return fail(ctx, SPH_E_INVALID, "bad step count");
  CK(cudaSetDevice(ctx->dev));
  if (nsteps == 0) return SPH_OK;
  return run_and_check(ctx, nsteps, last);
}

int sph_launch_steps(SphCtx* ctx, int32_t nsteps) {
  if (!ctx || nsteps < 0) return fail(ctx, SPH_E_INVALID, "bad step count");
  CK(cudaSetDevice(ctx->dev));
  for (int32_t i = 0; i < nsteps; ++i) {
    int rc = launch_step(ctx);
    if (rc) return rc;
  }
  return SPH_OK;
}

int sph_prepare(SphCtx* ctx) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  rc = ensure_graph(ctx);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return SPH_OK;
}

int sph_test_stall_barrier(SphCtx* ctx, int32_t block) {
  if (!ctx || block < -1) return fail(ctx, SPH_E_INVALID, "block must be -1 or a block index");
  if (ctx->stall_block != block) {
    ctx->stall_block = block;
    ctx->graph_dirty = true;
  }
  return SPH_OK;
}

int sph_test_withhold_mma(SphCtx* ctx, int32_t on) {
  if (!ctx || (on != 0 && on != 1)) return fail(ctx, SPH_E_INVALID, "on must be 0 or 1");
  if (ctx->withhold_mma != on) {
    ctx->withhold_mma = on;
    ctx->graph_dirty = true;
  }
  return SPH_OK;
}

int sph_launch_phase(SphCtx* ctx, int32_t phase) {
  if (!ctx || phase < 0 || phase > 3) return fail(ctx, SPH_E_INVALID, "phase must be 0, 1, 2 or 3");
  CK(cudaSetDevice(ctx->dev));
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  switch (phase) {
    case 0: return enqueue_front(ctx);
    case 1: return enqueue_solve(ctx);
    case 2: return enqueue_warm(ctx);
    default: return enqueue_jacobi(ctx);
  }
}

int sph_get_stats_history(SphCtx* ctx, SphStepStats* out, int32_t count) {
  if (!ctx || !out || count < 0 || count > sph::kStatsRing) return fail(ctx, SPH_E_INVALID, "bad count");
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  DevState s{};
  CK(cudaMemcpy(&s, ctx->st, sizeof(s), cudaMemcpyDeviceToHost));
  std::vector<SphStepStats> ring(sph::kStatsRing);
  CK(cudaMemcpy(ring.data(), ctx->ring, sizeof(SphStepStats) * sph::kStatsRing, cudaMemcpyDeviceToHost));
  const long long last = s.step_index;
  for (int i = 0; i < count; ++i) {
    const long long idx = last - count + i;  // 0-based step index
    if (idx < 0) std::memset(&out[i], 0, sizeof(SphStepStats));
    else out[i] = ring[idx % sph::kStatsRing];
  }
  return SPH_OK;
}

int sph_neighbor_search(SphCtx* ctx) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  rc = enqueue_front(ctx);
  if (rc) return rc;
  StepAcc acc{};
  CK(cudaMemcpyAsync(&acc, ctx->acc, sizeof(StepAcc), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (acc.flags & SPH_F_TIMEOUT) return fail(ctx, SPH_E_TIMEOUT, "the cell sort's scan waited too long (SPH_F_TIMEOUT)");
  if (acc.flags & (SPH_F_FF_OVERFLOW | SPH_F_FB_OVERFLOW)) {
    rc = grow_capacity(ctx, acc.max_ff, acc.max_fb);
    if (rc) return rc;
    rc = enqueue_front(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return SPH_OK;
}

int sph_get_fluid(SphCtx* ctx, float* x3, float* v3, float* p, float* rho, float* rho_adv) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  const int nn = int(ctx->n);
  if (nn == 0) return SPH_OK;
  const size_t n = size_t(nn);
  cudaStream_t s = ctx->stream;
  float* st = ctx->stage;  // x3 | v3 | p  (7 n floats); rho, rho_adv reuse after
  if (x3) CK(sph::launch_unsort4(nn, ctx->orig_s, ctx->pos_s, -1, st, s));
  if (v3) CK(sph::launch_unsort4(nn, ctx->orig_s, ctx->vel_s, -1, st + 3 * n, s));
  if (p) CK(sph::launch_unsort1(nn, ctx->orig_s, ctx->p_s, st + 6 * n, s));
  if (x3) CK(cudaMemcpyAsync(x3, st, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s));
  if (v3) CK(cudaMemcpyAsync(v3, st + 3 * n, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s));
  if (p) CK(cudaMemcpyAsync(p, st + 6 * n, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  if (rho || rho_adv) {
    CK(cudaStreamSynchronize(s));
    if (rho) {
      CK(sph::launch_unsort1(nn, ctx->orig_w, ctx->rho, st, s));
      CK(cudaMemcpyAsync(rho, st, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    }
    if (rho_adv) {
      CK(sph::launch_unsort4(nn, ctx->orig_w, ctx->bvec, 3, st + n, s));
      CK(cudaMemcpyAsync(rho_adv, st + n, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    }
  }
  CK(cudaStreamSynchronize(s));
  return SPH_OK;
}

int sph_get_terms(SphCtx* ctx, float* d_ii3, float* a_ii, float* s3, float* v_adv3, float* Ap) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t n = ctx->n;
  if (n == 0) return SPH_OK;
  std::vector<int> ow(n);
  CK(cudaMemcpy(ow.data(), ctx->orig_w, sizeof(int) * n, cudaMemcpyDeviceToHost));
  std::vector<float4> h(n);
  auto put3 = [&](float* out) {
    for (int64_t k = 0; k < n; ++k) {
      float* o = out + 3 * size_t(ow[k]);
      o[0] = h[k].x;
      o[1] = h[k].y;
      o[2] = h[k].z;
    }
  };
  if (d_ii3 || a_ii) {
    CK(cudaMemcpy(h.data(), ctx->dii_aii, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    if (d_ii3) put3(d_ii3);
    if (a_ii)
      for (int64_t k = 0; k < n; ++k) a_ii[ow[k]] = h[k].w;
  }
  if (s3) {
    // the solve keeps a = d_ii p + s of the final iterate (the kick's term);
    // s = a - d_ii p with the final p, which the step left in p_s in this order
    std::vector<float4> d(n);
    std::vector<float> p(n);
    CK(cudaMemcpy(h.data(), ctx->a4, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(d.data(), ctx->dii_aii, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(p.data(), ctx->p_s, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < n; ++k) {
      h[k].x = std::fma(-d[k].x, p[k], h[k].x);
      h[k].y = std::fma(-d[k].y, p[k], h[k].y);
      h[k].z = std::fma(-d[k].z, p[k], h[k].z);
    }
    put3(s3);
  }
  if (v_adv3) {
    CK(cudaMemcpy(h.data(), ctx->vadv, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    put3(v_adv3);
  }
  if (Ap) {
    std::vector<float> t(n);
    CK(cudaMemcpy(t.data(), ctx->Ap, sizeof(float) * n, cudaMemcpyDeviceToHost));
    unsort(t, ow, Ap, 1);
  }
  return SPH_OK;
}

int sph_get_boundary(SphCtx* ctx, float* xb3, float* psi) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t nb = ctx->nb;
  if (nb == 0) return SPH_OK;
  std::vector<float4> h(nb);
  std::vector<int> o(nb);
  CK(cudaMemcpy(h.data(), ctx->bpos, sizeof(float4) * nb, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(o.data(), ctx->borig, sizeof(int) * nb, cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < nb; ++k) {
    if (xb3) {
      xb3[3 * size_t(o[k])] = h[k].x;
      xb3[3 * size_t(o[k]) + 1] = h[k].y;
      xb3[3 * size_t(o[k]) + 2] = h[k].z;
    }
    if (psi) psi[o[k]] = h[k].w;
  }
  return SPH_OK;
}

int sph_get_neighbors(SphCtx* ctx, int64_t* ff_off, int32_t* ff_idx, int64_t ff_cap, int64_t* fb_off,
                      int32_t* fb_idx, int64_t fb_cap) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t n = ctx->n;
  std::vector<int> ow(n);
  if (n) CK(cudaMemcpy(ow.data(), ctx->orig_w, sizeof(int) * n, cudaMemcpyDeviceToHost));
  auto export_lists = [&](const int* d_nbr, const int* d_cnt, int K, const int* remap, int64_t* off, int32_t* idx,
                          int64_t cap) -> int {
    const int64_t tiles = (n + 31) / 32;
    std::vector<int> cnt(n), nbr(size_t(tiles) * 32 * K);
    if (n) {
      CK(cudaMemcpy(cnt.data(), d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(nbr.data(), d_nbr, sizeof(int) * nbr.size(), cudaMemcpyDeviceToHost));
    }
    std::vector<std::vector<int32_t>> lists(n);
    for (int64_t k = 0; k < n; ++k) {
      const int c = std::min(cnt[k], K);
      auto& L = lists[ow[k]];
      for (int t = 0; t < c; ++t) L.push_back(remap[nbr[(k >> 5) * 32 * K + t * 32 + (k & 31)]]);
      std::sort(L.begin(), L.end());
    }
    off[0] = 0;
    for (int64_t i = 0; i < n; ++i) off[i + 1] = off[i] + int64_t(lists[i].size());
    if (off[n] > cap) return fail(ctx, SPH_E_CAPACITY, "output capacity too small");
    for (int64_t i = 0; i < n; ++i) std::copy(lists[i].begin(), lists[i].end(), idx + off[i]);
    return SPH_OK;
  };
  if (ff_off) {
    int rc = export_lists(ctx->nbr_ff, ctx->cnt_ff, ctx->K_ff, ow.data(), ff_off, ff_idx, ff_cap);
    if (rc) return rc;
  }
  if (fb_off) {
    std::vector<int> bo(std::max<int64_t>(ctx->nb, 1));
    if (ctx->nb) CK(cudaMemcpy(bo.data(), ctx->borig, sizeof(int) * ctx->nb, cudaMemcpyDeviceToHost));
    int rc = export_lists(ctx->nbr_fb, ctx->cnt_fb, ctx->K_fb, bo.data(), fb_off, fb_idx, fb_cap);
    if (rc) return rc;
  }
  return SPH_OK;
}

int sph_create_batch(const SphParams* params, const SphSceneDesc* scenes, int32_t nscenes, SphCtx** out) {
  if (!params || !scenes || !out || nscenes < 1 || nscenes > sph::kMaxScenes) return SPH_E_INVALID;
  int64_t nf = 0, nbt = 0;
  for (int sc = 0; sc < nscenes; ++sc) {
    if (scenes[sc].n < 0 || scenes[sc].nb < 0 || (scenes[sc].n && !scenes[sc].x3) || (scenes[sc].nb && !scenes[sc].xb3))
      return SPH_E_INVALID;
    nf += scenes[sc].n;
    nbt += scenes[sc].nb;
  }
  if (nf > INT32_MAX / 64 || nbt > INT32_MAX / 2) return SPH_E_INVALID;
  int rc = sph_create(params, out);
  if (rc) return rc;
  SphCtx* ctx = *out;
  ctx->S = nscenes;
  ctx->f_off.assign(nscenes + 1, 0);
  ctx->b_off.assign(nscenes + 1, 0);
  ctx->domains.assign(6 * size_t(nscenes), 0.0);
  for (int sc = 0; sc < nscenes; ++sc) {
    ctx->f_off[sc + 1] = ctx->f_off[sc] + scenes[sc].n;
    ctx->b_off[sc + 1] = ctx->b_off[sc] + scenes[sc].nb;
    for (int a = 0; a < 3; ++a) {
      ctx->domains[6 * size_t(sc) + a] = scenes[sc].domain_min[a];
      ctx->domains[6 * size_t(sc) + 3 + a] = scenes[sc].domain_max[a];
    }
  }
  std::vector<float> x(3 * size_t(nf)), v(3 * size_t(nf), 0.f), xb(3 * size_t(nbt)), vb(3 * size_t(nbt), 0.f);
  bool any_vb = false;
  for (int sc = 0; sc < nscenes; ++sc) {
    const SphSceneDesc& d = scenes[sc];
    std::copy(d.x3, d.x3 + 3 * d.n, x.begin() + 3 * ctx->f_off[sc]);
    if (d.v3) std::copy(d.v3, d.v3 + 3 * d.n, v.begin() + 3 * ctx->f_off[sc]);
    if (d.nb) std::copy(d.xb3, d.xb3 + 3 * d.nb, xb.begin() + 3 * ctx->b_off[sc]);
    if (d.vb3) {
      std::copy(d.vb3, d.vb3 + 3 * d.nb, vb.begin() + 3 * ctx->b_off[sc]);
      any_vb = true;
    }
  }
  rc = sph_set_boundary(ctx, xb.data(), any_vb ? vb.data() : nullptr, nbt);
  if (!rc) rc = sph_set_fluid(ctx, x.data(), v.data(), nf);
  if (rc) {
    sph_destroy(ctx);
    *out = nullptr;
  }
  return rc;
}

int32_t sph_num_scenes(const SphCtx* ctx) { return ctx ? ctx->S : -1; }

int sph_get_scene_ranges(SphCtx* ctx, int64_t* fluid_off, int64_t* boundary_off) {
  if (!ctx) return SPH_E_INVALID;
  for (int sc = 0; sc <= ctx->S; ++sc) {
    if (fluid_off) fluid_off[sc] = ctx->f_off[sc];
    if (boundary_off) boundary_off[sc] = ctx->b_off[sc];
  }
  return SPH_OK;
}

int sph_get_scene_stats(SphCtx* ctx, int32_t* iterations, double* avg_err, double* v_max, double* dt,
                        double* sim_time) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  StepAcc acc{};
  DevState st{};
  CK(cudaMemcpy(&acc, ctx->acc, sizeof(acc), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&st, ctx->st, sizeof(st), cudaMemcpyDeviceToHost));
  for (int sc = 0; sc < ctx->S; ++sc) {
    if (iterations) iterations[sc] = acc.iterations[sc];
    if (avg_err) avg_err[sc] = acc.avg_err[sc];
    if (v_max) {
      float f;
      std::memcpy(&f, &acc.vmax_bits[sc], sizeof(f));
      v_max[sc] = f;
    }
    if (dt) dt[sc] = st.dt64[sc];
    if (sim_time) sim_time[sc] = st.sim_time[sc];
  }
  return SPH_OK;
}

int sph_set_mlp(SphCtx* ctx, const float* blob, int32_t n) {
  if (!ctx || !blob || n != SPH_MLP_BLOB) return fail(ctx, SPH_E_INVALID, "the network blob has SPH_MLP_BLOB floats");
  for (int c = 0; c < sph::kFeatures; ++c)
    if (!(blob[sph::kBlobSd + c] > 0)) return fail(ctx, SPH_E_INVALID, "input scales must be positive");
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  float* d_blob = nullptr;
  CK(dalloc(d_blob, SPH_MLP_BLOB));
  cudaError_t e = cudaMemcpy(d_blob, blob, sizeof(float) * SPH_MLP_BLOB, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !ctx->mlp) e = cudaMalloc(&ctx->mlp, sizeof(sph::MlpPacked));
  if (e == cudaSuccess) e = sph::launch_mlp_pack(d_blob, ctx->mlp, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_blob);
  if (e != cudaSuccess) return fail(ctx, SPH_E_CUDA, std::string("sph_set_mlp: ") + cudaGetErrorString(e));
  ctx->have_mlp = true;
  return SPH_OK;
}

int sph_set_record_features(SphCtx* ctx, int32_t on) {
  if (!ctx) return SPH_E_INVALID;
  if (ctx->record_feat != (on != 0)) ctx->graph_dirty = true;
  ctx->record_feat = (on != 0);
  return SPH_OK;
}

int sph_get_features(SphCtx* ctx, float* feat, float* target) {
  if (!ctx) return SPH_E_INVALID;
  if (!ctx->record_feat && ctx->P.warm_start != SPH_WARM_MLP)
    return fail(ctx, SPH_E_INVALID, "features are only computed with sph_set_record_features(ctx, 1)");
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t n = ctx->n;
  if (n == 0) return SPH_OK;
  std::vector<int> ow(n);
  CK(cudaMemcpy(ow.data(), ctx->orig_w, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (feat) {
    // device: feature-major over the sorted particles (leading dimension
    // n_cap); out: rows of kFeatures in original order
    std::vector<float> h(static_cast<size_t>(n));
    for (int c = 0; c < sph::kFeatures; ++c) {
      CK(cudaMemcpy(h.data(), ctx->feat + size_t(c) * size_t(ctx->n_cap), sizeof(float) * size_t(n),
                    cudaMemcpyDeviceToHost));
      for (int64_t k = 0; k < n; ++k) feat[size_t(ow[k]) * sph::kFeatures + c] = h[k];
    }
  }
  if (target) {
    // the last step's converged pressure, in the state order of that step (= orig_w)
    std::vector<float> h(n);
    CK(cudaMemcpy(h.data(), ctx->p_s, sizeof(float) * n, cudaMemcpyDeviceToHost));
    const double unit = 1.0 / (ctx->P.rho0 * ctx->P.gravity * ctx->P.h);
    for (int64_t k = 0; k < n; ++k) target[ow[k]] = float(std::asinh(double(h[k]) * unit));
  }
  return SPH_OK;
}

int sph_get_solve_start(SphCtx* ctx, float* p) {
  if (!ctx || !p) return SPH_E_INVALID;
  if (!ctx->record_feat)
    return fail(ctx, SPH_E_INVALID, "the solve's start is only kept with sph_set_record_features(ctx, 1)");
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  const int64_t n = ctx->n;
  if (n == 0) return SPH_OK;
  std::vector<int> ow(n);
  std::vector<float> h(n);
  CK(cudaMemcpy(ow.data(), ctx->orig_w, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.data(), ctx->p_start, sizeof(float) * n, cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < n; ++k) p[ow[k]] = h[k];
  return SPH_OK;
}

int sph_get_grid(SphCtx* ctx, int32_t scene, double* out) {
  if (!ctx || !out || scene < 0 || scene >= ctx->S) return fail(ctx, SPH_E_INVALID, "bad scene or output");
  if (!ctx->grid_valid) return fail(ctx, SPH_E_INVALID, "no grid yet: set the particles first");
  const Grid& g = ctx->grids[scene];
  const double v[9] = {g.ox, g.oy, g.oz, g.inv_cell, g.inv_cell_x, double(g.nx), double(g.ny), double(g.nz),
                       double(ctx->cell_base[scene])};
  for (int k = 0; k < 9; ++k) out[k] = v[k];
  return SPH_OK;
}

int sph_get_stats(SphCtx* ctx, SphStepStats* out) {
  if (!ctx || !out) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, ctx->last, sizeof(SphStepStats), cudaMemcpyDeviceToHost));
  return SPH_OK;
}

int sph_set_dt(SphCtx* ctx, double dt, double inv_dt) {
  if (!ctx || !(dt > 0) || !(inv_dt > 0)) return fail(ctx, SPH_E_INVALID, "dt must be positive");
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  DevState s{};
  CK(cudaMemcpy(&s, ctx->st, sizeof(s), cudaMemcpyDeviceToHost));
  for (int sc = 0; sc < ctx->S; ++sc) {
    s.dt64[sc] = dt;
    s.inv_dt64[sc] = inv_dt;
    s.dt[sc] = float(dt);
    s.inv_dt[sc] = float(inv_dt);
  }
  CK(cudaMemcpy(ctx->st, &s, sizeof(s), cudaMemcpyHostToDevice));
  return SPH_OK;
}

int sph_build_tables(const SphParams* params, float* w_table, float* g_table) {
  if (!params || !w_table || !g_table || params->w_table_size < 2 || params->g_table_size < 2) return SPH_E_INVALID;
  std::vector<float> w, g;
  build_tables(*params, w, g);
  std::copy(w.begin(), w.end(), w_table);
  std::copy(g.begin(), g.end(), g_table);
  return SPH_OK;
}

int sph_abi_info(int32_t* out, int32_t count) {
  const int32_t v[4] = {WPSPH_ABI_VERSION, int32_t(sizeof(SphParams)), int32_t(sizeof(SphStepStats)), 0};
  if (!out || count < 0) return SPH_E_INVALID;
  for (int32_t i = 0; i < count && i < 4; ++i) out[i] = v[i];
  return SPH_OK;
}

int64_t sph_num_fluid(const SphCtx* ctx) { return ctx ? ctx->n : -1; }
int64_t sph_num_boundary(const SphCtx* ctx) { return ctx ? ctx->nb : -1; }
void* sph_stream(SphCtx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int sph_synchronize(SphCtx* ctx) {
  if (!ctx) return SPH_E_INVALID;
  CK(cudaSetDevice(ctx->dev));
  CK(cudaStreamSynchronize(ctx->stream));
  return SPH_OK;
}

}  // extern "C"
