// CPU oracle of the reference IISPH time step (Mo-ZheHan/WarpSPH).
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / reference leg may load this library, and only as
// the checker.  The product (warpsph_b200) never calls it.
//
// Each function restates one reference kernel literally, expression for
// expression, so that the FP32 build (compiled with -ffp-contract=off, IEEE
// sqrt) mirrors the reference's float32 arithmetic and the FP64 build gives the
// "truth" the FP32 results are measured against.  Neighbour loops visit j in
// ascending original index; the reference visits them in hash-grid query order,
// so sums agree up to float32 reassociation.
//
// Parity pin: the golden vectors under tests/golden/ were produced by running
// the reference's own kernel code (IISPH.py, sph_funcs.py) under an emulated
// Warp runtime (tests/golden/warp_emu.py); tests/test_oracle_golden.py checks
// this oracle against them.  Warp itself (warp-lang 1.7.1) is not available
// here, so Warp's own codegen (FMA contraction, atomic order) is not pinned.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

typedef struct OracleParams {
  double h;          // SMOOTHING_LENGTH (main.py:57)
  double h_inv;      // 1/h (sph_funcs.py:8)
  double rho0;       // RHO_0 (main.py:30)
  double gravity;    // GRAVITY (main.py:25)
  double omega;      // OMEGA (main.py:27)
  double eta;        // ETA (main.py:28)
  double inv_small;  // INV_SMALL (main.py:29)
  double vis_mu;     // VIS_MU (main.py:61)
  double fluid_mass; // FLUID_MASS (main.py:59)
  double dt_max;     // TIME_STEP_MAX (main.py:58)
  double cfl_len;    // 0.4 * DIAMETER (IISPH.py:1369)
  int w_size;        // W_SIZE (sph_funcs.py:43)
  int g_size;        // GRAD_W_SIZE (sph_funcs.py:44)
  int max_loop;      // loop index after which the solve stops: 100 (IISPH.py:1202)
  int min_loop;      // minimum iterations: 2 (IISPH.py:1201)
  int fixed_iters;   // >= 0: run exactly this many iterations (parity tests)
  int err_fp32_seq;  // 1: accumulate the density error in float32, index order
  int nthreads;      // OpenMP threads (0 = runtime default)
  int warm_start;    // 0: p <- 0 (IISPH.py:173); 1: p <- 0.5 p (IISPH.py:174); 2: keep p
} OracleParams;

typedef struct OracleStep {
  int64_t n, nb;
  void* x;            // n*3, in/out
  void* v;            // n*3, in/out
  void* p;            // n, in (warm start) / out
  const void* bx;     // nb*3
  const void* bv;     // nb*3
  const void* psi;    // nb
  const void* w_table;
  const void* g_table;
  double dt, inv_dt;  // this step's dt and 1/dt as the reference passes them
  // optional per-particle outputs (NULL to skip)
  void* rho;
  void* v_adv;
  void* rho_adv;
  void* d_ii;
  void* a_ii;
  void* s;
  void* Ap;
  // optional neighbour export, CSR over original ids (NULL to skip)
  int64_t* ff_off;
  int32_t* ff_idx;
  int64_t ff_cap;
  int64_t* fb_off;
  int32_t* fb_idx;
  int64_t fb_cap;
  // outputs
  int iterations;
  int status;
  double avg_err;
  double v_max;
  double dt_next, inv_dt_next;
  int64_t n_ff_pairs, n_fb_pairs;
} OracleStep;

}  // extern "C"

namespace {

template <typename R>
struct V3 {
  R x, y, z;
};
template <typename R>
inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R>
inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R>
inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <typename R>
inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R>
inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename R>
inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <typename R>
inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R>
inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }

template <typename R>
struct Ctx {
  const OracleParams* P;
  R h, h_inv, rho0, g, omega, inv_small, mu, m;
  const R* W;
  const R* G;
  int SW, SG;

  // sph_funcs.py:92-102
  R spline_W(R r) const {
    if (r >= h) return R(0);
    R idx_float = r * (R(SW - 1) * h_inv);
    int idx_low = std::min(int(idx_float), SW - 2);
    R alpha = idx_float - R(idx_low);
    return (R(1) - alpha) * W[idx_low] + alpha * W[idx_low + 1];
  }
  // sph_funcs.py:105-118
  V3<R> grad_W(V3<R> r) const {
    R r_len = length(r);
    if (r_len >= h || r_len < R(1e-10)) return {R(0), R(0), R(0)};
    R idx_float = r_len * (R(SG - 1) * h_inv);
    int idx_low = std::min(int(idx_float), SG - 2);
    R alpha = idx_float - R(idx_low);
    R scalar = (R(1) - alpha) * G[idx_low] + alpha * G[idx_low + 1];
    return scalar * r;
  }
};

// Per-pair storage (hundreds of MB at 1M particles) left uninitialised: every
// element is written by a parallel loop before it is read, so its pages are
// first touched by the threads that use them instead of being zeroed serially.
template <typename T>
struct Uninit {
  std::unique_ptr<T[]> p;
  explicit Uninit(size_t n) : p(new T[n > 0 ? n : 1]) {}
  T& operator[](size_t i) { return p[i]; }
  const T& operator[](size_t i) const { return p[i]; }
};

// Exact-distance neighbour sets on a uniform grid of cell size slightly above h.
// N(i) = { j : |x_i - x_j| < h } (minus j = i when same == true), j ascending.
// This restates the filtered hash_grid_query loops of IISPH.py:70-72 (ff),
// IISPH.py:127-129 (fb) and IISPH.py:42-44 (boundary-boundary).
template <typename R>
void neighbours(const R* xq, int64_t nq, const R* xs, int64_t ns, R h, bool same,
                std::vector<int64_t>& off, std::vector<int32_t>& idx, int nthreads) {
  off.assign(nq + 1, 0);
  idx.clear();
  if (nq == 0) return;
  if (ns == 0) return;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < ns; ++i)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], double(xs[3 * i + a]));
      hi[a] = std::max(hi[a], double(xs[3 * i + a]));
    }
  double cell = double(h) * 1.01;
  int64_t dim[3];
  for (int a = 0; a < 3; ++a) dim[a] = std::max<int64_t>(1, int64_t((hi[a] - lo[a]) / cell) + 1);
  auto coord = [&](double v, int a) {
    int64_t c = int64_t(std::floor((v - lo[a]) / cell));
    return std::min<int64_t>(std::max<int64_t>(c, 0), dim[a] - 1);
  };
  int64_t ncell = dim[0] * dim[1] * dim[2];
  std::vector<int64_t> start(ncell + 1, 0);
  std::vector<int64_t> key(ns);
  for (int64_t i = 0; i < ns; ++i) {
    key[i] = (coord(xs[3 * i + 2], 2) * dim[1] + coord(xs[3 * i + 1], 1)) * dim[0] + coord(xs[3 * i], 0);
    start[key[i] + 1]++;
  }
  for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
  std::vector<int32_t> sorted(ns);
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t i = 0; i < ns; ++i) sorted[fill[key[i]]++] = int32_t(i);
  }
  // Two passes over the same candidates, count then fill, into one flat array
  // (no per-particle allocations); each segment is then sorted ascending.
  auto visit = [&](int64_t i, auto&& hit) {
    V3<R> xi{xq[3 * i], xq[3 * i + 1], xq[3 * i + 2]};
    int64_t c[3] = {coord(xi.x, 0), coord(xi.y, 1), coord(xi.z, 2)};
    for (int64_t cz = std::max<int64_t>(c[2] - 1, 0); cz <= std::min(c[2] + 1, dim[2] - 1); ++cz)
      for (int64_t cy = std::max<int64_t>(c[1] - 1, 0); cy <= std::min(c[1] + 1, dim[1] - 1); ++cy)
        for (int64_t cx = std::max<int64_t>(c[0] - 1, 0); cx <= std::min(c[0] + 1, dim[0] - 1); ++cx) {
          int64_t k = (cz * dim[1] + cy) * dim[0] + cx;
          for (int64_t t = start[k]; t < start[k + 1]; ++t) {
            int32_t j = sorted[t];
            V3<R> xj{xs[3 * j], xs[3 * j + 1], xs[3 * j + 2]};
            R distance = length(xi - xj);
            if (distance < h && !(same && j == i)) hit(j);
          }
        }
  };
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
  for (int64_t i = 0; i < nq; ++i) {
    int64_t n = 0;
    visit(i, [&](int32_t) { ++n; });
    off[i + 1] = n;
  }
  for (int64_t i = 0; i < nq; ++i) off[i + 1] += off[i];
  idx.resize(off[nq]);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
  for (int64_t i = 0; i < nq; ++i) {
    int64_t w = off[i];
    visit(i, [&](int32_t j) { idx[w++] = j; });
    std::sort(idx.begin() + off[i], idx.begin() + off[i + 1]);
  }
}

template <typename R>
Ctx<R> make_ctx(const OracleParams* P, const void* w, const void* g) {
  Ctx<R> c;
  c.P = P;
  c.h = R(P->h);
  c.h_inv = R(P->h_inv);
  c.rho0 = R(P->rho0);
  c.g = R(P->gravity);
  c.omega = R(P->omega);
  c.inv_small = R(P->inv_small);
  c.mu = R(P->vis_mu);
  c.m = R(P->fluid_mass);
  c.W = static_cast<const R*>(w);
  c.G = static_cast<const R*>(g);
  c.SW = P->w_size;
  c.SG = P->g_size;
  return c;
}

// IISPH.py:23-47 compute_boundary_density
template <typename R>
int psi(const OracleParams* P, int64_t nb, const R* bx, const R* w_table, R* out) {
  Ctx<R> C = make_ctx<R>(P, w_table, w_table);
  std::vector<int64_t> off;
  std::vector<int32_t> idx;
  int nt = P->nthreads > 0 ? P->nthreads : 1;
  neighbours<R>(bx, nb, bx, nb, C.h, true, off, idx, nt);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < nb; ++i) {
    V3<R> x{bx[3 * i], bx[3 * i + 1], bx[3 * i + 2]};
    R rho = C.spline_W(R(0));
    for (int64_t t = off[i]; t < off[i + 1]; ++t) {
      int32_t j = idx[t];
      R distance = length(x - V3<R>{bx[3 * j], bx[3 * j + 1], bx[3 * j + 2]});
      rho += C.spline_W(distance);
    }
    out[i] = C.rho0 / rho;
  }
  return 0;
}

template <typename R>
inline V3<R> ld3(const R* a, int64_t i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
template <typename R>
inline void st3(R* a, int64_t i, V3<R> v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }

template <typename R>
int step(const OracleParams* P, OracleStep* S) {
  const int64_t n = S->n, nb = S->nb;
  const int nt = P->nthreads > 0 ? P->nthreads : 1;
  Ctx<R> C = make_ctx<R>(P, S->w_table, S->g_table);
  R* x = static_cast<R*>(S->x);
  R* v = static_cast<R*>(S->v);
  R* p = static_cast<R*>(S->p);
  const R* bx = static_cast<const R*>(S->bx);
  const R* bv = static_cast<const R*>(S->bv);
  const R* phi = static_cast<const R*>(S->psi);
  const R dt = R(S->dt);
  const R inv_dt = R(S->inv_dt);
  const R m = C.m;

  // neighbor_search (IISPH.py:1408-1482): ff without self, fb with all
  std::vector<int64_t> ffo, fbo;
  std::vector<int32_t> ffi, fbi;
  neighbours<R>(x, n, x, n, C.h, true, ffo, ffi, nt);
  neighbours<R>(x, n, bx, nb, C.h, false, fbo, fbi, nt);
  const int64_t Pff = n ? ffo[n] : 0, Pfb = n ? fbo[n] : 0;
  S->n_ff_pairs = Pff;
  S->n_fb_pairs = Pfb;
  // stored distances (IISPH.py:100-103, 159-162)
  Uninit<R> ffd(Pff), fbd(Pfb);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    V3<R> xi = ld3(x, i);
    for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) ffd[t] = length(xi - ld3(x, ffi[t]));
    for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) fbd[t] = length(xi - ld3(bx, fbi[t]));
  }

  std::vector<R> rho(n), rho_adv(n), a_ii(n), Ap(n);
  std::vector<V3<R>> v_adv(n), d_ii(n), s(n);
  Uninit<V3<R>> d_ij(Pff), d_ji(Pff);

  // init_pressure (IISPH.py:166-174)
  if (P->warm_start == 0) std::fill(p, p + n, R(0));
  else if (P->warm_start == 1)
    for (int64_t i = 0; i < n; ++i) p[i] = p[i] / R(2);

  // compute_density (IISPH.py:177-214)
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    R t1 = 0, t2 = 0;
    for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) t1 += C.spline_W(ffd[t]);
    for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) t2 += C.spline_W(fbd[t]) * phi[fbi[t]];
    rho[i] = t1 * m + t2 + C.spline_W(R(0)) * m;
  }

  // predict_v_adv (IISPH.py:217-278)
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    V3<R> t1{0, 0, 0}, t2{0, 0, 0};
    V3<R> xi = ld3(x, i), vi = ld3(v, i);
    for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) {
      int32_t j = ffi[t];
      V3<R> x_ij = ld3(x, j) - xi;
      R d2 = ffd[t] * ffd[t];
      t1 = t1 - C.grad_W(x_ij) * dot(vi - ld3(v, j), x_ij) / rho[j] / d2;
    }
    for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) {
      int32_t b = fbi[t];
      V3<R> x_ib = ld3(bx, b) - xi;
      R d2 = fbd[t] * fbd[t];
      t2 = t2 - C.grad_W(x_ib) * phi[b] * dot(vi, x_ib) / d2;
    }
    V3<R> lap = R(10) * (t1 * m + t2 / C.rho0);
    V3<R> grav{R(0), -C.g, R(0)};
    v_adv[i] = ld3(v, i) + (lap * C.mu / rho[i] + grav) * dt;
  }

  // predict_rho_adv (IISPH.py:281-329)
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    R t1 = 0, t2 = 0;
    V3<R> xi = ld3(x, i), va = v_adv[i];
    for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) {
      int32_t j = ffi[t];
      t1 += dot(va - v_adv[j], C.grad_W(ld3(x, j) - xi));
    }
    for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) {
      int32_t b = fbi[t];
      t2 += dot(va - ld3(bv, b), C.grad_W(ld3(bx, b) - xi)) * phi[b];
    }
    rho_adv[i] = rho[i] + (t1 * m + t2) * dt;
  }

  // compute_term_d (IISPH.py:332-382)
  const R dt2 = dt * dt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    V3<R> t1{0, 0, 0}, t2{0, 0, 0};
    R t3 = m * dt2;
    V3<R> xi = ld3(x, i);
    R r = rho[i];
    for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) {
      int32_t j = ffi[t];
      V3<R> gw = C.grad_W(ld3(x, j) - xi);
      t1 = t1 - gw;
      d_ij[t] = -gw * t3 / (rho[j] * rho[j]);
      d_ji[t] = gw * t3 / (r * r);
    }
    for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) {
      int32_t b = fbi[t];
      t2 = t2 - C.grad_W(ld3(bx, b) - xi) * phi[b];
    }
    d_ii[i] = (t1 * m + t2) * dt2 / (r * r);
  }

  // compute_term_a (IISPH.py:385-428)
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    R t1 = 0, t2 = 0;
    V3<R> xi = ld3(x, i), dii = d_ii[i];
    for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t)
      t1 += dot(dii - d_ji[t], C.grad_W(ld3(x, ffi[t]) - xi));
    for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) {
      int32_t b = fbi[t];
      t2 += dot(dii, C.grad_W(ld3(bx, b) - xi)) * phi[b];
    }
    a_ii[i] = t1 * m + t2;
  }

  // compute_term_Ap_1 (IISPH.py:431-466)
  auto ap1 = [&]() {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
      R t1 = 0;
      V3<R> xi = ld3(x, i);
      V3<R> si{0, 0, 0};
      for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) {
        int32_t j = ffi[t];
        V3<R> term = d_ji[t] * p[i] - d_ii[j] * p[j];
        t1 += dot(term, C.grad_W(ld3(x, j) - xi));
        si = si + d_ij[t] * p[j];
      }
      s[i] = si;
      Ap[i] = t1 * m;
    }
  };
  // compute_term_Ap_2 (IISPH.py:469-518)
  auto ap2 = [&]() {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
      R t1 = 0, t2 = 0;
      V3<R> xi = ld3(x, i), si = s[i];
      for (int64_t t = ffo[i]; t < ffo[i + 1]; ++t) {
        int32_t j = ffi[t];
        t1 += dot(si - s[j], C.grad_W(ld3(x, j) - xi));
      }
      for (int64_t t = fbo[i]; t < fbo[i + 1]; ++t) {
        int32_t b = fbi[t];
        t2 += dot(si, C.grad_W(ld3(bx, b) - xi)) * phi[b];
      }
      Ap[i] = Ap[i] + (t1 * m + t2 + a_ii[i] * p[i]);
    }
  };
  // update_p (IISPH.py:521-539)
  auto update_p = [&]() {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
      R a = a_ii[i];
      if (a > -C.inv_small && a < C.inv_small) a = (a < R(0) ? R(-1) : R(1)) * C.inv_small;
      p[i] = p[i] + (C.rho0 - rho_adv[i] - Ap[i]) * C.omega / a;
      p[i] = std::max(p[i], R(0));
    }
  };
  // update_rho_error (IISPH.py:542-568) + average_rho_error (IISPH.py:1489-1494)
  auto rho_error = [&]() -> double {
    int64_t cnt = 0;
    double sum = 0.0;
    if (P->err_fp32_seq) {
      R acc = 0;
      for (int64_t i = 0; i < n; ++i) {
        R upd = rho_adv[i] + Ap[i];
        if (upd > C.rho0) {
          acc = acc + std::fabs(upd / C.rho0 - R(1));
          cnt++;
        }
      }
      sum = double(acc);
    } else {
#pragma omp parallel for schedule(static) num_threads(nt) reduction(+ : sum, cnt)
      for (int64_t i = 0; i < n; ++i) {
        R upd = rho_adv[i] + Ap[i];
        if (upd > C.rho0) {
          sum += double(std::fabs(upd / C.rho0 - R(1)));
          cnt++;
        }
      }
    }
    if (cnt == 0) return 0.0;
    return sum / double(cnt);
  };

  // pressure solve (IISPH.py:1155-1296)
  ap1();
  ap2();
  int loop = 0;
  double avg = 0.0;
  if (P->fixed_iters >= 0) {
    for (loop = 0; loop < P->fixed_iters; ++loop) {
      update_p();
      ap1();
      ap2();
      avg = rho_error();
    }
  } else {
    while (loop < P->min_loop || avg > P->eta) {
      if (loop > P->max_loop) break;
      update_p();
      ap1();
      ap2();
      avg = rho_error();
      loop++;
    }
  }
  S->iterations = loop;
  S->avg_err = avg;

  // kick (IISPH.py:674-688), drift (IISPH.py:691-699)
  R vmax = 0;
  for (int64_t i = 0; i < n; ++i) {
    V3<R> dv = inv_dt * (d_ii[i] * p[i] + s[i]);
    V3<R> vn = v_adv[i] + dv;
    st3(v, i, vn);
    vmax = std::max(vmax, length(vn));
  }
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) st3(x, i, ld3(x, i) + ld3(v, i) * dt);
  S->v_max = double(vmax);

  // CFL (IISPH.py:1367-1371).  With numpy >= 2 the float32 v_max makes
  // 0.4*DIAMETER / v_max a float32 division; wp.min then keeps whichever is smaller.
  if (sizeof(R) == 4 && double(vmax) >= double(float(P->inv_small))) {
    float q = float(P->cfl_len) / float(vmax);
    if (q < float(P->dt_max)) {
      S->dt_next = double(q);
      S->inv_dt_next = double(1.0f / q);
    } else {
      S->dt_next = P->dt_max;
      S->inv_dt_next = 1.0 / P->dt_max;
    }
  } else {
    double q = P->cfl_len / std::max(double(vmax), P->inv_small);
    S->dt_next = std::min(q, P->dt_max);
    S->inv_dt_next = 1.0 / S->dt_next;
  }

  // optional exports
  auto put1 = [&](void* dst, const std::vector<R>& a) {
    if (dst) std::memcpy(dst, a.data(), sizeof(R) * n);
  };
  auto put3 = [&](void* dst, const std::vector<V3<R>>& a) {
    if (dst) std::memcpy(dst, a.data(), sizeof(R) * 3 * n);
  };
  put1(S->rho, rho);
  put1(S->rho_adv, rho_adv);
  put1(S->a_ii, a_ii);
  put1(S->Ap, Ap);
  put3(S->v_adv, v_adv);
  put3(S->d_ii, d_ii);
  put3(S->s, s);
  int status = 0;
  if (S->ff_off) {
    std::memcpy(S->ff_off, ffo.data(), sizeof(int64_t) * (n + 1));
    if (Pff <= S->ff_cap) std::memcpy(S->ff_idx, ffi.data(), sizeof(int32_t) * Pff);
    else status = -2;
  }
  if (S->fb_off) {
    std::memcpy(S->fb_off, fbo.data(), sizeof(int64_t) * (n + 1));
    if (Pfb <= S->fb_cap) std::memcpy(S->fb_idx, fbi.data(), sizeof(int32_t) * Pfb);
    else status = -2;
  }
  S->status = status;
  return status;
}

}  // namespace

extern "C" {

int oracle_psi_f32(const OracleParams* P, int64_t nb, const float* bx, const float* w, float* out) {
  return psi<float>(P, nb, bx, w, out);
}
int oracle_psi_f64(const OracleParams* P, int64_t nb, const double* bx, const double* w, double* out) {
  return psi<double>(P, nb, bx, w, out);
}
int oracle_step_f32(const OracleParams* P, OracleStep* S) { return step<float>(P, S); }
int oracle_step_f64(const OracleParams* P, OracleStep* S) { return step<double>(P, S); }

// Neighbour sets only (bit-exact reference for the GPU neighbour build).
int oracle_neighbors_f32(const OracleParams* P, int64_t nq, const float* xq, int64_t ns, const float* xs,
                         int same, int64_t* off, int32_t* idx, int64_t cap) {
  std::vector<int64_t> o;
  std::vector<int32_t> id;
  neighbours<float>(xq, nq, xs, ns, float(P->h), same != 0, o, id, P->nthreads > 0 ? P->nthreads : 1);
  std::memcpy(off, o.data(), sizeof(int64_t) * (nq + 1));
  if (nq && o[nq] > cap) return -2;
  if (nq) std::memcpy(idx, id.data(), sizeof(int32_t) * o[nq]);
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
