// Solid sampling of a closed triangle mesh on a lattice (scene generation).
//
// The reference voxel-samples OBJ meshes into boundary particles
// (wp_sph/solver/model.py:14-60): a lattice np.arange(lo, hi, spacing) per
// axis over the mesh's bounds, meshgrid in "ij" order, trimesh's
// mesh.contains on every lattice point, then `points @ rot + pos`.
// init_particles uses it for the HOUSE, PLANE and HAND scenes
// (IISPH.py:952-989).
//
// Inside test: parity of the crossings of a ray from the point along +x.
// Every lattice point of one (y, z) column shares the ray's line, so a column
// is one block: its threads intersect the line with the column's candidate
// triangles (binned on the host by their y, z extent), collect the crossing
// x-coordinates in shared memory, and then each point of the column counts
// the crossings beyond it.  Crossings are counted exactly once on a closed
// mesh, also where the line runs through an edge or a vertex: the 2-D edge
// functions are evaluated on each edge in a canonical (lexicographic)
// direction, so the two triangles sharing an edge see exactly opposite
// values, and a zero is resolved by a symbolic perturbation of the query
// point by (e, e^2) (simulation of simplicity), which both triangles resolve
// the same way.  All arithmetic is FP64 with explicitly rounded operations,
// so a CPU restatement in the same order reproduces the point set bit for
// bit.
#include <algorithm>
#include <vector>

#include "sph_internal.cuh"

namespace sph {
namespace {

constexpr int kColThreads = 128;
constexpr int kMaxHits = 1024;  // crossings of one lattice line with the mesh

struct Tri {
  double ax, ay, az, bx, by, bz, cx, cy, cz;
};

// Edge function of the 2-D edge p -> q at (y, z), in (y, z) coordinates,
// evaluated in the canonical direction of the edge and perturbed on a zero.
// Returns the unperturbed value in *e and the sign of the perturbed one.
__device__ inline int edge_sign(double py, double pz, double qy, double qz, double y, double z, double* e) {
  const bool swap = (py > qy) || (py == qy && pz > qz);
  if (swap) {
    double t = py;
    py = qy;
    qy = t;
    t = pz;
    pz = qz;
    qz = t;
  }
  const double d1 = __dsub_rn(qy, py), d2 = __dsub_rn(z, pz), d3 = __dsub_rn(qz, pz), d4 = __dsub_rn(y, py);
  double v = __dsub_rn(__dmul_rn(d1, d2), __dmul_rn(d3, d4));
  int s = (v > 0) - (v < 0);
  // the query moved to (y + e, z + e^2): first-order term -d3 e, then d1 e^2
  if (s == 0) s = (d3 != 0) ? ((d3 < 0) - (d3 > 0)) : ((d1 > 0) - (d1 < 0));
  if (swap) {
    v = -v;
    s = -s;
  }
  *e = v;
  return s;
}

// Whether the line {(x, y, z)} crosses triangle t, and where (*x).
__device__ inline bool crossing(const Tri& t, double y, double z, double* x) {
  double e0, e1, e2;
  const int s0 = edge_sign(t.by, t.bz, t.cy, t.cz, y, z, &e0);
  const int s1 = edge_sign(t.cy, t.cz, t.ay, t.az, y, z, &e1);
  const int s2 = edge_sign(t.ay, t.az, t.by, t.bz, y, z, &e2);
  if (s0 == 0 || s0 != s1 || s1 != s2) return false;
  const double den = __dadd_rn(__dadd_rn(e0, e1), e2);
  if (den == 0.0) return false;  // no area in the projection
  // x_a + (e1 (x_b - x_a) + e2 (x_c - x_a)) / den: exact on faces normal to x
  const double num = __dadd_rn(__dmul_rn(e1, __dsub_rn(t.bx, t.ax)), __dmul_rn(e2, __dsub_rn(t.cx, t.ax)));
  *x = __dadd_rn(t.ax, __ddiv_rn(num, den));
  return true;
}

// One block per lattice line (iy, iz): the line's crossings, then the parity
// of the crossings beyond each lattice point of the line.
__global__ void __launch_bounds__(kColThreads) k_mesh_columns(
    int nx, int ny, int nz, const double* __restrict__ xs, const double* __restrict__ ys,
    const double* __restrict__ zs, const Tri* __restrict__ tris, const long long* __restrict__ col_off,
    const int* __restrict__ col_tri, unsigned char* __restrict__ inside, int* overflow) {
  __shared__ double s_hit[kMaxHits];
  __shared__ int s_n;
  const int col = blockIdx.x;  // iy * nz + iz
  const int iy = col / nz, iz = col % nz;
  const double y = ys[iy], z = zs[iz];
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (long long k = col_off[col] + threadIdx.x; k < col_off[col + 1]; k += blockDim.x) {
    double xh;
    if (crossing(tris[col_tri[k]], y, z, &xh)) {
      const int slot = atomicAdd(&s_n, 1);
      if (slot < kMaxHits) s_hit[slot] = xh;
    }
  }
  __syncthreads();
  const int nh = s_n;
  if (nh > kMaxHits) {
    if (threadIdx.x == 0) atomicOr(overflow, 1);
    return;
  }
  for (int ix = threadIdx.x; ix < nx; ix += blockDim.x) {
    const double x = xs[ix];
    int c = 0;
    for (int h = 0; h < nh; ++h) c += (s_hit[h] > x) ? 1 : 0;
    inside[((long long)ix * ny + iy) * nz + iz] = (unsigned char)(c & 1);
  }
}

constexpr int kChunk = 1024;  // lattice points per counting block

__global__ void __launch_bounds__(kChunk) k_mesh_count(long long npts, const unsigned char* __restrict__ inside,
                                                      long long* __restrict__ chunk_count) {
  const long long i = (long long)blockIdx.x * kChunk + threadIdx.x;
  const int v = (i < npts) ? inside[i] : 0;
  const int c = __syncthreads_count(v);
  if (threadIdx.x == 0) chunk_count[blockIdx.x] = c;
}

// exclusive scan of the chunk counts in one block, in place; total in *total
__global__ void __launch_bounds__(1024) k_mesh_scan(long long nchunks, long long* __restrict__ c, long long* total) {
  __shared__ long long s_part[1024];
  const long long per = (nchunks + 1023) / 1024;
  const long long b = threadIdx.x * per, e = min(b + per, nchunks);
  long long s = 0;
  for (long long k = b; k < e; ++k) s += c[k];
  s_part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int t = 0; t < 1024; ++t) {
      const long long v = s_part[t];
      s_part[t] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  long long run = s_part[threadIdx.x];
  for (long long k = b; k < e; ++k) {
    const long long v = c[k];
    c[k] = run;
    run += v;
  }
}

// inside lattice points in lattice order, rotated and translated:
// out = p @ rot + pos (row vector times the 3 x 3 matrix), in float32
__global__ void __launch_bounds__(kChunk) k_mesh_emit(long long npts, int ny, int nz, const double* __restrict__ xs,
                                                     const double* __restrict__ ys, const double* __restrict__ zs,
                                                     const unsigned char* __restrict__ inside,
                                                     const long long* __restrict__ chunk_off, const double* __restrict__ rt,
                                                     long long cap, float* __restrict__ out) {
  __shared__ int s_warp[kChunk / 32];
  const long long i = (long long)blockIdx.x * kChunk + threadIdx.x;
  const int v = (i < npts) ? inside[i] : 0;
  const unsigned int ball = __ballot_sync(0xffffffffu, v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) s_warp[w] = __popc(ball);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < kChunk / 32; ++k) {
      const int t = s_warp[k];
      s_warp[k] = run;
      run += t;
    }
  }
  __syncthreads();
  if (!v) return;
  const long long slot = chunk_off[blockIdx.x] + s_warp[w] + __popc(ball & ((1u << lane) - 1u));
  if (slot >= cap) return;
  const long long ix = i / ((long long)ny * nz), rem = i % ((long long)ny * nz);
  const double p[3] = {xs[ix], ys[rem / nz], zs[rem % nz]};
  for (int k = 0; k < 3; ++k) {
    double acc = __dadd_rn(__dmul_rn(p[0], rt[0 * 3 + k]), __dmul_rn(p[1], rt[1 * 3 + k]));
    acc = __dadd_rn(acc, __dmul_rn(p[2], rt[2 * 3 + k]));
    out[3 * slot + k] = float(__dadd_rn(acc, rt[9 + k]));
  }
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(n, 1)); }
};

// first index k with a[k] >= v (a ascending)
int64_t lower(const double* a, int n, double v) { return std::lower_bound(a, a + n, v) - a; }
// one past the last index k with a[k] <= v
int64_t upper(const double* a, int n, double v) { return std::upper_bound(a, a + n, v) - a; }

}  // namespace
}  // namespace sph

extern "C" int sph_sample_solid(const double* verts3, int64_t nv, const int32_t* tris3, int64_t nt, const double* xs,
                                int32_t nx, const double* ys, int32_t ny, const double* zs, int32_t nz,
                                const double* rot9, const double* pos3, float* out3, int64_t cap, int64_t* count,
                                int32_t device) {
  using namespace sph;
  if (!count || nv < 0 || nt < 0 || nx < 0 || ny < 0 || nz < 0 || cap < 0) return SPH_E_INVALID;
  if ((nt > 0 && (!verts3 || !tris3)) || (nx && !xs) || (ny && !ys) || (nz && !zs) || !rot9 || !pos3 ||
      (cap > 0 && !out3))
    return SPH_E_INVALID;
  *count = 0;
  const long long npts = (long long)nx * ny * nz;
  if (npts == 0 || nt == 0) return SPH_OK;
  if (npts > (1ll << 40)) return SPH_E_INVALID;
  for (int a = 1; a < nx; ++a)
    if (!(xs[a] > xs[a - 1])) return SPH_E_INVALID;
  for (int a = 1; a < ny; ++a)
    if (!(ys[a] > ys[a - 1])) return SPH_E_INVALID;
  for (int a = 1; a < nz; ++a)
    if (!(zs[a] > zs[a - 1])) return SPH_E_INVALID;

  // triangles as 9 doubles each, and each triangle's candidate lattice lines
  std::vector<Tri> tri(nt);
  std::vector<int64_t> y0(nt), y1(nt), z0(nt), z1(nt);
  std::vector<long long> col_cnt((size_t)ny * nz + 1, 0);
  for (int64_t t = 0; t < nt; ++t) {
    const int32_t* f = tris3 + 3 * t;
    for (int k = 0; k < 3; ++k)
      if (f[k] < 0 || f[k] >= nv) return SPH_E_INVALID;
    const double* A = verts3 + 3 * f[0];
    const double* B = verts3 + 3 * f[1];
    const double* C = verts3 + 3 * f[2];
    tri[t] = Tri{A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1], C[2]};
    const double ylo = std::min({A[1], B[1], C[1]}), yhi = std::max({A[1], B[1], C[1]});
    const double zlo = std::min({A[2], B[2], C[2]}), zhi = std::max({A[2], B[2], C[2]});
    if (!(ylo == ylo) || !(yhi == yhi) || !(zlo == zlo) || !(zhi == zhi)) return SPH_E_INVALID;
    // lines with ylo <= y <= yhi and zlo <= z <= zhi (the exact test decides)
    y0[t] = lower(ys, ny, ylo);
    y1[t] = upper(ys, ny, yhi);
    z0[t] = lower(zs, nz, zlo);
    z1[t] = upper(zs, nz, zhi);
    for (int64_t iy = y0[t]; iy < y1[t]; ++iy)
      for (int64_t iz = z0[t]; iz < z1[t]; ++iz) col_cnt[iy * nz + iz + 1] += 1;
  }
  for (size_t c = 1; c < col_cnt.size(); ++c) col_cnt[c] += col_cnt[c - 1];
  const long long npairs = col_cnt.back();
  if (npairs > (1ll << 31) - 1) return SPH_E_TOO_LARGE;
  std::vector<int> col_tri(std::max<long long>(npairs, 1));
  {
    std::vector<long long> fill(col_cnt.begin(), col_cnt.end() - 1);
    for (int64_t t = 0; t < nt; ++t)
      for (int64_t iy = y0[t]; iy < y1[t]; ++iy)
        for (int64_t iz = z0[t]; iz < z1[t]; ++iz) col_tri[fill[iy * nz + iz]++] = int(t);
  }

  if (cudaSetDevice(device) != cudaSuccess) return SPH_E_CUDA;
  DevBuf<double> dx, dy, dz, drt;
  DevBuf<Tri> dtri;
  DevBuf<long long> doff, dchunk, dtotal;
  DevBuf<int> dcol, dover;
  DevBuf<unsigned char> dinside;
  DevBuf<float> dout;
  const long long nchunks = (npts + kChunk - 1) / kChunk;
  const long long ncap = std::min<long long>(cap, npts);
  if (dx.alloc(nx) || dy.alloc(ny) || dz.alloc(nz) || drt.alloc(12) || dtri.alloc(nt) ||
      doff.alloc(col_cnt.size()) || dcol.alloc(col_tri.size()) || dover.alloc(1) || dinside.alloc(npts) ||
      dchunk.alloc(nchunks) || dtotal.alloc(1) || dout.alloc(3 * std::max<long long>(ncap, 1)))
    return SPH_E_NOMEM;
  double rt[12];
  for (int k = 0; k < 9; ++k) rt[k] = rot9[k];
  for (int k = 0; k < 3; ++k) rt[9 + k] = pos3[k];
  cudaError_t e = cudaSuccess;
  auto up = [&](void* d, const void* h, size_t b) {
    if (e == cudaSuccess) e = cudaMemcpy(d, h, b, cudaMemcpyHostToDevice);
  };
  up(dx.p, xs, sizeof(double) * nx);
  up(dy.p, ys, sizeof(double) * ny);
  up(dz.p, zs, sizeof(double) * nz);
  up(drt.p, rt, sizeof(rt));
  up(dtri.p, tri.data(), sizeof(Tri) * nt);
  up(doff.p, col_cnt.data(), sizeof(long long) * col_cnt.size());
  up(dcol.p, col_tri.data(), sizeof(int) * col_tri.size());
  if (e == cudaSuccess) e = cudaMemset(dover.p, 0, sizeof(int));
  if (e != cudaSuccess) return SPH_E_CUDA;

  k_mesh_columns<<<ny * nz, kColThreads>>>(nx, ny, nz, dx.p, dy.p, dz.p, dtri.p, doff.p, dcol.p, dinside.p, dover.p);
  k_mesh_count<<<unsigned(nchunks), kChunk>>>(npts, dinside.p, dchunk.p);
  k_mesh_scan<<<1, 1024>>>(nchunks, dchunk.p, dtotal.p);
  k_mesh_emit<<<unsigned(nchunks), kChunk>>>(npts, ny, nz, dx.p, dy.p, dz.p, dinside.p, dchunk.p, drt.p, ncap, dout.p);
  if (cudaGetLastError() != cudaSuccess) return SPH_E_CUDA;
  int over = 0;
  long long total = 0;
  if (cudaMemcpy(&over, dover.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SPH_E_CUDA;
  if (over) return SPH_E_CAPACITY;  // more than kMaxHits crossings on one lattice line
  if (cudaMemcpy(&total, dtotal.p, sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess) return SPH_E_CUDA;
  *count = total;
  if (total > cap) return SPH_E_TOO_LARGE;
  if (total > 0 &&
      cudaMemcpy(out3, dout.p, sizeof(float) * 3 * size_t(total), cudaMemcpyDeviceToHost) != cudaSuccess)
    return SPH_E_CUDA;
  return SPH_OK;
}
