// Boundary volumes (psi) without any memory allocation.
//
// Who needs this: callers that are not allowed to call cudaMalloc.  Typical
// cases are a host framework that owns all device memory through its own
// pool and forbids foreign allocations (an allocation behind its back can fail
// or fragment memory it has already handed out), and embedded or real-time
// callers that must not allocate after start-up because an allocation can
// block or fail at an arbitrary time.  Such a caller allocates its inputs and
// outputs itself and needs the library to bring its own scratch memory.
//
// sph_boundary_psi_noalloc computes the same psi as sph_set_boundary (the
// reference's compute_boundary_density, IISPH.py:23-49), but its scratch — the
// packed positions, the cell counting sort and the cell table — lives in one
// file-scope __device__ array, g_noalloc_scratch, sized for at most
// SPH_NOALLOC_MAX_BOUNDARY particles and SPH_NOALLOC_MAX_CELLS grid cells.
// Every device that loads this library holds that array until the process
// exits.  All calls share it, and it keeps the previous call's contents: the
// per-cell counters are cleared at the start of every call, everything else is
// fully overwritten.  Two calls whose work overlaps on the GPU (different
// streams, or different host threads without ordering) race on the array.
// The array's device address is looked up once per device, on that device's
// first call, and kept: after a cudaDeviceReset of that device the module is
// loaded anew and the kept address is stale, so the entry point must not be
// used on a device after it has been reset.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "sph_internal.cuh"

namespace sph {
namespace {

constexpr long long kMaxB = SPH_NOALLOC_MAX_BOUNDARY;
constexpr long long kMaxCells = SPH_NOALLOC_MAX_CELLS;
constexpr long long kScanParts = kMaxCells / 4096 + 2;
// largest explicit domain extent accepted, in support radii per axis
constexpr double kMaxDomainCells = 1e7;

// byte offsets inside the scratch array (each 256-byte aligned)
constexpr long long al(long long b) { return (b + 255) / 256 * 256; }
constexpr long long kOffPosIn = 0;
constexpr long long kOffPosSorted = kOffPosIn + al(16 * kMaxB);
constexpr long long kOffKey = kOffPosSorted + al(16 * kMaxB);
constexpr long long kOffRank = kOffKey + al(4 * kMaxB);
constexpr long long kOffSrc = kOffRank + al(4 * kMaxB);
constexpr long long kOffOrig = kOffSrc + al(4 * kMaxB);
constexpr long long kOffSortedOrig = kOffOrig + al(4 * kMaxB);
constexpr long long kOffPsi = kOffSortedOrig + al(4 * kMaxB);
constexpr long long kOffCellCount = kOffPsi + al(4 * kMaxB);
constexpr long long kOffCellStart = kOffCellCount + al(4 * kMaxCells);
constexpr long long kOffScanPart = kOffCellStart + al(4 * (kMaxCells + 1));
constexpr long long kOffBox = kOffScanPart + al(4 * kScanParts);
constexpr long long kScratchBytes = kOffBox + al(4 * 8);
static_assert(kScratchBytes <= 24ll * 1024 * 1024, "the no-allocation scratch is documented as at most 24 MiB");

// The scratch array.  In host code this name is only a host-side stand-in for
// the symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per device.
cudaError_t scratch_address(int dev, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return cudaSuccess;
}

__global__ void k_pack_points(int n, const float* __restrict__ x3, float4* __restrict__ pos,
                              int* __restrict__ orig) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[i] = make_float4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], 0.f);
  orig[i] = i;
}

// Bounding box of the (finite) points, one block: box = {min xyz, max xyz}.
__global__ void __launch_bounds__(1024) k_bbox(int n, const float4* __restrict__ pos, float* box) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 p = pos[i];
    const float v[3] = {p.x, p.y, p.z};
    for (int a = 0; a < 3; ++a)
      if (isfinite(v[a])) {
        lo[a] = fminf(lo[a], v[a]);
        hi[a] = fmaxf(hi[a], v[a]);
      }
  }
  __shared__ float s_lo[3][32], s_hi[3][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
    if (lane == 0) {
      s_lo[a][w] = lo[a];
      s_hi[a][w] = hi[a];
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int a = threadIdx.x;
    float l = INFINITY, h = -INFINITY;
    for (int k = 0; k < int(blockDim.x >> 5); ++k) {
      l = fminf(l, s_lo[a][k]);
      h = fmaxf(h, s_hi[a][k]);
    }
    box[a] = l;
    box[3 + a] = h;
  }
}

// Smallest float r2 with sqrtf(r2) >= h (same rule as the context path).
float r2_limit(float h) {
  float t = h * h;
  while (std::sqrt(t) >= h) t = std::nextafter(t, 0.0f);
  while (std::sqrt(t) < h) t = std::nextafter(t, INFINITY);
  return t;
}

}  // namespace
}  // namespace sph

extern "C" int sph_boundary_psi_noalloc(const SphParams* params, const float* d_xb3, int64_t nb,
                                        const float* d_w_table, float* d_psi, void* stream) {
  using namespace sph;
  if (!params || nb < 0 || (nb > 0 && (!d_xb3 || !d_w_table || !d_psi))) return SPH_E_INVALID;
  if (nb > kMaxB) return SPH_E_TOO_LARGE;  // more than SPH_NOALLOC_MAX_BOUNDARY particles
  if (!(params->h > 0) || !std::isfinite(params->h) || params->w_table_size < 2) return SPH_E_INVALID;
  if (!std::isfinite(params->rho0)) return SPH_E_INVALID;
  // an explicit grid extent must be finite and not absurdly many cells wide:
  // the cell count below is computed from it before any kernel is launched
  bool have_domain = false;
  for (int a = 0; a < 3; ++a) {
    const double dmin = params->domain_min[a], dmax = params->domain_max[a];
    if (!std::isfinite(dmin) || !std::isfinite(dmax)) return SPH_E_INVALID;
    have_domain = have_domain || (dmax > dmin);
  }
  if (have_domain)
    for (int a = 0; a < 3; ++a)
      if (params->domain_max[a] - params->domain_min[a] > kMaxDomainCells * params->h)
        return SPH_E_INVALID;
  if (nb == 0) return SPH_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SPH_E_CUDA;
  unsigned char* base = nullptr;
  if (scratch_address(dev, &base) != cudaSuccess) return SPH_E_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = int(nb);
  float4* pos_in = reinterpret_cast<float4*>(base + kOffPosIn);
  float4* pos_sorted = reinterpret_cast<float4*>(base + kOffPosSorted);
  int* orig = reinterpret_cast<int*>(base + kOffOrig);
  int* sorted_orig = reinterpret_cast<int*>(base + kOffSortedOrig);
  float* psi_sorted = reinterpret_cast<float*>(base + kOffPsi);
  float* box = reinterpret_cast<float*>(base + kOffBox);

  k_pack_points<<<(n + 255) / 256, 256, 0, s>>>(n, d_xb3, pos_in, orig);
  if (cudaGetLastError() != cudaSuccess) return SPH_E_CUDA;

  // grid extent: params.domain when given, else the points' bounding box
  // (read back to the host: this synchronises `stream`)
  double lo[3], hi[3];
  if (have_domain) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = params->domain_min[a];
      hi[a] = params->domain_max[a];
    }
  } else {
    float hb[6];
    k_bbox<<<1, 1024, 0, s>>>(n, pos_in, box);
    if (cudaMemcpyAsync(hb, box, sizeof(hb), cudaMemcpyDeviceToHost, s) != cudaSuccess) return SPH_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return SPH_E_CUDA;
    for (int a = 0; a < 3; ++a) {
      lo[a] = hb[a] <= hb[3 + a] ? hb[a] : 0.0;
      hi[a] = hb[a] <= hb[3 + a] ? hb[3 + a] : 0.0;
    }
  }
  // Cell counts are formed in double (the extents are finite: checked above,
  // or the bounding box of finite coordinates), so nothing overflows before
  // the comparison; each pass grows the cell by 1.25, so the loop ends.
  double cell = double(float(params->h)) * 1.01;
  const double pad = 2.0 * params->h;
  long long dims[3], tot;
  for (;;) {
    double dd[3], td = 1.0;
    for (int a = 0; a < 3; ++a) {
      const double w = a == 0 ? cell / kXSplit : cell;
      dd[a] = std::max(1.0, std::ceil((hi[a] - lo[a] + 2 * pad) / w) + 1.0);
      td *= dd[a];
    }
    if (td <= double(kMaxCells)) {
      tot = 1;
      for (int a = 0; a < 3; ++a) {
        dims[a] = (long long)dd[a];
        tot *= dims[a];
      }
      break;
    }
    cell *= 1.25;  // coarser cells keep the search complete
  }
  Grid g{};
  g.ox = float(lo[0] - pad);
  g.oy = float(lo[1] - pad);
  g.oz = float(lo[2] - pad);
  g.inv_cell = float(1.0 / cell);
  g.inv_cell_x = float(kXSplit / cell);
  g.nx = int(dims[0]);
  g.ny = int(dims[1]);
  g.nz = int(dims[2]);
  g.ncells = int(tot);

  SortArgs sa{};
  sa.n = n;
  sa.grid = g;
  sa.pos = pos_in;
  sa.orig = orig;
  sa.key = reinterpret_cast<int*>(base + kOffKey);
  sa.rank = reinterpret_cast<int*>(base + kOffRank);
  sa.cell_count = reinterpret_cast<int*>(base + kOffCellCount);  // cleared by launch_sort
  sa.cell_start = reinterpret_cast<int*>(base + kOffCellStart);
  sa.scan_part = reinterpret_cast<int*>(base + kOffScanPart);
  sa.sort_src = reinterpret_cast<int*>(base + kOffSrc);
  sa.sort_orig = sorted_orig;
  if (launch_sort(sa, g.ncells, s) != cudaSuccess) return SPH_E_CUDA;
  // reuse the rank array as the gather's (unused) original-id output
  if (launch_gather(n, sa.sort_src, sorted_orig, pos_in, nullptr, nullptr, pos_sorted, nullptr, sa.rank, nullptr,
                    s) != cudaSuccess)
    return SPH_E_CUDA;

  PsiArgs pa{};
  pa.nb = n;
  pa.grid = g;
  pa.c.h = float(params->h);
  pa.c.r2_limit = r2_limit(pa.c.h);
  pa.c.sw = params->w_table_size;
  pa.c.w_scale = float(params->w_table_size - 1) * float(1.0 / params->h);
  pa.c.rho0 = float(params->rho0);
  pa.w_table = d_w_table;
  // spline_W(0) = W_table[0], read by the kernel from the caller's table
  pa.w0_from_table = 1;
  pa.bpos = pos_sorted;
  pa.bcell_start = sa.cell_start;
  if (launch_psi_sorted(pa, psi_sorted, 256, s) != cudaSuccess) return SPH_E_CUDA;
  if (launch_unsort1(n, sorted_orig, psi_sorted, d_psi, s) != cudaSuccess) return SPH_E_CUDA;
  return SPH_OK;
}
