// Cell counting sort of particles (replaces wp.HashGrid.build, used at
// IISPH.py:811 and IISPH.py:1414, and hash_grid_point_id at the 12 call sites
// listed in IISPH.py:33-532).
//
// Order produced: ascending (cell index, original id).  The cell index runs x
// fastest (over half cells, Grid), so the x-adjacent cells of each of a
// particle's 3x3 neighbour rows are one contiguous particle range.  Within a
// cell, particles are ordered by original
// id, which makes the sorted order a pure function of the positions (no
// dependence on atomics or on the previous step's order).
//
//   1. k_cell_keys   cell key per particle; rank inside its cell from a
//                    warp-aggregated atomic on the cell counter
//   2. k_scan_onepass  exclusive scan -> cell_start in one kernel: each tile
//                    of cells publishes its sum, then looks back over the
//                    tiles before it (decoupled look-back) for its prefix
//      (or, where no status buffer is given, k_scan_part: per-block sums of
//      the cell counters, then k_scan_final: each block first sums the
//      partials before it, no inter-block waiting)
//   3. k_scatter     new slot = cell_start[key] + rank
//   4. k_cell_sort   order each cell's slots by original id
#include "sph_internal.cuh"

namespace sph {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;  // cells per thread
constexpr int kScanTile = kScanThreads * kScanItems;
int scan_tiles(int ncells) { return (ncells + kScanTile - 1) / kScanTile; }

__global__ void k_cell_keys(SortArgs a, int scan_tiles) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (a.scan_status && blockIdx.x == 0) {
    // the single-pass scan's tile states and ticket start from zero
    for (int t = threadIdx.x; t < scan_tiles; t += blockDim.x) a.scan_status[t] = 0ull;
    if (threadIdx.x == 0) *a.scan_ticket = 0u;
  }
  bool live = i < a.n;
  int key = -1;
  if (live) {
    const float4 x = a.pos[i];
    const CellFrame f = frame_of(a.scenes, a.grid, a.boundary != 0, i);
    key = f.base + cell_index(f.g, cell_coord(f.g, x.x, x.y, x.z));
    a.key[i] = key;
  }
  unsigned int active = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  // lanes sharing a cell: one atomic per group, ranks by lane order
  unsigned int peers = __match_any_sync(active, key);
  int leader = __ffs(peers) - 1;
  int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == leader) base = atomicAdd(&a.cell_count[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  a.rank[i] = base + __popc(peers & ((1u << lane) - 1u));
}

__device__ inline int block_sum_int(int v, int* sm) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sm[w] = v;
  __syncthreads();
  int nw = blockDim.x >> 5;
  int t = (threadIdx.x < nw) ? sm[threadIdx.x] : 0;
  if (w == 0) t = warp_sum(t);
  __syncthreads();
  if (threadIdx.x == 0) sm[0] = t;
  __syncthreads();
  int r = sm[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_part(const int* __restrict__ count, int ncells, int* part) {
  __shared__ int sm[32];
  int base = blockIdx.x * kScanTile;
  int v = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int c = base + k * kScanThreads + threadIdx.x;
    if (c < ncells) v += count[c];
  }
  v = block_sum_int(v, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_final(const int* __restrict__ count, int ncells,
                                                             const int* __restrict__ part, int* start, int n) {
  __shared__ int sm[32];
  __shared__ int warp_tot[kScanThreads / 32];
  // prefix of earlier tiles
  int pre = 0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += kScanThreads) pre += part[b];
  pre = block_sum_int(pre, sm);
  // each thread scans kScanItems consecutive cells
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int tot = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int c = base + k;
    v[k] = (c < ncells) ? count[c] : 0;
    tot += v[k];
  }
  // exclusive scan of thread totals
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    int t = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
    int ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += u;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = ti - t;
  }
  __syncthreads();
  int run = pre + warp_tot[w] + inc - tot;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int c = base + k;
    if (c < ncells) start[c] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) start[ncells] = n;
}

// Tile states of the single-pass scan: flag in the high word.
constexpr unsigned long long kTileAggregate = 1ull << 32;  // the tile's own sum is published
constexpr unsigned long long kTilePrefix = 2ull << 32;     // the inclusive prefix through the tile
constexpr long long kLookBackPolls = 1ll << 22;            // bound on one look-back wait

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive scan of the cell counters into cell_start in one kernel.  Tiles
// are taken in ticket order, so every tile before this one has started and
// publishes its sum without waiting on anything: each look-back wait ends.
// It is still bounded (kLookBackPolls); if one ran out, SPH_F_TIMEOUT is set
// and the step's results are discarded by the host.
__global__ void __launch_bounds__(kScanThreads) k_scan_onepass(const int* __restrict__ count, int ncells,
                                                               unsigned long long* status, unsigned int* ticket,
                                                               int* start, int n, int* err) {
  __shared__ int s_tile, s_pre;
  __shared__ int warp_tot[kScanThreads / 32];
  if (threadIdx.x == 0) s_tile = int(atomicAdd(ticket, 1u));
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int tot = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int c = base + k;
    v[k] = (c < ncells) ? count[c] : 0;
    tot += v[k];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int t = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
    int ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += u;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = ti - t;
    if (lane == kScanThreads / 32 - 1) {
      // ti is the tile's sum: publish it, find the prefix, publish that
      const unsigned int agg = unsigned(ti);
      int pre = 0;
      if (tile == 0) {
        st_release_u64(status, kTilePrefix | agg);
      } else {
        st_release_u64(status + tile, kTileAggregate | agg);
        long long polls = 0;
        for (int t = tile - 1; t >= 0;) {
          const unsigned long long st = ld_acquire_u64(status + t);
          const unsigned long long flag = st & ~0xffffffffull;
          if (flag == 0ull) {
            if (++polls > kLookBackPolls) {
              atomicOr(err, SPH_F_TIMEOUT);
              break;
            }
            __nanosleep(32);
            continue;
          }
          pre += int(unsigned(st & 0xffffffffull));
          if (flag == kTilePrefix) break;
          --t;
        }
        st_release_u64(status + tile, kTilePrefix | unsigned(pre + int(agg)));
      }
      s_pre = pre;
    }
  }
  __syncthreads();
  int run = s_pre + warp_tot[w] + inc - tot;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int c = base + k;
    if (c < ncells) start[c] = run;
    run += v[k];
  }
  if (tile == int(gridDim.x) - 1 && threadIdx.x == 0) start[ncells] = n;
}

__global__ void k_scatter(SortArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int dst = a.cell_start[a.key[i]] + a.rank[i];
  a.sort_src[dst] = i;
  a.sort_orig[dst] = a.orig[i];
}

// Insertion sort of one cell's slots by original id.  Cells hold ~8 particles
// at rest density; the register path covers up to 32, larger cells sort in place.
__global__ void k_cell_sort(const int* __restrict__ start, int ncells, int* src, int* orig) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  int b = start[c], e = start[c + 1];
  int len = e - b;
  if (len < 2) return;
  if (len <= 32) {
    int ko[32], ks[32];
    for (int t = 0; t < len; ++t) {
      int o = orig[b + t], s = src[b + t];
      int u = t;
      while (u > 0 && ko[u - 1] > o) {
        ko[u] = ko[u - 1];
        ks[u] = ks[u - 1];
        --u;
      }
      ko[u] = o;
      ks[u] = s;
    }
    for (int t = 0; t < len; ++t) {
      orig[b + t] = ko[t];
      src[b + t] = ks[t];
    }
  } else {
    for (int t = b + 1; t < e; ++t) {
      int o = orig[t], s = src[t];
      int u = t;
      while (u > b && orig[u - 1] > o) {
        orig[u] = orig[u - 1];
        src[u] = src[u - 1];
        --u;
      }
      orig[u] = o;
      src[u] = s;
    }
  }
}

__global__ void k_gather(int n, const int* __restrict__ sort_src, const int* __restrict__ sort_orig,
                         const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                         const float* __restrict__ p_in, float4* __restrict__ pos_out,
                         float4* __restrict__ vel_out, int* __restrict__ orig_out, float* __restrict__ p_out,
                         float2* __restrict__ yz_out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int s = sort_src[k];
  const float4 x = pos_in[s];
  pos_out[k] = x;
  if (yz_out) yz_out[k] = make_float2(x.y, x.z);
  if (vel_out) {
    float4 v = vel_in[s];
    // with the (y, z) copy, the velocity record carries x in its .w: the
    // build then gathers a neighbour's position and velocity as 24 bytes
    if (yz_out) v.w = x.x;
    vel_out[k] = v;
  }
  orig_out[k] = sort_orig[k];
  if (p_out) p_out[k] = p_in[s];
}

cudaError_t launch_sort(const SortArgs& a, int ncells, cudaStream_t s) {
  if (a.n <= 0) return cudaMemsetAsync(a.cell_start, 0, sizeof(int) * (ncells + 1), s);
  cudaError_t e = cudaMemsetAsync(a.cell_count, 0, sizeof(int) * ncells, s);
  if (e != cudaSuccess) return e;
  const int T = 256;
  int gb = (a.n + T - 1) / T;
  int tiles = (ncells + kScanTile - 1) / kScanTile;
  k_cell_keys<<<gb, T, 0, s>>>(a, tiles);
  if (a.scan_status) {
    k_scan_onepass<<<tiles, kScanThreads, 0, s>>>(a.cell_count, ncells, a.scan_status, a.scan_ticket, a.cell_start,
                                                 a.n, a.err);
  } else {
    k_scan_part<<<tiles, kScanThreads, 0, s>>>(a.cell_count, ncells, a.scan_part);
    k_scan_final<<<tiles, kScanThreads, 0, s>>>(a.cell_count, ncells, a.scan_part, a.cell_start, a.n);
  }
  k_scatter<<<gb, T, 0, s>>>(a);
  k_cell_sort<<<(ncells + T - 1) / T, T, 0, s>>>(a.cell_start, ncells, a.sort_src, a.sort_orig);
  return cudaGetLastError();
}

cudaError_t launch_gather(int n, const int* sort_src, const int* sort_orig, const float4* pos_in,
                          const float4* vel_in, const float* p_in, float4* pos_out, float4* vel_out,
                          int* orig_out, float* p_out, cudaStream_t s, float2* yz_out) {
  if (n <= 0) return cudaSuccess;
  const int T = 256;
  k_gather<<<(n + T - 1) / T, T, 0, s>>>(n, sort_src, sort_orig, pos_in, vel_in, p_in, pos_out, vel_out,
                                        orig_out, p_out, yz_out);
  return cudaGetLastError();
}

}  // namespace sph
