// Host-buffer state exchange for the C ABI: packed xyz float3 in original
// particle order <-> the float4 cell-sorted device layout.  One coalesced
// host<->device copy per field plus one gather/scatter kernel, instead of
// host-side loops.
#include "sph_internal.cuh"

namespace sph {

// Particles [base, base + n) of the state from packed host-order float3
// arrays (and pressures, NULL = 0); their original ids are base + (index in
// the arrays).
__global__ void k_pack_fluid(int n, int base, const float* __restrict__ x3, const float* __restrict__ v3,
                             const float* __restrict__ p_in, float4* __restrict__ pos, float4* __restrict__ vel,
                             int* __restrict__ orig, float* __restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = base + i;
  pos[k] = make_float4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], 0.f);
  vel[k] = v3 ? make_float4(v3[3 * i], v3[3 * i + 1], v3[3 * i + 2], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
  orig[k] = k;
  p[k] = p_in ? p_in[i] : 0.f;
}

// out[orig[k]] = src[k].xyz  (component = -1)  or  src[k].{x,y,z,w}[component]
__global__ void k_unsort4(int n, const int* __restrict__ orig, const float4* __restrict__ src, int component,
                          float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float4 v = src[k];
  const int o = orig[k];
  if (component < 0) {
    out[3 * o] = v.x;
    out[3 * o + 1] = v.y;
    out[3 * o + 2] = v.z;
  } else {
    out[o] = component == 0 ? v.x : component == 1 ? v.y : component == 2 ? v.z : v.w;
  }
}

__global__ void k_unsort1(int n, const int* __restrict__ orig, const float* __restrict__ src,
                          float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[orig[k]] = src[k];
}

__global__ void k_sort1(int n, const int* __restrict__ orig, const float* __restrict__ src,
                        float* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = src[orig[k]];
}

cudaError_t launch_pack_fluid(int n, int base, const float* x3, const float* v3, float4* pos, float4* vel,
                              int* orig, float* p, cudaStream_t s, const float* p_in) {
  if (n <= 0) return cudaSuccess;
  k_pack_fluid<<<(n + 255) / 256, 256, 0, s>>>(n, base, x3, v3, p_in, pos, vel, orig, p);
  return cudaGetLastError();
}

cudaError_t launch_unsort4(int n, const int* orig, const float4* src, int component, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_unsort4<<<(n + 255) / 256, 256, 0, s>>>(n, orig, src, component, out);
  return cudaGetLastError();
}

cudaError_t launch_unsort1(int n, const int* orig, const float* src, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_unsort1<<<(n + 255) / 256, 256, 0, s>>>(n, orig, src, out);
  return cudaGetLastError();
}

cudaError_t launch_sort1(int n, const int* orig, const float* src, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_sort1<<<(n + 255) / 256, 256, 0, s>>>(n, orig, src, out);
  return cudaGetLastError();
}

}  // namespace sph
