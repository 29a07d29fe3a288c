// composite.cu — nearest-depth composite of the frames of one animation's
// subtrees.  Each subtree is a scene of its own traced over the whole image
// (depth -1 where its rays miss); per pixel the part with the least key
// (depth bits, then subtree index) wins.  Both kernels are elementwise and
// HBM-bound: a grid-stride loop over pixels, one thread per pixel a step,
// every access coalesced.
#include "composite.h"

namespace tsi {

// Positive depths order like their bit patterns; misses sort after every hit.
__device__ __forceinline__ unsigned long long part_key(float d, uint32_t id) {
  const uint32_t hi = (d >= 0.0f) ? (__float_as_uint(d) & 0x7fffffffu) : 0x7fffffffu;
  return ((unsigned long long)hi << 32) | id;
}

__global__ void __launch_bounds__(256) composite_kernel(const CompositeParts P, uint64_t npix,
                                                        float4 *__restrict__ rgba, float *__restrict__ depth,
                                                        float *__restrict__ normal,
                                                        unsigned long long *__restrict__ key) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
       i += (uint64_t)gridDim.x * blockDim.x) {
    unsigned long long best = ~0ull;
    uint32_t win = 0;
    for (uint32_t s = 0; s < P.n; ++s) {
      const unsigned long long k = part_key(__ldg(P.depth[s] + i), P.id[s]);
      if (k < best) {
        best = k;
        win = s;
      }
    }
    depth[i] = P.depth[win][i];
    rgba[i] = P.rgba[win][i];
    const float *n = P.normal[win] + 3 * i;
    normal[3 * i + 0] = n[0];
    normal[3 * i + 1] = n[1];
    normal[3 * i + 2] = n[2];
    key[i] = best;
  }
}

__global__ void __launch_bounds__(256) keep_nearest_kernel(const unsigned long long *__restrict__ key,
                                                           const unsigned long long *__restrict__ global_key,
                                                           uint64_t npix, float4 *__restrict__ rgba,
                                                           float *__restrict__ depth, float *__restrict__ normal) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (key[i] != global_key[i]) {
      rgba[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      depth[i] = 0.0f;
      normal[3 * i + 0] = 0.0f;
      normal[3 * i + 1] = 0.0f;
      normal[3 * i + 2] = 0.0f;
    }
  }
}

namespace {
int grid_for(uint64_t npix, int grid) {
  const uint64_t need = (npix + 255) / 256;
  return (int)(need < (uint64_t)grid ? (need ? need : 1) : (uint64_t)grid);
}
}  // namespace

cudaError_t launch_composite(const CompositeParts &parts, uint64_t npix, float4 *rgba, float *depth,
                             float *normal, unsigned long long *key, int grid, cudaStream_t st) {
  if (npix == 0) return cudaSuccess;
  composite_kernel<<<grid_for(npix, grid), 256, 0, st>>>(parts, npix, rgba, depth, normal, key);
  return cudaGetLastError();
}

cudaError_t launch_keep_nearest(const unsigned long long *key, const unsigned long long *global_key, uint64_t npix,
                                float4 *rgba, float *depth, float *normal, int grid, cudaStream_t st) {
  if (npix == 0) return cudaSuccess;
  keep_nearest_kernel<<<grid_for(npix, grid), 256, 0, st>>>(key, global_key, npix, rgba, depth, normal);
  return cudaGetLastError();
}

}  // namespace tsi
