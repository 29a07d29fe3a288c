// composite.h — nearest-depth composite of the frames of one animation's
// subtrees (kernels in composite.cu, called by the C ABI in api.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tsi.h"

namespace tsi {

// Kernel parameter block: the parts' frames and their subtree indices.
struct CompositeParts {
  const float4 *rgba[TSI_COMPOSITE_MAX];
  const float *depth[TSI_COMPOSITE_MAX];
  const float *normal[TSI_COMPOSITE_MAX];
  uint32_t id[TSI_COMPOSITE_MAX];
  uint32_t n;
};

// Writes out's rgba/depth/normal/key for npix pixels from the part with the
// least key per pixel.
cudaError_t launch_composite(const CompositeParts &parts, uint64_t npix, float4 *rgba, float *depth,
                             float *normal, unsigned long long *key, int grid, cudaStream_t st);
// Zeroes the pixels whose key differs from global_key.
cudaError_t launch_keep_nearest(const unsigned long long *key, const unsigned long long *global_key, uint64_t npix,
                                float4 *rgba, float *depth, float *normal, int grid, cudaStream_t st);

}  // namespace tsi
