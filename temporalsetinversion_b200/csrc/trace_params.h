// trace_params.h — arguments of trace_kernel (compute.wgsl `rt_main`), shared
// by the host runtime that fills them and the kernel that reads them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_types.h"

namespace tsi {

struct TraceParams {
  float eye[3];
  float m[16];        // view matrix after the scene rotation, column major
  float zdist;        // res.y / tan(radians(fov) / 2)
  float yshift;       // scene 0 shift of the pixel row (compute.wgsl:4681-4683)
  uint32_t W, H;
  float time;
  float rendermode;
  uint32_t normal_viz;
  float darken;       // octree_darken_factor
  VoxelPoolDev pool;
  // fast normals: the scene's full tape, evaluated at points (nullptr: off)
  const uint2 *code;
  uint32_t len, nregs, out_reg;
  uint32_t swept;
  // cinematic path tracing (compute.wgsl:3499, 3506-3507): samples per
  // pixel, primary misses see the sky, the scene's sun and material
  uint32_t cinematic, samples, see_background;
  int32_t scene_id;
  float4 *rgba;
  float *depth;
  float *normal;      // 3 floats per pixel
  unsigned long long *visits;
};

// T: the host copy (grid size, variant); Tdev: the same in device memory, read by the kernel.
cudaError_t launch_trace(const TraceParams &T, const TraceParams *Tdev, cudaStream_t st);

}  // namespace tsi
