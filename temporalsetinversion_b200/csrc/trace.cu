// trace.cu — octree ray tracer, one thread per pixel (compute.wgsl `rt_main`
// 4650-4688 with `cinematic` off, `trace` 4189-4403).
//
// Each pixel walks the octree top-down (trace_walk.cuh) and is shaded by the
// age colour of the leaf it hits.  The cinematic path tracer is in
// cinematic.cu.  This file is compiled with --fmad=false so that the
// arithmetic is the plain f32 sequence of the reference (no FMA
// contraction).
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "device_types.h"
#include "fmath.cuh"
#include "interp.cuh"
#include "trace_params.h"
#include "trace_walk.cuh"

namespace tsi {

// FAST: normals by finite differences of the tape (a separate instance, so
// the plain tracer carries no point-evaluation code).
template <bool FAST>
__global__ void __launch_bounds__(256, 4) trace_kernel(const TraceParams *__restrict__ Tp) {
  const TraceParams &T = *Tp;
  // a block covers a 32x8 pixel tile and each warp a 4x8 column of it, so
  // the rays of a warp are close together and walk similar nodes (8x4 and
  // 8x8-per-two-warps tiles measured 1-2% slower on the benchmark frames)
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * 32u + warp * 4u + (lane & 3u);
  const uint32_t py = blockIdx.y * 8u + (lane >> 2);
  const bool valid = px < T.W && py < T.H;
  const uint64_t pix = (uint64_t)py * T.W + px;
  // ray_direction (4590-4594) and the view transform (4629-4631)
  const F3 rd = primary_dir(T, (float)px, (float)py - T.yshift);
  const F3 ro = f3(T.eye[0], T.eye[1], T.eye[2]);
  const F3 inv = rcp3(rd);  // the slab tests' reciprocal direction, once per ray

  Walk w;
  w.c = f3(1.0f, 1.0f, 1.0f);
  w.nrm = f3(0.0f, 0.0f, 0.0f);
  w.end = ro;
  w.since = 0.0f;
  w.tnorm = T.time;
  w.hit = false;
  w.visits = 0;
  if (valid && T.rendermode == 0.0f) walk_octree<true>(T, ro, rd, inv, w);
  if (FAST) {  // fast normals (compute.wgsl:4337-4342)
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (__any_sync(0xffffffffu, w.hit)) {
      const F3 n = tape_normal(T, tid & 31u, tid >> 5, w.end, w.tnorm);
      if (w.hit) w.nrm = n;
    }
  }
  F3 c = w.c;
  float dist = -1.0f;
  if (valid && T.rendermode == 0.0f) shade_walk(T, w, ro, c, dist);
  const bool intersected = w.hit;
  const F3 nrm = w.nrm;
  const uint32_t visits = w.visits;
  // get_color_single / get_color_supersample, non-cinematic (4444-4516, 4620-4648)
  float cr = c.x, cg = c.y, cb = c.z, ca = 1.0f;
  if (T.rendermode != 0.0f) {
    cr = cg = cb = ca = 0.0f;
  } else if (T.normal_viz && !intersected) {
    cr = cg = cb = 10.0f;
    ca = 0.0f;
  }
  if (valid && T.rgba) T.rgba[pix] = make_float4(fm_powf(cr, 0.45f), fm_powf(cg, 0.45f), fm_powf(cb, 0.45f), ca);
  if (valid && T.depth) T.depth[pix] = dist;
  if (valid && T.normal) {
    T.normal[pix * 3 + 0] = nrm.x;
    T.normal[pix * 3 + 1] = nrm.y;
    T.normal[pix * 3 + 2] = nrm.z;
  }
  if (T.visits) {
    // one atomic per warp
    unsigned long long v = visits;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0) atomicAdd(T.visits, v);
  }
}

// Shared memory of one block with fast normals: 8 warps' register files.
size_t trace_smem_bytes(const TraceParams &T) { return T.code ? (size_t)8 * T.nregs * 32 * sizeof(float2) : 0; }

cudaError_t launch_cinematic(const TraceParams &T, const TraceParams *Tdev, size_t smem, cudaStream_t st);

cudaError_t launch_trace(const TraceParams &T, const TraceParams *Tdev, cudaStream_t st) {
  const size_t smem = trace_smem_bytes(T);
  if (T.cinematic) return launch_cinematic(T, Tdev, smem, st);
  if (smem > (48u << 10)) {  // the attribute is per kernel and device: only ever raise it
    static std::mutex mu;
    static size_t set_bytes[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64 || smem > set_bytes[dev]) {
      e = cudaFuncSetAttribute(trace_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) set_bytes[dev] = smem;
    }
  }
  dim3 block(256);
  dim3 grid((T.W + 31) / 32, (T.H + 7) / 8);
  if (T.code) trace_kernel<true><<<grid, block, smem, st>>>(Tdev);
  else trace_kernel<false><<<grid, block, 0, st>>>(Tdev);
  return cudaGetLastError();
}

}  // namespace tsi
