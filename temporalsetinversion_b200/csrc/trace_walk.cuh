// trace_walk.cuh — the octree walk of one ray (compute.wgsl `trace`
// 4189-4403, `efficient_slabs` 4059-4070), shared by the frame tracer
// (trace.cu, rt_main) and the cinematic path tracer (cinematic.cu).
//
// The walk follows the reference's state machine step for step: slab test
// of the current node, a 2x2x2 DDA over its children, descent into children
// with f <= 0 whose eps-padded box the ray hits, hit at the first leaf,
// including its handling of the DDA leaving the node and of out-of-range
// child indices, with a 32-entry stack instead of 16 so octrees deeper than
// 8 levels do not overflow.  Compiled with --fmad=false: the arithmetic is
// the plain f32 sequence of the reference (no FMA contraction).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_types.h"
#include "fmath.cuh"
#include "interp.cuh"
#include "trace_params.h"

namespace tsi {

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3(float a, float b, float c) { return F3{a, b, c}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator*(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ F3 operator/(F3 a, F3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ F3 muls(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ F3 rcp3(F3 a) { return f3(1.0f / a.x, 1.0f / a.y, 1.0f / a.z); }
__device__ __forceinline__ float len3(F3 a) { return sqrtf((a.x * a.x + a.y * a.y) + a.z * a.z); }
__device__ __forceinline__ float sgn(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

__device__ __forceinline__ F3 slabs(F3 p0, F3 p1, F3 ro, F3 inv) {
  const F3 t0 = (p0 - ro) * inv, t1 = (p1 - ro) * inv;
  const float mnx = fm_min(t0.x, t1.x), mny = fm_min(t0.y, t1.y), mnz = fm_min(t0.z, t1.z);
  const float mxx = fm_max(t0.x, t1.x), mxy = fm_max(t0.y, t1.y), mxz = fm_max(t0.z, t1.z);
  const float d1 = fm_max(mnx, fm_max(mny, mnz));
  const float d2 = fm_min(mxx, fm_min(mxy, mxz));
  return f3((d1 <= d2 && d2 >= 0.0f) ? 1.0f : 0.0f, fm_max(d1, 0.0f), fm_max(d2, 0.0f));
}

__device__ __forceinline__ void node_box(const VoxelPoolDev &pool, uint32_t v, F3 &p0, F3 &p1) {
  const float4 a = pool.box_xy[v];
  const float2 b = pool.box_z[v];
  p0 = f3(a.x, a.z, b.x);
  p1 = f3(a.y, a.w, b.y);
}

// Dynamic shared memory of trace_kernel: with fast normals, one interval
// register file per warp for the point evaluations.
extern __shared__ __align__(16) unsigned char trace_smem[];

// finite_diff_normal (compute.wgsl:4143-4184) for any tape: the tetrahedron
// of points p + k h (h = 0.01, k in {(1,-1,-1), (-1,-1,1), (-1,1,-1),
// (1,1,1)}) with f evaluated by the tape on point boxes (round to nearest),
// normalised as v / |v|.  The reference pastes a per-scene function here;
// the tape makes it work for every scene.  Called by the whole warp; lanes
// without a hit evaluate a point too and discard it.
static __device__ __noinline__ F3 tape_normal(const TraceParams &T, uint32_t lane, uint32_t warp, F3 p, float t) {
  float2 *rf = reinterpret_cast<float2 *>(trace_smem) + (size_t)warp * T.nregs * 32u;
  const float h = 0.01f;
  const float kx[4] = {1.0f, -1.0f, -1.0f, 1.0f}, ky[4] = {-1.0f, -1.0f, 1.0f, 1.0f};
  const float kz[4] = {-1.0f, 1.0f, -1.0f, 1.0f};
  float f[4];
  for (int q = 0; q < 4; ++q) {
    const Iv r = forward_pass<false>(T.code, T.len, T.out_reg, rf, lane, iv(p.x + kx[q] * h), iv(p.y + ky[q] * h),
                                     iv(p.z + kz[q] * h), iv(t), nullptr, nullptr);
    f[q] = r.lo;
  }
  F3 v = f3(kx[0] * f[0], ky[0] * f[0], kz[0] * f[0]);
  for (int q = 1; q < 4; ++q) v = v + f3(kx[q] * f[q], ky[q] * f[q], kz[q] * f[q]);
  const float l = len3(v);
  return f3(v.x / l, v.y / l, v.z / l);
}

// What the walk of one ray leaves: the colour darkened along the way
// (COLOR), the leaf's stored normal, where the walk ended, the time since
// the leaf was evaluated and the time of its finite-difference normal.
struct Walk {
  F3 c, nrm, end;
  float since, tnorm;
  bool hit;
  uint32_t visits;
};

template <bool COLOR>
__device__ __forceinline__ void walk_octree(const TraceParams &T, F3 ro, F3 rd, F3 inv, Walk &w) {
  const VoxelPoolDev &pool = T.pool;
  const float TEPS = 0.0001f;
  F3 c = f3(1.0f, 1.0f, 1.0f);
  F3 nrm = f3(0.0f, 0.0f, 0.0f);
  uint32_t visits = 0;
  bool intersected = false;
  float hit_since = 0.0f;  // time since the leaf was evaluated
  float hit_t = T.time;    // time of the finite-difference normal
  uint32_t stack[32];
  uint32_t sp = 0;
  F3 ro2 = ro;
  stack[sp++] = 0u;
  uint32_t region = 0u;
  F3 p0, p1;
  node_box(pool, region, p0, p1);
  F3 hit = slabs(p0, p1, ro2, inv);
  bool done = (hit.x == 0.0f);
  for (uint32_t iter = 0; iter < 5000u && !done; ++iter) {
    if (intersected) break;
    if (sp == 0) {
      done = true;
      break;
    }
    region = stack[--sp];
    if (hit.x == 0.0f) {
      if (sp == 0) continue;
      node_box(pool, stack[sp - 1], p0, p1);
      hit = slabs(p0, p1, ro2, inv);
      continue;
    }
    const F3 two = f3(2.0f, 2.0f, 2.0f);
    const F3 rol = muls((ro2 + muls(rd, hit.y + TEPS)) - p0, 2.0f) / (p1 - p0);
    const F3 rdl = rd * (two / (p1 - p0));
    int mp0 = (int)floorf(rol.x), mp1 = (int)floorf(rol.y), mp2 = (int)floorf(rol.z);
    const float dd0 = 1.0f / fabsf(rdl.x), dd1 = 1.0f / fabsf(rdl.y), dd2 = 1.0f / fabsf(rdl.z);
    const float s0 = sgn(rdl.x), s1 = sgn(rdl.y), s2 = sgn(rdl.z);
    const int st0 = (int)s0, st1 = (int)s1, st2 = (int)s2;
    float sd0 = ((s0 * ((float)mp0 - rol.x) + s0 * 0.5f) + 0.5f) * dd0;
    float sd1 = ((s1 * ((float)mp1 - rol.y) + s1 * 0.5f) + 0.5f) * dd1;
    float sd2 = ((s2 * ((float)mp2 - rol.z) + s2 * 0.5f) + 0.5f) * dd2;
    float m0 = 0.0f, m1 = 0.0f, m2 = 0.0f;
    const F3 old_ro2 = ro2;
    // per node: the darkening of every DDA step and the children's brick
    const bool darken = !T.normal_viz && fm_max(p1.x - p0.x, fm_max(p1.y - p0.y, p1.z - p0.z)) < 1.0f;
    const uint32_t cbase = pool.child[region];
    // ro2 = old_ro2 + rd t after every step, as in the reference; it is
    // only read where a child is tested, where the walk leaves this node's
    // loop and at the end, so it is formed there (`moved`: not yet formed
    // for the last step)
    float t = 0.0f;
    bool moved = false;
    for (int i = 0; i < 32; ++i) {
      if (COLOR && darken) c = muls(c, T.darken);
      const F3 mv = f3(m0 * (sd0 - dd0), m1 * (sd1 - dd1), m2 * (sd2 - dd2));
      // the reference adds its sphere-march step here, which is always 0
      // (and t > 0 or NaN, so adding 0 changes no bit)
      t = (len3(mv) + hit.y) + TEPS;
      moved = true;
      if (t >= hit.z - TEPS) {  // left the node (4277-4292)
        ro2 = old_ro2 + muls(rd, hit.z);
        moved = false;
        if (sp == 0) {
          hit = f3(0.0f, 0.0f, 0.0f);
          break;
        }
        node_box(pool, stack[sp - 1], p0, p1);
        hit = slabs(p0, p1, ro2, inv);
        break;
      }
      const int ci = mp0 + 2 * mp1 + 4 * mp2;
      if (ci < 0 || ci >= 8) break;
      const uint32_t child = cbase + (uint32_t)ci;
      if (cbase != TSI_NONE) ++visits;
      if (cbase != TSI_NONE && pool.f[child] <= 0.0f) {
        ro2 = old_ro2 + muls(rd, t);
        moved = false;
        F3 q0, q1;
        node_box(pool, child, q0, q1);
        const F3 tp0 = f3(q0.x - TEPS, q0.y - TEPS, q0.z - TEPS);
        const F3 tp1 = f3(q1.x + TEPS, q1.y + TEPS, q1.z + TEPS);
        const F3 th = slabs(tp0, tp1, ro2, inv);
        if (th.x == 1.0f) {
          if (pool.child[child] != TSI_NONE) {
            if (sp < 32) stack[sp++] = region;
            if (sp < 32) stack[sp++] = child;
            p0 = tp0;
            p1 = tp1;
            hit = th;
            break;
          }
          // the leaf's colour is set after the walk (the fast normal is
          // evaluated by the whole warp there)
          intersected = true;
          const float4 nv = pool.normal[child];
          nrm = f3(nv.x, nv.y, nv.z);
          hit_since = T.time - pool.t[child];
          if (T.swept) hit_t = pool.t[region];  // compute.wgsl:4339-4341
          break;
        }
      }
      // 4389-4391
      const float n0 = (sd0 <= fm_min(sd1, sd2)) ? 1.0f : 0.0f;
      const float n1 = (sd1 <= fm_min(sd2, sd0)) ? 1.0f : 0.0f;
      const float n2 = (sd2 <= fm_min(sd0, sd1)) ? 1.0f : 0.0f;
      m0 = n0;
      m1 = n1;
      m2 = n2;
      sd0 = sd0 + m0 * dd0;
      sd1 = sd1 + m1 * dd1;
      sd2 = sd2 + m2 * dd2;
      mp0 = mp0 + (int)m0 * st0;
      mp1 = mp1 + (int)m1 * st1;
      mp2 = mp2 + (int)m2 * st2;
    }
    if (moved) ro2 = old_ro2 + muls(rd, t);
  }
  w.end = ro2;
  w.c = c;
  w.nrm = nrm;
  w.since = hit_since;
  w.tnorm = hit_t;
  w.hit = intersected;
  w.visits = visits;
}

// The colour of `trace` at the end of a walk from ro (4322-4401): the age
// colour of the leaf (or its normal, normal_viz) on the darkened colour,
// clamped; the hit distance |end - ro|, -1 for a miss.
__device__ __forceinline__ void shade_walk(const TraceParams &T, const Walk &w, F3 ro, F3 &c, float &dist) {
  c = w.c;
  dist = -1.0f;
  if (w.hit) {
    if (T.normal_viz) {
      const float nl = len3(w.nrm);
      c = f3(w.nrm.x / nl * 0.5f + 0.5f, w.nrm.y / nl * 0.5f + 0.5f, w.nrm.z / nl * 0.5f + 0.5f);
    } else {
      // c - mix(1 - movement, 1 - base, clamp(60 t, 0, 1)), movement (1,0,0), base (1,1,1)
      const float tt = fm_min(fm_max(w.since * 60.0f, 0.0f), 1.0f);
      const F3 a = f3(0.0f, 1.0f, 1.0f), b = f3(0.0f, 0.0f, 0.0f);
      const F3 lerp = f3(a.x * (1.0f - tt) + b.x * tt, a.y * (1.0f - tt) + b.y * tt, a.z * (1.0f - tt) + b.z * tt);
      c = c - lerp;
    }
    c = f3(fm_max(fm_min(c.x, 1.0f), 0.0f), fm_max(fm_min(c.y, 1.0f), 0.0f), fm_max(fm_min(c.z, 1.0f), 0.0f));
    dist = fabsf(len3(w.end - ro));
  } else {
    c = f3(fm_max(fm_min(c.x, 1.0f), 0.0f), fm_max(fm_min(c.y, 1.0f), 0.0f), fm_max(fm_min(c.z, 1.0f), 0.0f));
  }
}

// The primary ray through pixel position (pxf, pyf), pyf already shifted for
// scene 0 (ray_direction 4590-4594, the view transform 4629-4631).
__device__ __forceinline__ F3 primary_dir(const TraceParams &T, float pxf, float pyf) {
  float xy0 = (pxf - (float)T.W / 2.0f) + 0.5f;
  float xy1 = (pyf - (float)T.H / 2.0f) + 0.5f;
  F3 d = f3(xy0, -xy1, -T.zdist);
  const float dl = len3(d);
  d = f3(d.x / dl, d.y / dl, d.z / dl);
  F3 rd;
  rd.x = ((T.m[0] * d.x + T.m[4] * d.y) + T.m[8] * d.z) + T.m[12] * 0.0f;
  rd.y = ((T.m[1] * d.x + T.m[5] * d.y) + T.m[9] * d.z) + T.m[13] * 0.0f;
  rd.z = ((T.m[2] * d.x + T.m[6] * d.y) + T.m[10] * d.z) + T.m[14] * 0.0f;
  return rd;
}

}  // namespace tsi
