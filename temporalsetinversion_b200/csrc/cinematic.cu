// cinematic.cu — path tracing of the octree (compute.wgsl `rt_main` with
// `cinematic` on, 3499).
//
// Per pixel, `samples` jittered primary rays (get_color_supersample
// 4620-4648), each a two-bounce path (get_color_single 4444-4523): at a hit
// the path continues in a cosine-power lobe around the normal
// (getSampleBiased 4429-4438) with its luminance scaled by the surface
// colour; a shadow ray towards a jittered sun direction adds sun light and
// a specular highlight when it escapes the octree; a path that escapes sees
// the sky model (sunsky 520-677), a primary miss sees white unless
// see_background.  The random numbers are the PCG hash of frand / frand0to1
// (2451-2472) on rt_main's per-pixel seed (4664), drawn in the reference's
// order, so every pixel is deterministic.  The walks are trace_walk.cuh's,
// the elementary functions fmath.cuh's (sin, cos, exp, acos, pow), so the
// image equals the CPU oracle's bit for bit.
//
// One thread per pixel; the bounce loop is uniform across the warp (lanes
// whose path ended idle), so finite-difference normals are evaluated by the
// whole warp as in trace.cu.  Depth and normal outputs are those of the
// first sample's primary ray.  Compiled with --fmad=false.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "trace_walk.cuh"

namespace tsi {

namespace {

__device__ __forceinline__ uint32_t pcg_word(uint32_t s) {
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
__device__ __forceinline__ float frand(uint32_t &seed) {  // -1 to 1
  seed = seed * 747796405u + 1u;
  return __fsub_rn(__fmul_rn(__fdiv_rn(__uint2float_rn(pcg_word(seed)), 4294967295.0f), 2.0f), 1.0f);
}
__device__ __forceinline__ float frand0to1(uint32_t &seed) {
  seed = seed * 747796405u + 1u;
  return __fdiv_rn(__uint2float_rn(pcg_word(seed)), 4294967295.0f);
}

__device__ __forceinline__ float dot3(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ F3 normalize3(F3 a) {
  const float l = len3(a);
  return f3(a.x / l, a.y / l, a.z / l);
}
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fm_min(fm_max(x, lo), hi); }
__device__ __forceinline__ F3 pow3(F3 a, F3 b) { return f3(fm_powf(a.x, b.x), fm_powf(a.y, b.y), fm_powf(a.z, b.z)); }

__device__ __forceinline__ F3 from_spherical(float px, float py) {  // 497-518
  return f3(fm_cos(px) * fm_sin(py), fm_sin(px) * fm_sin(py), fm_cos(py));
}

__device__ __forceinline__ F3 ortho(F3 v) {  // 4405-4427
  if (fabsf(v.x) > fabsf(v.z)) return f3(-v.y, v.x, 0.0f);
  return f3(0.0f, -v.z, v.y);
}

__device__ F3 sample_biased(F3 d, float power, uint32_t &seed) {  // getSampleBiased 4429-4438
  const F3 dir = normalize3(d);
  const F3 o1 = normalize3(ortho(dir));
  const F3 o2 = normalize3(cross3(dir, o1));
  float rx = frand0to1(seed);
  float ry = frand0to1(seed);
  rx = (rx * 2.0f) * 3.1415927410125732f;
  ry = fm_powf(ry, 1.0f / (power + 1.0f));
  const float oneminus = sqrtf(1.0f - ry * ry);
  return (muls(o1, fm_cos(rx) * oneminus) + muls(o2, fm_sin(rx) * oneminus)) + muls(dir, ry);
}

// sunsky (520-677) with turbidity 1, sunSize 1 and the sky's sun intensity
// 1000 (the private globals of 421-427); it returns 0.01 * sky.  pow with the
// constant exponent 2.0 is x * x, the rewrite shader compilers apply; it is
// defined for the negative cosines between view and sun.
__device__ F3 sunsky(F3 view, float spx, float spy) {
  const float pi = 3.1415927410125732f;
  const float sun_cos = fm_cos((1.0f * pi) / 180.0f);
  const F3 sun_dir = normalize3(from_spherical((spx - 0.0f) * 6.28000020980835f, (spy - 0.5f) * 3.140000104904175f));
  const float cos_view_sun = dot3(view, sun_dir);
  const float cos_sun_up = dot3(sun_dir, f3(0.0f, 0.0f, 1.0f));
  const float cos_up_view = dot3(f3(0.0f, 0.0f, 1.0f), view);
  if (sun_cos == 1.0f) return f3(1.0f, 0.0f, 0.0f);
  const float sunE = 1000.0f * fm_max(0.0f, 1.0f - fm_exp(-((1.6110731611233942f - fm_acos(cos_sun_up)) / 1.5f)));
  const F3 rayleigh = f3(5.176821105123963e-6f, 1.2785348189936485e-5f, 2.8530756026157178e-5f);
  const float c = (0.20000000298023224f * 1.0f) * 9.99999983775159e-18f;  // totalMie 438-456, T = 1
  const F3 lambda = f3(6.800000278417428e-7f, 5.499999815583578e-7f, 4.4999998749517545e-7f);
  const F3 K = f3(0.6859999895095825f, 0.6779999732971191f, 0.6660000085830688f);
  const float two_pi = 2.0f * 3.1415927410125732f;
  const F3 q = f3(two_pi, two_pi, two_pi) / lambda;  // pow(q, vec3(4.0 - 2.0)) = q * q
  const F3 tm = muls(q * q, (0.4339999854564667f * c) * 3.1415927410125732f) * K;
  const F3 mie = muls(tm, 0.004999999888241291f);
  const float zenith = fm_max(0.0f, cos_up_view);
  const float r_len = 8400.0f / zenith, m_len = 1250.0f / zenith;
  const F3 fex = f3(fm_exp(-(rayleigh.x * r_len + mie.x * m_len)), fm_exp(-(rayleigh.y * r_len + mie.y * m_len)),
                    fm_exp(-(rayleigh.z * r_len + mie.z * m_len)));
  const float rphase = (3.0f / (16.0f * 3.1415927410125732f)) * (1.0f + (cos_view_sun * cos_view_sun));  // 429-436
  const float g = 0.800000011920929f;  // hgPhase 458-480
  const float hg = (1.0f / (4.0f * 3.1415927410125732f)) *
                   ((1.0f - (g * g)) / fm_powf((1.0f - (2.0f * g) * cos_view_sun) + (g * g), 1.5f));
  const F3 r_eye = muls(rayleigh, rphase), m_eye = muls(mie, hg);
  const F3 total = rayleigh + mie, light = r_eye + m_eye;
  const F3 se = muls(light / total, sunE);
  F3 sky = se * (f3(1.0f, 1.0f, 1.0f) - fex);
  const float t = clampf(fm_powf(1.0f - dot3(f3(0.0f, 0.0f, 1.0f), sun_dir), 5.0f), 0.0f, 1.0f);
  const F3 pw = pow3(se * fex, f3(0.5f, 0.5f, 0.5f));
  const F3 mx = f3(1.0f * (1.0f - t) + pw.x * t, 1.0f * (1.0f - t) + pw.y * t, 1.0f * (1.0f - t) + pw.z * t);
  sky = sky * mx;
  return muls(sky, 0.009999999776482582f);
}

__device__ __forceinline__ float linear_to_srgb(float x) {  // LinearToSRGB 4600-4607, one channel
  const float rgb = clampf(x, 0.0f, 1.0f);
  const float m = (rgb < 0.0031308f) ? 1.0f : 0.0f;
  const float a = fm_powf(rgb, 1.0f / 2.4f) * 1.055f - 0.055f;
  const float b = rgb * 12.92f;
  return a * (1.0f - m) + b * m;
}

struct Sun {
  float spx, spy, intensity, specular, albedo, size, bg;
};

__device__ __forceinline__ Sun scene_sun(int32_t scene) {  // 4449-4471
  Sun s{-0.1f, 0.7f, 3.0f, 1.0f, 1.0f, 0.01f, 1.0f};
  if (scene == 3) {
    s.spx = 0.36f;
    s.spy = 0.72f;
    s.specular = 1.0f;
    s.size = 0.1f;
    s.albedo = 1.5f;
    s.bg = 2.0f;
    s.intensity = 2.0f;
  } else if (scene == 4) {
    s.spx = -0.1f;
    s.spy = 0.57f;
    s.size = 0.01f;
  } else if (scene == 5) {
    s.spx = 0.63f;
    s.spy = 0.65f;
    s.size = 0.02f;
  }
  return s;
}

}  // namespace

template <bool FAST>
__global__ void __launch_bounds__(256, 2) cinematic_kernel(const TraceParams *__restrict__ Tp) {
  const TraceParams &T = *Tp;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * 32u + (warp & 3u) * 8u + (lane & 7u);
  const uint32_t py = blockIdx.y * 8u + (warp >> 2) * 4u + (lane >> 3);
  const bool valid = px < T.W && py < T.H;
  const uint64_t pix = (uint64_t)py * T.W + px;
  const F3 eye = f3(T.eye[0], T.eye[1], T.eye[2]);
  const Sun sun = scene_sun(T.scene_id);
  // seed3 of rt_main (4664)
  uint32_t seed = (uint32_t)pix + (uint32_t)(12345.0f * (fm_sin(T.time * 12345.0f) * 0.5f + 0.5f));
  float acc_r = 0.0f, acc_g = 0.0f, acc_b = 0.0f, acc_a = 0.0f, d0 = -1.0f;
  F3 n0 = f3(0.0f, 0.0f, 0.0f);
  for (uint32_t smp = 0; smp < T.samples; ++smp) {
    const float ox = frand(seed), oy = frand(seed);
    const float pxf = (float)px + (ox * 1.0f) * 0.5f;
    const float pyf = ((float)py - T.yshift) + (oy * 1.0f) * 0.5f;
    if (T.rendermode != 0.0f) continue;  // uniform
    // get_color_single (4444-4523), cinematic
    F3 frm = eye, dir = primary_dir(T, pxf, pyf);
    F3 lum = f3(1.0f, 1.0f, 1.0f), direct = f3(0.0f, 0.0f, 0.0f);
    float out_r = 0.0f, out_g = 0.0f, out_b = 0.0f, out_a = 0.0f;
    bool active = valid, ended = false;
    for (int i = 0; i < 2; ++i) {
      Walk w;
      w.c = f3(1.0f, 1.0f, 1.0f);
      w.nrm = f3(0.0f, 0.0f, 0.0f);
      w.end = frm;
      w.since = 0.0f;
      w.tnorm = T.time;
      w.hit = false;
      w.visits = 0;
      if (active) walk_octree<true>(T, frm, dir, rcp3(dir), w);
      if (FAST) {
        if (__any_sync(0xffffffffu, active && w.hit)) {
          const F3 n = tape_normal(T, lane, warp, w.end, w.tnorm);
          if (active && w.hit) w.nrm = n;
        }
      }
      if (!active) continue;
      F3 sc;
      float dist;
      shade_walk(T, w, frm, sc, dist);
      if (i == 0 && smp == 0) {
        d0 = dist;
        n0 = w.nrm;
      }
      const F3 n = w.nrm;
      const F3 hitpoint = frm + muls(dir, dist);
      if (dist >= 0.0f) {
        const F3 old = dir;
        dir = sample_biased(n, 3.0f, seed);
        lum = muls(lum * sc, sun.albedo);
        frm = hitpoint + muls(n, 0.05f);
        const F3 sd = normalize3(from_spherical((sun.spx - 0.0f) * 6.28f, (sun.spy - 0.5f) * 3.14f));
        const F3 sundir = f3(sd.x, sd.z, sd.y);
        const float jx = frand(seed), jy = frand(seed), jz = frand(seed);
        const F3 sample_dir = normalize3(sundir + muls(f3(jx, jy, jz), sun.size));
        const float sunlight = dot3(n, sample_dir);
        Walk sh;
        sh.hit = false;
        walk_octree<false>(T, frm, sample_dir, rcp3(sample_dir), sh);
        if (sunlight > 0.0f && !sh.hit) {  // facing the sun and not in shadow
          direct = direct + muls(muls(lum, sunlight), sun.intensity);
          const F3 half = normalize3(f3(-old.x, -old.y, -old.z) + sundir);
          const float spec = (100.0f * fm_powf(fm_max(dot3(n, half), 0.0f), 30.0f)) * sun.specular;
          direct = direct + muls(lum, spec);
        }
      } else {
        if (i == 0 && !T.see_background) {
          out_r = out_g = out_b = 10.0f;
          out_a = 0.0f;
        } else {
          const F3 sky = sunsky(f3(dir.x, dir.z, dir.y), sun.spx, sun.spy);  // getBackground 4440-4442
          const F3 cc = direct + lum * sky;
          out_r = cc.x * sun.bg;
          out_g = cc.y * sun.bg;
          out_b = cc.z * sun.bg;
          out_a = 1.0f * sun.bg;
        }
        ended = true;
        active = false;
      }
    }
    if (!ended) {
      out_r = direct.x;
      out_g = direct.y;
      out_b = direct.z;
      out_a = 1.0f;
    }
    acc_r = acc_r + out_r;
    acc_g = acc_g + out_g;
    acc_b = acc_b + out_b;
    acc_a = acc_a + out_a;
  }
  const float fs = (float)T.samples;
  const float cr = linear_to_srgb(acc_r / fs), cg = linear_to_srgb(acc_g / fs), cb = linear_to_srgb(acc_b / fs);
  const float ca = acc_a / fs;
  if (valid && T.rgba) T.rgba[pix] = make_float4(fm_powf(cr, 0.45f), fm_powf(cg, 0.45f), fm_powf(cb, 0.45f), ca);
  if (valid && T.depth) T.depth[pix] = d0;
  if (valid && T.normal) {
    T.normal[pix * 3 + 0] = n0.x;
    T.normal[pix * 3 + 1] = n0.y;
    T.normal[pix * 3 + 2] = n0.z;
  }
}

cudaError_t launch_cinematic(const TraceParams &T, const TraceParams *Tdev, size_t smem, cudaStream_t st) {
  if (smem > (48u << 10)) {  // the attribute is per kernel and device: only ever raise it
    static std::mutex mu;
    static size_t set_bytes[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64 || smem > set_bytes[dev]) {
      e = cudaFuncSetAttribute(cinematic_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) set_bytes[dev] = smem;
    }
  }
  dim3 block(256);
  dim3 grid((T.W + 31) / 32, (T.H + 7) / 8);
  if (T.code) cinematic_kernel<true><<<grid, block, smem, st>>>(Tdev);
  else cinematic_kernel<false><<<grid, block, 0, st>>>(Tdev);
  return cudaGetLastError();
}

}  // namespace tsi
