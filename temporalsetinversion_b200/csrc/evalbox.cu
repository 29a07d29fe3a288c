// evalbox.cu — interval evaluation of one tape on a list of space-time boxes.
//
// The body of compute.wgsl:3632-3970 without the octree: forward tape,
// reverse interval AD seeded with 1 at the output, sensitivities of the four
// arguments.  One thread per box, registers and the operand log in global
// scratch.  Used by tsi_tape_eval_boxes (op-level parity tests).
#include <cuda_runtime.h>
#include <stdint.h>

#include "interval.cuh"

namespace tsi {

template <bool D>
__global__ void evalbox_kernel(const uint2 *code, uint32_t len, uint32_t nregs, uint32_t out_reg, uint32_t n,
                               const float *boxes, int reverse, float *out, float2 *regs, float4 *log) {
  using A = IA<D>;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float2 *R = regs + (size_t)i * nregs;
  float4 *L = log + (size_t)i * len;
  const float *b = boxes + (size_t)i * 8;
  for (int q = 0; q < 4; ++q) R[q] = make_float2(b[2 * q], b[2 * q + 1]);
  for (uint32_t j = 0; j < len; ++j) {
    const uint2 w = code[j];
    const uint32_t h = TSI_W0_H(w.x);
    const float lit = __uint_as_float(w.y);
    const float2 a = R[TSI_W0_A(w.x)];
    const Iv Av = Iv{a.x, a.y};
    Iv Bv = iv(lit);
    if (TSI_H_IS_II(h)) {
      const float2 bb = R[w.y & 255u];
      Bv = Iv{bb.x, bb.y};
    }
    L[j] = make_float4(Av.lo, Av.hi, Bv.lo, Bv.hi);
    const Iv r = A::forward(h, Av, Bv, lit);
    R[TSI_W0_DST(w.x)] = make_float2(r.lo, r.hi);
  }
  float *o = out + (size_t)i * 10;
  const float2 f = R[out_reg];
  o[0] = f.x;
  o[1] = f.y;
  for (int q = 2; q < 10; ++q) o[q] = 0.0f;
  if (!reverse) return;
  for (uint32_t r = 0; r < nregs; ++r) R[r] = make_float2(0.0f, 0.0f);
  R[out_reg] = make_float2(1.0f, 1.0f);
  for (int j = (int)len - 1; j >= 0; --j) {
    const uint2 w = code[j];
    const uint32_t h = TSI_W0_H(w.x);
    const uint32_t d = TSI_W0_DST(w.x), a = TSI_W0_A(w.x), bq = w.y & 255u;
    const float lit = __uint_as_float(w.y);
    const float4 lg = L[j];
    const Iv Av = Iv{lg.x, lg.y}, Bv = Iv{lg.z, lg.w};
    const float2 sv = R[d];
    const Iv s = Iv{sv.x, sv.y};
    R[d] = make_float2(0.0f, 0.0f);
    if (h == H_CONST) continue;
    const bool s0 = (s.lo == 0.0f && s.hi == 0.0f);
    if (TSI_H_IS_II(h)) {
      if (s0 && TSI_W0_FA(w.x) && TSI_W0_FB(w.x)) {
        R[a] = make_float2(0.0f, 0.0f);
        R[bq] = make_float2(0.0f, 0.0f);
      } else {
        Iv r0, r1;
        A::reverse_rule(h, Av, Bv, lit, r0, r1);
        r0 = A::mul(A::fix(r0), s);
        r1 = A::mul(A::fix(r1), s);
        const float2 pa = R[a], pb = R[bq];
        const Iv n0 = A::add(r0, Iv{pa.x, pa.y});
        const Iv n1 = A::add(r1, Iv{pb.x, pb.y});
        R[a] = make_float2(n0.lo, n0.hi);
        R[bq] = make_float2(n1.lo, n1.hi);
      }
    } else {
      if (s0 && TSI_W0_FA(w.x)) {
        R[a] = make_float2(0.0f, 0.0f);
      } else {
        Iv r0, r1;
        A::reverse_rule(h, Av, Bv, lit, r0, r1);
        r0 = A::mul(A::fix(r0), s);
        const float2 pa = R[a];
        const Iv n0 = A::add(r0, Iv{pa.x, pa.y});
        R[a] = make_float2(n0.lo, n0.hi);
      }
    }
  }
  for (int q = 0; q < 4; ++q) {
    o[2 + 2 * q] = R[q].x;
    o[3 + 2 * q] = R[q].y;
  }
}

// elementwise checks of the f32 math and min/max (GPU math tests)
__global__ void math_kernel(int which, uint32_t n, const float *a, const float *b, float *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float r;
  switch (which) {
    case 0: r = fm_sin(a[i]); break;
    case 1: r = fm_exp(a[i]); break;
    case 2: r = fm_log(a[i]); break;
    case 3: r = fm_atan2(a[i], b[i]); break;
    case 4: r = fm_powi(a[i], (int)b[i]); break;
    case 5: r = fm_min(a[i], b[i]); break;
    case 6: r = fm_max(a[i], b[i]); break;
    case 7: r = fminf(a[i], b[i]); break;
    case 8: r = fmaxf(a[i], b[i]); break;
    default: r = 0.0f; break;
  }
  out[i] = r;
}

cudaError_t launch_evalbox(bool directed, const uint2 *code, uint32_t len, uint32_t nregs, uint32_t out_reg,
                           uint32_t n, const float *boxes, int reverse, float *out, float2 *regs, float4 *log,
                           cudaStream_t st) {
  const int block = 128;
  const int grid = (int)((n + block - 1) / block);
  if (directed)
    evalbox_kernel<true><<<grid, block, 0, st>>>(code, len, nregs, out_reg, n, boxes, reverse, out, regs, log);
  else
    evalbox_kernel<false><<<grid, block, 0, st>>>(code, len, nregs, out_reg, n, boxes, reverse, out, regs, log);
  return cudaGetLastError();
}

// Loads both instances of the box kernel on the current device (module
// loading is lazy, so without this the first launch of each would load it).
cudaError_t evalbox_preload() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, evalbox_kernel<true>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, evalbox_kernel<false>);
  return e;
}

cudaError_t launch_math(int which, uint32_t n, const float *a, const float *b, float *out, cudaStream_t st) {
  math_kernel<<<(n + 255) / 256, 256, 0, st>>>(which, n, a, b, out);
  return cudaGetLastError();
}

}  // namespace tsi
