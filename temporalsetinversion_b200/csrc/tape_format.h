// tape_format.h — packed device tape shared by the host compiler and kernels.
//
// The reference keeps one 32-byte GPUInstruction per SSA slot and a
// per-thread copy of the whole tape in global memory (compute.wgsl:2989-3001,
// 3562, 3769-3771).  Here the tape is register allocated on the host and
// packed into 8 bytes per instruction:
//
//   w0  bits  0..5   handler (op x operand kind, table below)
//       bit   6      operand A is single-use  (ir.rs uses.len() == 1)
//       bit   7      operand B is single-use
//       bits  8..15  reserved
//       bits 16..23  destination register
//       bits 24..31  register A (larg, or rarg for the literal-left kinds)
//   w1  register B in bits 0..7 (two-register handlers) or the f32 literal
//
// The handler folds compute.wgsl's two-level switch (op_top at 3642, op at
// 3647/3714/3753) into one warp-uniform dispatch.  Unsupported (op, op_top)
// pairs keep the reference's behaviour (I_FROM(-inf), 3705/3745/3760).
#pragma once
#include <stdint.h>

#define TSI_MAX_REGS 256u
#define TSI_NONE 0xFFFFFFFFu

enum tsi_handler {
  H_CONST = 0,   // [lit, lit]; op_top 3 slots evaluate to [0,0] (compute.wgsl:3765)
  H_COPY = 1,    // RET (3696-3698) and pruned min/max
  H_ADD_II = 2, H_SUB_II = 3, H_MUL_II = 4, H_DIV_II = 5, H_MIN_II = 6, H_MAX_II = 7,
  H_POW_II = 8, H_MOD_II = 9, H_ATAN2_II = 10, H_BAD_II = 11,
  H_ADD_IF = 12, H_SUB_IF = 13, H_MUL_IF = 14, H_DIV_IF = 15, H_MIN_IF = 16, H_MAX_IF = 17,
  H_POW_IF = 18, H_MOD_IF = 19, H_ATAN2_IF = 20,
  H_SQR = 21, H_SQRT = 22, H_EXP = 23, H_LOG = 24, H_NEG = 25, H_ABS = 26, H_FLOOR = 27,
  H_SIN = 28, H_COS = 29, H_BAD_I = 30,
  H_SUB_FI = 31, H_DIV_FI = 32, H_BAD_FI = 33,
  H_COUNT = 34
};

#define TSI_W0(h, fa, fb, dst, a) \
  ((uint32_t)(h) | ((uint32_t)(fa) << 6) | ((uint32_t)(fb) << 7) | ((uint32_t)(dst) << 16) | ((uint32_t)(a) << 24))
#define TSI_W0_H(w) ((w) & 63u)
#define TSI_W0_FA(w) (((w) >> 6) & 1u)
#define TSI_W0_FB(w) (((w) >> 7) & 1u)
#define TSI_W0_DST(w) (((w) >> 16) & 255u)
#define TSI_W0_A(w) ((w) >> 24)

// Handler classes.
#define TSI_H_IS_II(h) ((h) >= H_ADD_II && (h) <= H_BAD_II)
#define TSI_H_IS_FI(h) ((h) >= H_SUB_FI && (h) <= H_BAD_FI)
#define TSI_H_HAS_A(h) ((h) != H_CONST)
// Handler field of a padding slot of the bundled (wide) tape: no operation.
#define TSI_H_PAD 63u
#define TSI_H_IS_MINMAX(h) ((h) == H_MIN_II || (h) == H_MAX_II || (h) == H_MIN_IF || (h) == H_MAX_IF)
