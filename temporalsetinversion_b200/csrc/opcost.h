// opcost.h — algorithmic FP32 operation counts per interval instruction.
//
// One table read by the kernels' counters and by bench.py's roofline: the
// forward cost of each handler (compute.wgsl:2539-2975 op by op: adds,
// multiplies, min/max and compares of the interval formula), plus 4 for the
// `fix` clamp applied after every op (3768).  A reverse step costs the
// reverse rule (2806-2918) plus, per register operand, one MUL_II (10), one
// ADD_II (2) and one fix (4) (3871-3874, 3922-3930).  Transcendentals count
// as the f32 ops of their evaluation in this library's math (range
// reduction and polynomial).
#pragma once
#include "tape_format.h"

#define TSI_FIX_COST 4u
#define TSI_REV_OPERAND_COST 16u

// forward cost, indexed by tsi_handler
#define TSI_OPCOST_FWD_INIT                                                                   \
  {                                                                                           \
    /* CONST */ 0, /* COPY */ 0,                                                               \
    /* ADD_II */ 2, /* SUB_II */ 2, /* MUL_II */ 10, /* DIV_II */ 10, /* MIN_II */ 2,          \
    /* MAX_II */ 2, /* POW_II */ 24, /* MOD_II */ 18, /* ATAN2_II */ 40, /* BAD_II */ 0,       \
    /* ADD_IF */ 2, /* SUB_IF */ 2, /* MUL_IF */ 3, /* DIV_IF */ 10, /* MIN_IF */ 2,           \
    /* MAX_IF */ 2, /* POW_IF */ 24, /* MOD_IF */ 18, /* ATAN2_IF */ 40,                       \
    /* SQR */ 6, /* SQRT */ 4, /* EXP */ 4, /* LOG */ 4, /* NEG */ 0, /* ABS */ 4,             \
    /* FLOOR */ 2, /* SIN */ 20, /* COS */ 20, /* BAD_I */ 0,                                  \
    /* SUB_FI */ 2, /* DIV_FI */ 10, /* BAD_FI */ 0                                            \
  }

// reverse-rule cost, indexed by tsi_handler
#define TSI_OPCOST_RR_INIT                                                                    \
  {                                                                                           \
    /* CONST */ 0, /* COPY */ 0,                                                               \
    /* ADD_II */ 0, /* SUB_II */ 0, /* MUL_II */ 0, /* DIV_II */ 26, /* MIN_II */ 2,           \
    /* MAX_II */ 2, /* POW_II */ 60, /* MOD_II */ 0, /* ATAN2_II */ 40, /* BAD_II */ 0,        \
    /* ADD_IF */ 0, /* SUB_IF */ 0, /* MUL_IF */ 0, /* DIV_IF */ 10, /* MIN_IF */ 2,           \
    /* MAX_IF */ 2, /* POW_IF */ 30, /* MOD_IF */ 0, /* ATAN2_IF */ 20,                        \
    /* SQR */ 3, /* SQRT */ 18, /* EXP */ 4, /* LOG */ 10, /* NEG */ 0, /* ABS */ 2,           \
    /* FLOOR */ 2, /* SIN */ 20, /* COS */ 20, /* BAD_I */ 0,                                  \
    /* SUB_FI */ 0, /* DIV_FI */ 16, /* BAD_FI */ 0                                            \
  }

// register operands per handler (reverse accumulations)
#define TSI_H_NREG(h) (TSI_H_IS_II(h) ? 2u : ((h) == H_CONST ? 0u : 1u))
