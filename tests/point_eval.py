"""Float64 point evaluation of a tape in the ir.rs 32-byte layout, for the
rigour tests of the directed-rounding mode: the value of f(x, y, z, t) that
the tape's instructions define, evaluated at many points at once with
numpy.  Operand order and op_top follow ir.rs:141-171; ATAN2 takes its
operands swapped (compute.wgsl:2724: ATAN2_II(x = larg, y = rarg), so the
value is atan2(rarg, larg)), MOD is floor-mod (2819)."""
from __future__ import annotations

import numpy as np

ADD, SUB, MUL, DIV, EXP, LOG, SQR, SQRT, POW, SIN, COS, NEG, MIN, MAX, ABS = 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19
FLOOR, RET, MOD, ATAN2 = 25, 28, 29, 30


def evaluate(tape: np.ndarray, x, y, z, t) -> np.ndarray:
    """f at the points (x, y, z, t) (broadcast arrays), float64."""
    x, y, z, t = np.broadcast_arrays(*(np.asarray(v, dtype=np.float64) for v in (x, y, z, t)))
    vals = [x, y, z, t]
    with np.errstate(all="ignore"):
        for j in range(4, len(tape)):
            ou = int(tape[j]["opcode_uses"])
            op, top = (ou >> 16) & 0x3FFF, ou >> 30
            lr = int(tape[j]["larg_rarg"])
            lit = np.float64(np.float32(tape[j]["literal"]))
            a = vals[lr >> 16] if top in (0, 1) else lit
            b = vals[lr & 0xFFFF] if top in (0, 2) else lit
            if top == 2 and op not in (SUB, DIV):
                raise ValueError("literal-left op %d has no value (compute.wgsl:3760)" % op)
            if op == ADD: v = a + b
            elif op == SUB: v = a - b
            elif op == MUL: v = a * b
            elif op == DIV: v = a / b
            elif op == EXP: v = np.exp(a)
            elif op == LOG: v = np.log(a)
            elif op == SQR: v = a * a
            elif op == SQRT: v = np.sqrt(a)
            elif op == POW: v = np.power(a, b)
            elif op == SIN: v = np.sin(a)
            elif op == COS: v = np.cos(a)
            elif op == NEG: v = -a
            elif op == MIN: v = np.minimum(a, b)
            elif op == MAX: v = np.maximum(a, b)
            elif op == ABS: v = np.abs(a)
            elif op == FLOOR: v = np.floor(a)
            elif op == RET: v = a
            elif op == MOD: v = a - b * np.floor(a / b)
            elif op == ATAN2: v = np.arctan2(b, a)  # ATAN2_II(x = larg, y = rarg): atan2(rarg, larg)
            else:
                raise ValueError("opcode %d not handled by the point evaluator" % op)
            vals.append(np.broadcast_to(v, x.shape).astype(np.float64))
    return vals[-1]
