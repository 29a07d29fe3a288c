"""TEST INFRASTRUCTURE: pure-Python restatement of the reference's tape lowering.

Follows src/ir.rs:190-366 (parseLLVMIR, IR::new, Instruction::to_gpu) token by
token.  It exists only to check the library's C++ lowering
(temporalsetinversion_b200/csrc/ir_lower.cpp) from an independent
implementation; tests/ and the golden-fixture script import it, the product
never does.  Inputs on which ir.rs would panic raise ValueError here.
"""
from __future__ import annotations

import struct

OPCODES = [
    "NOP", "ARGX", "ARGY", "ARGZ", "ARGW", "ADD", "SUB", "MUL", "DIV", "EXP", "LOG", "SQR",
    "SQRT", "POW", "SIN", "COS", "NEG", "MIN", "MAX", "ABS", "CUP", "CAP", "BR", "PHI",
    "TRUNC", "FLOOR", "CEIL", "SIGN", "RET", "MOD", "ATAN2",
]  # ir.rs:9-41
OP = {name: i for i, name in enumerate(OPCODES)}
UNARY = {OP[n] for n in ["NOP", "ARGX", "ARGY", "ARGZ", "LOG", "SQR", "SQRT", "SIN", "COS",
                         "NEG", "EXP", "TRUNC", "FLOOR", "CEIL", "SIGN", "ABS", "RET"]}  # ir.rs:45-52
TAIL = {OP[n] for n in ["EXP", "LOG", "SQRT", "MIN", "MAX", "FLOOR", "CEIL", "ABS", "SIN", "COS",
                        "POW", "MOD", "ATAN2"]}  # ir.rs:54-58


def _f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", x))[0]


def _hex_lit(s: str) -> float:
    bits = int(s, 16)
    return _f32(struct.unpack("<d", struct.pack("<Q", bits))[0])


class Instr:
    __slots__ = ("index", "op", "uses", "larg", "rarg", "val")

    def __init__(self, index, op, larg=("L", 0.0), rarg=("L", 0.0)):
        self.index = index
        self.op = op
        self.uses = 0
        self.larg = larg
        self.rarg = rarg
        self.val = (0.0, 0.0)


def _reg(tok, a, b):
    s = tok[a:len(tok) - b]
    if not s.isdigit():
        raise ValueError(f"bad register {tok!r}")
    return ("R", int(s))


def _dec(tok, b):
    s = tok[0:len(tok) - b]
    try:
        return ("L", _f32(float(s)))
    except ValueError as e:
        raise ValueError(f"bad literal {tok!r}") from e


def _hex(tok, b):
    return ("L", _hex_lit(tok[2:len(tok) - b]))


def _tail_op(t):  # ir.rs:212-229
    for key, name in [("sqrt", "SQRT"), ("log", "LOG"), ("exp", "EXP"), ("min", "MIN"),
                      ("max", "MAX"), ("floor", "FLOOR"), ("abs", "ABS"), ("sin", "SIN"),
                      ("cos", "COS"), ("pow", "POW"), ("mod", "MOD"), ("atan2", "ATAN2")]:
        if key in t:
            return OP[name]
    return OP["NOP"]


def parse_llvm_ir(text: str, instructions: list) -> None:
    """ir.rs:190-331"""
    a = text.index("fffff")
    b = text[a:]
    start = b.index("\n")
    end = b.index("}")
    f = b[start:end - 1]
    lines = f.split("\n")
    for line in lines[1:]:
        tokens = line.split()
        ins = Instr(len(instructions), OP["NOP"])
        if tokens[0] == "ret":
            ins.op = OP["RET"]
        else:
            k = tokens[2]
            ins.op = {"fadd": OP["ADD"], "fneg": OP["NEG"], "fsub": OP["SUB"], "fmul": OP["MUL"],
                      "fdiv": OP["DIV"]}.get(k, None)
            if ins.op is None:
                ins.op = _tail_op(tokens[5]) if k == "tail" else OP["NOP"]
        op = ins.op
        if op in TAIL and op in UNARY:
            t = tokens[6]
            ins.larg = _reg(t, 1, 1) if "%" in t else (_hex(t, 1) if "0x" in t else _dec(t, 0))
        elif op in TAIL:
            t = tokens[6]
            ins.larg = _reg(t, 1, 1) if "%" in t else _dec(t, 0)
            t = tokens[8]
            ins.rarg = _reg(t, 1, 1) if "%" in t else (_hex(t, 1) if "0x" in t else _dec(t, 1))
        elif op in UNARY:
            if tokens[0] == "ret":
                ins.larg = _reg(tokens[2], 1, 0)
            else:
                t = tokens[4]
                ins.larg = _reg(t, 1, 0) if "%" in t else _dec(t, 0)
            ins.rarg = ("L", 0.0)
        else:
            t = tokens[4]
            ins.larg = _reg(t, 1, 1) if "%" in t else (_hex(t, 1) if "0x" in t else _dec(t, 1))
            t = tokens[5]
            ins.rarg = _reg(t, 1, 0) if "%" in t else (_hex(t, 0) if "0x" in t else _dec(t, 0))
        # ir.rs:297-307
        if ins.larg[0] == "R" and ins.larg[1] > 3:
            ins.larg = ("R", ins.larg[1] - 1)
        if ins.rarg[0] == "R" and ins.rarg[1] > 3:
            ins.rarg = ("R", ins.rarg[1] - 1)
        # ir.rs:309-313
        if ins.op == OP["MUL"] and ins.larg == ins.rarg:
            ins.op = OP["SQR"]
            ins.rarg = ("L", 0.0)
        # ir.rs:315-327
        for arg in (ins.larg, ins.rarg):
            if arg[0] == "R":
                if arg[1] >= len(instructions):
                    raise ValueError("register used before its definition")
                instructions[arg[1]].uses += 1
        instructions.append(ins)


def ir_new(text: str, time: float = 0.0, lo: float = -5.0, hi: float = 5.0) -> list:
    """ir.rs:334-366 (without the 4096 cap)."""
    ins = [Instr(i, OP["ARGX"] + i) for i in range(4)]
    for i in range(3):
        ins[i].val = (lo, hi)
    ins[3].val = (time, time)
    try:
        parse_llvm_ir(text, ins)
    except (IndexError, KeyError) as e:  # where ir.rs panics on an index or unwrap
        raise ValueError("cannot lower: %r" % e) from e
    ins[-1].uses += 1
    return ins


def to_gpu(ins: Instr) -> tuple:
    """ir.rs:140-181 -> (index_, opcode_uses, larg_rarg, literal, val0, val1, sens0, sens1)."""
    literal = 0.0
    side = 3
    if ins.larg[0] == "R":
        side -= 2
        larg = ins.larg[1] & 0xFFFF
    else:
        literal = ins.larg[1]
        larg = 0
    if ins.rarg[0] == "R":
        side -= 1
        rarg = ins.rarg[1] & 0xFFFF
    else:
        literal = ins.rarg[1]
        rarg = 0
    op = (ins.op | (side << 14)) & 0xFFFF
    return (ins.index & 0xFFFF, (op << 16) | (ins.uses & 0xFFFF), (larg << 16) | rarg, literal,
            ins.val[0], ins.val[1], 0.0, 0.0)


def lower(text: str, time: float = 0.0) -> list:
    return [to_gpu(i) for i in ir_new(text, time)]
