// ir_lower.cpp — restatement of src/ir.rs:190-366 in C++.
//
// The token positions, literal decoding (hex = f64 bit pattern rounded to
// f32, ir.rs:241-245), register shift (ir.rs:297-307), x*x -> SQR rewrite
// (ir.rs:309-313) and use counting (ir.rs:315-327) follow the reference
// exactly; every input on which ir.rs would panic (unwrap on a bad token,
// index out of range) is reported as a parse error instead.
#include "ir_lower.h"

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace tsi {
namespace {

bool is_unary(uint32_t op) {  // ir.rs:45-52
  switch (op) {
    case TSI_OP_NOP: case TSI_OP_ARGX: case TSI_OP_ARGY: case TSI_OP_ARGZ:
    case TSI_OP_LOG: case TSI_OP_SQR: case TSI_OP_SQRT: case TSI_OP_SIN:
    case TSI_OP_COS: case TSI_OP_NEG: case TSI_OP_EXP: case TSI_OP_TRUNC:
    case TSI_OP_FLOOR: case TSI_OP_CEIL: case TSI_OP_SIGN: case TSI_OP_ABS:
    case TSI_OP_RET:
      return true;
    default:
      return false;
  }
}

bool is_tail(uint32_t op) {  // ir.rs:54-58
  switch (op) {
    case TSI_OP_EXP: case TSI_OP_LOG: case TSI_OP_SQRT: case TSI_OP_MIN: case TSI_OP_MAX:
    case TSI_OP_FLOOR: case TSI_OP_CEIL: case TSI_OP_ABS: case TSI_OP_SIN: case TSI_OP_COS:
    case TSI_OP_POW: case TSI_OP_MOD: case TSI_OP_ATAN2:
      return true;
    default:
      return false;
  }
}

std::vector<std::string> split_ws(const std::string &s) {
  std::vector<std::string> out;
  size_t i = 0, n = s.size();
  while (i < n) {
    while (i < n && (s[i] == ' ' || s[i] == '\t' || s[i] == '\r' || s[i] == '\v' || s[i] == '\f'))
      ++i;
    size_t j = i;
    while (j < n && !(s[j] == ' ' || s[j] == '\t' || s[j] == '\r' || s[j] == '\v' || s[j] == '\f'))
      ++j;
    if (j > i) out.push_back(s.substr(i, j - i));
    i = j;
  }
  return out;
}

// Rust `&token[a..b]` with bounds checks (ir.rs panics when out of range).
bool slice(const std::string &t, size_t a, size_t b, std::string &out) {
  if (a > b || b > t.size()) return false;
  out = t.substr(a, b - a);
  return true;
}

bool parse_u32(const std::string &s, uint32_t &v) {  // str::parse::<u32>
  if (s.empty()) return false;
  size_t i = (s[0] == '+') ? 1 : 0;
  if (i == s.size()) return false;
  uint64_t acc = 0;
  for (; i < s.size(); ++i) {
    if (s[i] < '0' || s[i] > '9') return false;
    acc = acc * 10 + uint64_t(s[i] - '0');
    if (acc > 0xFFFFFFFFull) return false;
  }
  v = uint32_t(acc);
  return true;
}

bool parse_f32(const std::string &s, float &v) {  // str::parse::<f32>
  if (s.empty()) return false;
  for (char c : s)
    if (c == ' ' || c == '\t' || c == 'x' || c == 'X') return false;  // no hex floats
  errno = 0;
  char *end = nullptr;
  v = std::strtof(s.c_str(), &end);
  return end == s.c_str() + s.size();
}

bool parse_hex_f64_as_f32(const std::string &s, float &v) {  // u64::from_str_radix + f64::from_bits
  if (s.empty() || s.size() > 17) return false;
  size_t i = (s[0] == '+') ? 1 : 0;
  if (i == s.size()) return false;
  uint64_t bits = 0;
  for (; i < s.size(); ++i) {
    char c = s[i];
    int d;
    if (c >= '0' && c <= '9') d = c - '0';
    else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
    else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
    else return false;
    if (bits >> 60) return false;  // overflow of u64
    bits = (bits << 4) | uint64_t(d);
  }
  double dv;
  std::memcpy(&dv, &bits, sizeof(dv));
  v = float(dv);  // `val as f32`: round to nearest even
  return true;
}

bool contains(const std::string &t, const char *needle) { return t.find(needle) != std::string::npos; }

// REGISTER(token[ra..len-rb].parse())
bool reg_arg(const std::string &t, size_t strip_front, size_t strip_back, IrArg &a) {
  std::string s;
  if (t.size() < strip_back || !slice(t, strip_front, t.size() - strip_back, s)) return false;
  uint32_t v;
  if (!parse_u32(s, v)) return false;
  a.is_reg = true;
  a.reg = v;
  return true;
}

bool hex_arg(const std::string &t, size_t strip_back, IrArg &a) {
  std::string s;
  if (t.size() < strip_back || !slice(t, 2, t.size() - strip_back, s)) return false;
  float v;
  if (!parse_hex_f64_as_f32(s, v)) return false;
  a.is_reg = false;
  a.lit = v;
  return true;
}

bool dec_arg(const std::string &t, size_t strip_back, IrArg &a) {
  std::string s;
  if (t.size() < strip_back || !slice(t, 0, t.size() - strip_back, s)) return false;
  float v;
  if (!parse_f32(s, v)) return false;
  a.is_reg = false;
  a.lit = v;
  return true;
}

uint32_t tail_op(const std::string &t) {  // ir.rs:212-229, first match wins
  if (contains(t, "sqrt")) return TSI_OP_SQRT;
  if (contains(t, "log")) return TSI_OP_LOG;
  if (contains(t, "exp")) return TSI_OP_EXP;
  if (contains(t, "min")) return TSI_OP_MIN;
  if (contains(t, "max")) return TSI_OP_MAX;
  if (contains(t, "floor")) return TSI_OP_FLOOR;
  if (contains(t, "abs")) return TSI_OP_ABS;
  if (contains(t, "sin")) return TSI_OP_SIN;
  if (contains(t, "cos")) return TSI_OP_COS;
  if (contains(t, "pow")) return TSI_OP_POW;
  if (contains(t, "mod")) return TSI_OP_MOD;
  if (contains(t, "atan2")) return TSI_OP_ATAN2;
  return TSI_OP_NOP;  // "cannot parse"
}

// One line of the function body -> instruction (ir.rs:199-329).
bool parse_line(const std::string &line, std::vector<IrInstr> &instructions, std::string &why) {
  std::vector<std::string> tok = split_ws(line);
  if (tok.empty()) {
    why = "empty line inside the function body";
    return false;
  }
  auto need = [&](size_t k) {
    if (tok.size() <= k) {
      why = "too few tokens";
      return false;
    }
    return true;
  };
  IrInstr ins;
  ins.index = uint32_t(instructions.size());
  ins.larg = IrArg{};  // LITERAL(0.0)
  ins.rarg = IrArg{};

  if (tok[0] == "ret") {
    ins.op = TSI_OP_RET;
  } else {
    if (!need(2)) return false;
    const std::string &k = tok[2];
    if (k == "fadd") ins.op = TSI_OP_ADD;
    else if (k == "fneg") ins.op = TSI_OP_NEG;
    else if (k == "fsub") ins.op = TSI_OP_SUB;
    else if (k == "fmul") ins.op = TSI_OP_MUL;
    else if (k == "fdiv") ins.op = TSI_OP_DIV;
    else if (k == "tail") {
      if (!need(5)) return false;
      ins.op = tail_op(tok[5]);
    } else {
      ins.op = TSI_OP_NOP;
    }
  }

  const uint32_t op = ins.op;
  bool ok = true;
  if (is_tail(op) && is_unary(op)) {  // ir.rs:238-248
    if (!need(6)) return false;
    const std::string &t = tok[6];
    if (contains(t, "%")) ok = reg_arg(t, 1, 1, ins.larg);
    else if (contains(t, "0x")) ok = hex_arg(t, 1, ins.larg);
    else ok = dec_arg(t, 0, ins.larg);
  } else if (is_tail(op) && !is_unary(op)) {  // ir.rs:249-263
    if (!need(8)) return false;
    const std::string &l = tok[6];
    if (contains(l, "%")) ok = reg_arg(l, 1, 1, ins.larg);
    else ok = dec_arg(l, 0, ins.larg);
    const std::string &r = tok[8];
    if (ok) {
      if (contains(r, "%")) ok = reg_arg(r, 1, 1, ins.rarg);
      else if (contains(r, "0x")) ok = hex_arg(r, 1, ins.rarg);
      else ok = dec_arg(r, 1, ins.rarg);
    }
  } else if (is_unary(op)) {  // ir.rs:264-273
    if (tok[0] == "ret") {
      if (!need(2)) return false;
      ok = reg_arg(tok[2], 1, 0, ins.larg);
    } else {
      if (!need(4)) return false;
      const std::string &t = tok[4];
      if (contains(t, "%")) ok = reg_arg(t, 1, 0, ins.larg);
      else ok = dec_arg(t, 0, ins.larg);
    }
    ins.rarg = IrArg{};
  } else {  // ir.rs:274-293
    if (!need(5)) return false;
    const std::string &l = tok[4];
    if (contains(l, "%")) ok = reg_arg(l, 1, 1, ins.larg);
    else if (contains(l, "0x")) ok = hex_arg(l, 1, ins.larg);
    else ok = dec_arg(l, 1, ins.larg);
    const std::string &r = tok[5];
    if (ok) {
      if (contains(r, "%")) ok = reg_arg(r, 1, 0, ins.rarg);
      else if (contains(r, "0x")) ok = hex_arg(r, 0, ins.rarg);
      else ok = dec_arg(r, 0, ins.rarg);
    }
  }
  if (!ok) {
    why = "unparsable operand";
    return false;
  }

  const uint32_t num_args = 4;  // ir.rs:297-307
  if (ins.larg.is_reg && ins.larg.reg > num_args - 1) ins.larg.reg -= 1;
  if (ins.rarg.is_reg && ins.rarg.reg > num_args - 1) ins.rarg.reg -= 1;

  if (ins.op == TSI_OP_MUL && ins.larg == ins.rarg) {  // ir.rs:309-313
    ins.op = TSI_OP_SQR;
    ins.rarg = IrArg{};
  }

  for (const IrArg *a : {&ins.larg, &ins.rarg}) {  // ir.rs:315-327
    if (a->is_reg) {
      if (a->reg >= instructions.size()) {
        why = "register used before its definition";
        return false;
      }
      instructions[a->reg].uses += 1;
    }
  }
  instructions.push_back(ins);
  return true;
}

}  // namespace

bool ir_new(const std::string &text, float time, const float root_lo[3], const float root_hi[3],
            std::vector<IrInstr> &out, IrError &err) {
  out.clear();
  for (uint32_t i = 0; i < 4; ++i) {  // ir.rs:335-348
    IrInstr a;
    a.index = i;
    a.op = TSI_OP_ARGX + i;
    if (i < 3) {
      a.val[0] = root_lo[i];
      a.val[1] = root_hi[i];
    } else {
      a.val[0] = time;
      a.val[1] = time;
    }
    out.push_back(a);
  }
  // parseLLVMIR, ir.rs:190-197
  size_t a = text.find("fffff");
  if (a == std::string::npos) {
    err = {0, "no function named *fffff* (the scene function f(x,y,z,t))"};
    return false;
  }
  std::string b = text.substr(a);
  size_t start = b.find('\n');
  size_t end = b.find('}');
  if (start == std::string::npos || end == std::string::npos || end == 0 || end - 1 < start) {
    err = {0, "malformed function body"};
    return false;
  }
  std::string f = b.substr(start, end - 1 - start);
  std::vector<std::string> lines;
  size_t p = 0;
  while (true) {
    size_t q = f.find('\n', p);
    if (q == std::string::npos) {
      lines.push_back(f.substr(p));
      break;
    }
    lines.push_back(f.substr(p, q - p));
    p = q + 1;
  }
  for (size_t i = 1; i < lines.size(); ++i) {
    std::string why;
    if (!parse_line(lines[i], out, why)) {
      err = {int(i), why + ": '" + lines[i] + "'"};
      return false;
    }
  }
  out.back().uses += 1;  // ir.rs:355, dummy use of the last instruction
  return true;
}

tsi_gpu_instruction ir_to_gpu(const IrInstr &in) {  // ir.rs:140-181
  float literal = 0.0f;
  uint32_t literal_side = 3;
  uint32_t larg = 0, rarg = 0;
  if (in.larg.is_reg) {
    literal_side -= 2;
    larg = in.larg.reg & 0xFFFFu;
  } else {
    literal = in.larg.lit;
  }
  if (in.rarg.is_reg) {
    literal_side -= 1;
    rarg = in.rarg.reg & 0xFFFFu;
  } else {
    literal = in.rarg.lit;
  }
  uint32_t op = (in.op | (literal_side << 14)) & 0xFFFFu;
  tsi_gpu_instruction g;
  g.index_ = in.index & 0xFFFFu;
  g.opcode_uses = (op << 16) | (in.uses & 0xFFFFu);
  g.larg_rarg = (larg << 16) | rarg;
  g.literal = literal;
  g.val[0] = in.val[0];
  g.val[1] = in.val[1];
  g.sens[0] = in.sens[0];
  g.sens[1] = in.sens[1];
  return g;
}

bool ir_from_gpu(const tsi_gpu_instruction *g, uint32_t n, std::vector<IrInstr> &out,
                 tsi_status &status, std::string &why) {
  out.assign(n, IrInstr{});
  for (uint32_t j = 0; j < n; ++j) {
    IrInstr &ins = out[j];
    uint32_t op16 = g[j].opcode_uses >> 16;
    uint32_t op = op16 & 0x3FFFu;
    uint32_t top = op16 >> 14;
    ins.index = j;
    ins.op = op;
    ins.uses = g[j].opcode_uses & 0xFFFFu;
    ins.val[0] = g[j].val[0];
    ins.val[1] = g[j].val[1];
    ins.sens[0] = g[j].sens[0];
    ins.sens[1] = g[j].sens[1];
    uint32_t l = g[j].larg_rarg >> 16, r = g[j].larg_rarg & 0xFFFFu;
    ins.larg = IrArg{};
    ins.rarg = IrArg{};
    if (top == 0 || top == 1) ins.larg = IrArg{true, l, 0.0f};
    else ins.larg.lit = g[j].literal;
    if (top == 0 || top == 2) ins.rarg = IrArg{true, r, 0.0f};
    else ins.rarg.lit = g[j].literal;
    if (j < 4) continue;  // ARG slots are overwritten per cell (compute.wgsl:3622-3625)
    if (op > TSI_OP_ATAN2) {
      status = TSI_ERR_BAD_OPCODE;
      why = "opcode " + std::to_string(op) + " at slot " + std::to_string(j);
      return false;
    }
    for (const IrArg *a : {&ins.larg, &ins.rarg}) {
      if (a->is_reg && a->reg >= j) {
        status = TSI_ERR_INVALID_ARGUMENT;
        why = "slot " + std::to_string(j) + " reads slot " + std::to_string(a->reg) +
              " that is not computed before it";
        return false;
      }
    }
    if (top == 0 && op == TSI_OP_NOP) {
      status = TSI_ERR_INVALID_ARGUMENT;
      why = "NOP with two register operands at slot " + std::to_string(j) +
            " (no lowering in ir.rs produces it)";
      return false;
    }
  }
  return true;
}

}  // namespace tsi
