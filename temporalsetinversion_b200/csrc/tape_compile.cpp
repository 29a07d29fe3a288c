// tape_compile.cpp — handler selection and register allocation.
#include "tape_compile.h"

#include <algorithm>
#include <set>
#include <utility>
#include <cstring>

#include "opcost.h"

namespace tsi {
namespace {

uint32_t op_top_of(const IrInstr &in) {  // ir.rs:146-171
  uint32_t side = 3;
  if (in.larg.is_reg) side -= 2;
  if (in.rarg.is_reg) side -= 1;
  return side;
}

uint32_t handler_of(uint32_t op, uint32_t top) {
  switch (top) {
    case 0:  // compute.wgsl:3710-3749
      switch (op) {
        case TSI_OP_ADD: return H_ADD_II;
        case TSI_OP_SUB: return H_SUB_II;
        case TSI_OP_DIV: return H_DIV_II;
        case TSI_OP_MUL: return H_MUL_II;
        case TSI_OP_MIN: return H_MIN_II;
        case TSI_OP_MAX: return H_MAX_II;
        case TSI_OP_POW: return H_POW_II;
        case TSI_OP_MOD: return H_MOD_II;
        case TSI_OP_ATAN2: return H_ATAN2_II;
        default: return H_BAD_II;
      }
    case 1:  // compute.wgsl:3643-3709
      switch (op) {
        case TSI_OP_SQR: return H_SQR;
        case TSI_OP_SQRT: return H_SQRT;
        case TSI_OP_EXP: return H_EXP;
        case TSI_OP_LOG: return H_LOG;
        case TSI_OP_NEG: return H_NEG;
        case TSI_OP_ABS: return H_ABS;
        case TSI_OP_FLOOR: return H_FLOOR;
        case TSI_OP_SIN: return H_SIN;
        case TSI_OP_COS: return H_COS;
        case TSI_OP_ADD: return H_ADD_IF;
        case TSI_OP_SUB: return H_SUB_IF;
        case TSI_OP_DIV: return H_DIV_IF;
        case TSI_OP_MUL: return H_MUL_IF;
        case TSI_OP_MIN: return H_MIN_IF;
        case TSI_OP_MAX: return H_MAX_IF;
        case TSI_OP_POW: return H_POW_IF;
        case TSI_OP_RET: return H_COPY;
        case TSI_OP_MOD: return H_MOD_IF;
        case TSI_OP_ATAN2: return H_ATAN2_IF;
        default: return H_BAD_I;
      }
    case 2:  // compute.wgsl:3750-3764
      switch (op) {
        case TSI_OP_SUB: return H_SUB_FI;
        case TSI_OP_DIV: return H_DIV_FI;
        default: return H_BAD_FI;
      }
    default:  // compute.wgsl:3765, the value stays I_FROM(0.0)
      return H_CONST;
  }
}

}  // namespace

bool compile_tape(const std::vector<IrInstr> &ins, PackedTape &out, tsi_status &status,
                  std::string &why) {
  const uint32_t n = uint32_t(ins.size());
  if (n < 4) {
    status = TSI_ERR_INVALID_ARGUMENT;
    why = "a tape needs the four ARG slots";
    return false;
  }
  out = PackedTape{};
  out.count = n;
  // last use of every slot; the field (slot n-1) stays live to the end
  std::vector<int64_t> last_use(n, -1);
  for (uint32_t j = 4; j < n; ++j) {
    const IrInstr &in = ins[j];
    uint32_t top = op_top_of(in);
    if (top == 0 || top == 1) last_use[in.larg.reg] = j;
    if (top == 0 || top == 2) last_use[in.rarg.reg] = j;
  }
  last_use[n - 1] = int64_t(n);

  uint8_t used[TSI_MAX_REGS];
  std::memset(used, 0, sizeof(used));
  std::vector<uint32_t> reg(n, 0);
  for (uint32_t a = 0; a < 4; ++a) {
    reg[a] = a;
    used[a] = (last_use[a] >= 0) ? 1 : 0;
  }
  uint32_t maxreg = 3;
  static const uint32_t fwd_cost[H_COUNT] = TSI_OPCOST_FWD_INIT;
  static const uint32_t rr_cost[H_COUNT] = TSI_OPCOST_RR_INIT;
  out.code.reserve(size_t(n - 4) * 2);
  for (uint32_t j = 4; j < n; ++j) {
    const IrInstr &in = ins[j];
    const uint32_t top = op_top_of(in);
    const uint32_t h = handler_of(in.op, top);
    uint32_t a_slot = 0, b_slot = 0;
    bool has_a = false, has_b = false;
    uint32_t w1 = 0;
    float lit = 0.0f;
    if (top == 1) lit = in.rarg.lit;
    else if (top == 2 || top == 3) lit = in.larg.is_reg ? 0.0f : in.larg.lit;
    if (top == 3) lit = in.rarg.lit;  // ir.rs:160-168 keeps the rarg literal last
    if (top == 0) {
      a_slot = in.larg.reg; b_slot = in.rarg.reg; has_a = has_b = true;
    } else if (top == 1) {
      a_slot = in.larg.reg; has_a = true;
    } else if (top == 2) {
      a_slot = in.rarg.reg; has_a = true;
    }
    const uint32_t ra = has_a ? reg[a_slot] : 0;
    const uint32_t rb = has_b ? reg[b_slot] : 0;
    const uint32_t fa = has_a ? (((ins[a_slot].uses & 0xFFFFu) == 1u) ? 1u : 0u) : 0u;
    const uint32_t fb = has_b ? (((ins[b_slot].uses & 0xFFFFu) == 1u) ? 1u : 0u) : 0u;
    if (top == 0) {
      w1 = rb;
    } else {
      float v = (h == H_CONST) ? 0.0f : lit;  // op_top 3 evaluates to [0,0]
      std::memcpy(&w1, &v, 4);
    }
    // free operands at their last use (before allocating the destination)
    if (has_a && last_use[a_slot] == int64_t(j)) used[ra] = 0;
    if (has_b && last_use[b_slot] == int64_t(j)) used[rb] = 0;
    uint32_t d = 0;
    while (d < TSI_MAX_REGS && used[d]) ++d;
    if (d >= TSI_MAX_REGS) {
      status = TSI_ERR_TAPE_TOO_WIDE;
      why = "more than 256 interval values live at slot " + std::to_string(j);
      return false;
    }
    reg[j] = d;
    used[d] = (last_use[j] >= 0) ? 1 : 0;  // a never-read value frees at once
    if (d > maxreg) maxreg = d;
    out.code.push_back(TSI_W0(h, fa, fb, d, ra));
    out.code.push_back(w1);
    if (TSI_H_IS_MINMAX(h)) out.n_minmax++;
    out.fwd_cost += fwd_cost[h] + TSI_FIX_COST;
    out.rev_cost += rr_cost[h] + TSI_REV_OPERAND_COST * TSI_H_NREG(h);
  }
  out.nregs = maxreg + 1;
  out.out_reg = reg[n - 1];
  out.slot_reg = reg;
  return true;
}

bool compile_wide(const std::vector<IrInstr> &ins, const PackedTape &narrow, WideTape &out, tsi_status &status,
                  std::string &why) {
  const uint32_t n = uint32_t(ins.size());
  out = WideTape{};
  if (n <= 4) return true;
  if (n >= (1u << 24)) {
    status = TSI_ERR_TAPE_TOO_WIDE;
    why = "bundled tape limited to 2^24 slots";
    return false;
  }
  // operands of every slot
  std::vector<uint32_t> opa(n, TSI_NONE), opb(n, TSI_NONE);
  for (uint32_t j = 4; j < n; ++j) {
    const uint32_t top = op_top_of(ins[j]);
    if (top == 0) {
      opa[j] = ins[j].larg.reg;
      opb[j] = ins[j].rarg.reg;
    } else if (top == 1) {
      opa[j] = ins[j].larg.reg;
    } else if (top == 2) {
      opa[j] = ins[j].rarg.reg;
    }
  }
  auto handler = [&](uint32_t j) { return TSI_W0_H(narrow.code[2 * (j - 4)]); };
  // users of every value, in program order (an instruction reading one value
  // through both operands is one user)
  std::vector<std::vector<uint32_t>> users(n);
  for (uint32_t j = 4; j < n; ++j) {
    if (opa[j] != TSI_NONE) users[opa[j]].push_back(j);
    if (opb[j] != TSI_NONE && opb[j] != opa[j]) users[opb[j]].push_back(j);
  }
  // The reverse pass accumulates a value's sensitivity user by user, in
  // reverse program order, and that order fixes the rounding.  A value with
  // one user receives it directly; a value with several gets one
  // contribution record per user, which the value sums in that order when
  // the reverse pass reaches it.  The skip rule (zero sensitivity of a
  // single-use operand) relies on the ir.rs use count agreeing with the
  // users found here.
  for (uint32_t j = 4; j < n; ++j) {
    const uint32_t w0 = narrow.code[2 * (j - 4)];
    if ((TSI_W0_FA(w0) && opa[j] != TSI_NONE && users[opa[j]].size() != 1) ||
        (TSI_W0_FB(w0) && opb[j] != TSI_NONE && users[opb[j]].size() != 1)) {
      status = TSI_ERR_INVALID_ARGUMENT;
      why = "single-use flag on a value with several users";
      return false;
    }
  }
  std::vector<uint32_t> gbase(n, TSI_NONE), rec_a(n, TSI_NONE), rec_b(n, TSI_NONE);
  uint32_t ncontrib = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (users[v].size() < 2) continue;
    gbase[v] = ncontrib;
    for (size_t u = users[v].size(); u-- > 0;) {  // last user first
      const uint32_t j = users[v][u];
      if (opa[j] == v) rec_a[j] = ncontrib;
      if (opb[j] == v) rec_b[j] = ncontrib;
      ++ncontrib;
    }
  }
  // List scheduling into bundles of warp groups: a bundle is one block step,
  // at most 8 groups of at most 32 mutually independent instructions, each
  // group of one handler (so a warp runs its group without divergence and
  // groups of different handlers share a step).  Priority is the longest
  // chain from the instruction to the field; a step repeatedly takes the 32
  // highest-priority ready instructions of the handler whose best ready
  // instruction has the highest priority (the oldest instruction on a tie).
  // Users of a step's instructions become ready at the next step.
  const uint32_t groups_per_bundle = WideTape::kWidth / 32u;
  // the handlers the device evaluates inline (interp.cuh op_forward
  // and constants); the others run out of line
  auto inline_handler = [](uint32_t h) {
    switch (h) {
      case H_CONST: case H_COPY: case H_ADD_II: case H_SUB_II: case H_MUL_II: case H_MIN_II: case H_MAX_II:
      case H_ADD_IF: case H_SUB_IF: case H_MUL_IF: case H_MIN_IF: case H_MAX_IF: case H_SQR: case H_SQRT:
      case H_NEG: case H_ABS: case H_SUB_FI:
        return true;
      default:
        return false;
    }
  };
  std::vector<uint32_t> prio(n, 0);
  for (uint32_t j = n; j-- > 4;) {
    uint32_t p = 0;
    for (uint32_t u : users[j]) p = std::max(p, prio[u]);
    prio[j] = p + 1u;
  }
  std::vector<uint32_t> indeg(n, 0);
  for (uint32_t j = 4; j < n; ++j) {
    if (opa[j] != TSI_NONE && opa[j] >= 4) ++indeg[j];
    if (opb[j] != TSI_NONE && opb[j] >= 4 && opb[j] != opa[j]) ++indeg[j];
  }
  using Key = std::pair<uint32_t, uint32_t>;  // (~priority, instruction): highest priority, then oldest, first
  std::vector<std::set<Key>> ready(64);
  for (uint32_t j = 4; j < n; ++j)
    if (indeg[j] == 0) ready[handler(j)].insert(Key(~prio[j], j));
  std::vector<std::vector<std::vector<uint32_t>>> bundles;  // bundle -> groups -> instructions
  uint32_t scheduled = 0;
  std::vector<uint32_t> next;
  while (scheduled < n - 4) {
    std::vector<std::vector<uint32_t>> groups;
    // an out-of-line handler waits while it has slack (its best ready
    // instruction is off the step's critical path) and inline work is ready,
    // so that its instructions gather into few steps
    uint32_t cp = 0;
    bool inline_ready = false;
    for (uint32_t h = 0; h < 64; ++h)
      if (!ready[h].empty()) {
        cp = std::max(cp, ~ready[h].begin()->first);
        inline_ready = inline_ready || inline_handler(h);
      }
    auto eligible = [&](uint32_t h) {
      return inline_handler(h) || !inline_ready || ~ready[h].begin()->first >= cp;
    };
    while (groups.size() < groups_per_bundle) {
      uint32_t hb = 64;
      for (uint32_t h = 0; h < 64; ++h)
        if (!ready[h].empty() && eligible(h) && (hb == 64 || *ready[h].begin() < *ready[hb].begin())) hb = h;
      if (hb == 64) break;
      // a group of an out-of-line handler (elementary functions, divisions:
      // a step of them costs several steps of the others) takes every ready
      // instruction of its handler into this step, so that such handlers
      // occupy as few steps as possible
      do {
        std::vector<uint32_t> g;
        while (g.size() < 32u && !ready[hb].empty()) {
          g.push_back(ready[hb].begin()->second);
          ready[hb].erase(ready[hb].begin());
        }
        groups.push_back(std::move(g));
      } while (!inline_handler(hb) && !ready[hb].empty() && groups.size() < groups_per_bundle);
    }
    if (groups.empty()) {
      status = TSI_ERR_INVALID_ARGUMENT;
      why = "bundle scheduling made no progress";
      return false;
    }
    next.clear();
    for (const auto &g : groups)
      for (uint32_t j : g) {
        ++scheduled;
        for (uint32_t u : users[j])
          if (--indeg[u] == 0) next.push_back(u);
      }
    for (uint32_t u : next) ready[handler(u)].insert(Key(~prio[u], u));
    bundles.push_back(std::move(groups));
  }
  const uint32_t nb = uint32_t(bundles.size());
  // slots: a bundle's groups at 32-slot strides (lane = slot - first - 32 x
  // group); the lanes a group leaves free are padding slots (handler
  // TSI_H_PAD, no operands, no records)
  uint32_t nslots = 0;
  for (const auto &bg : bundles) nslots += 32u * uint32_t(bg.size() - 1) + uint32_t(bg.back().size());
  out.slots.assign(size_t(nslots) * 12, 0);
  out.bundles.assign(size_t(nb) * 2, 0);
  out.narrow_mm.assign(n - 4, TSI_NONE);
  {
    uint32_t mm = 0;
    for (uint32_t j = 4; j < n; ++j) {
      const uint32_t h = TSI_W0_H(narrow.code[2 * (j - 4)]);
      if (TSI_H_IS_MINMAX(h)) out.narrow_mm[j - 4] = mm++;
    }
  }
  uint32_t off = 0;
  for (uint32_t k = 0; k < nb; ++k) {
    const auto &bg = bundles[k];
    const uint32_t count = 32u * uint32_t(bg.size() - 1) + uint32_t(bg.back().size());
    for (uint32_t s = 0; s < count; ++s) {
      uint32_t *S = &out.slots[size_t(off + s) * 12];
      const auto &g = bg[s / 32u];
      if (s % 32u >= g.size()) {  // padding
        S[0] = TSI_H_PAD;
        S[5] = S[6] = S[7] = S[8] = S[9] = S[10] = TSI_NONE;
        continue;
      }
      const uint32_t j = g[s % 32u];
      const uint32_t w0 = narrow.code[2 * (j - 4)], w1 = narrow.code[2 * (j - 4) + 1];
      const uint32_t h = TSI_W0_H(w0);
      S[0] = h | (TSI_W0_FA(w0) << 6) | (TSI_W0_FB(w0) << 7) | (j << 8);
      // the min/max ordinal sits in the word the handler does not use: the
      // literal's for two registers, B's for a register and a literal
      const uint32_t mmo = TSI_H_IS_MINMAX(h) ? out.narrow_mm[j - 4] : 0u;
      S[1] = opa[j] != TSI_NONE ? opa[j] : 0u;
      S[2] = opb[j] != TSI_NONE ? opb[j] : (TSI_H_IS_II(h) ? 0u : mmo);
      S[3] = TSI_H_IS_II(h) ? mmo : w1;  // literal bits
      S[4] = j;
      S[5] = out.narrow_mm[j - 4];
      S[6] = opa[j];
      S[7] = opb[j];
      S[8] = rec_a[j];
      S[9] = rec_b[j];
      S[10] = gbase[j];
      S[11] = gbase[j] == TSI_NONE ? 0u : uint32_t(users[j].size());
    }
    out.bundles[2 * k] = off;
    out.bundles[2 * k + 1] = count;
    off += count;
  }
  for (uint32_t a = 0; a < 4; ++a) {
    out.arg_gbase[a] = gbase[a];
    out.arg_gcount[a] = gbase[a] == TSI_NONE ? 0u : uint32_t(users[a].size());
  }
  out.ncontrib = ncontrib;
  out.nvalues = n;
  out.nbundles = nb;
  return true;
}

}  // namespace tsi
