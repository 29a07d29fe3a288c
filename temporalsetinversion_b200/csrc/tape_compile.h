// tape_compile.h — IrInstr list -> packed, register-allocated device tape.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "ir_lower.h"
#include "tape_format.h"

namespace tsi {

struct PackedTape {
  std::vector<uint32_t> code;  // 2 words per instruction (slots 4..count-1)
  uint32_t count = 0;          // instruction_count including the 4 ARG slots
  uint32_t nregs = 0;          // registers used (>= 4)
  uint32_t out_reg = 0;        // register holding the field (slot count-1)
  uint32_t n_minmax = 0;
  uint64_t fwd_cost = 0;       // opcost.h, forward, one cell
  uint64_t rev_cost = 0;       // opcost.h, reverse, one cell
  std::vector<uint32_t> slot_reg;  // register of every SSA slot (debug, tests)
};

// Bundled ("wide") form of a full tape, for evaluating one cell with a whole
// block: instructions are list-scheduled into bundles (block steps) of at
// most kWidth / 32 groups of at most 32 mutually independent instructions,
// one handler per group, so every warp runs its group without divergence
// while groups of different handlers share a step.  A group fills the 32
// slots of its warp; lanes it leaves free hold padding slots (handler
// TSI_H_PAD).  Every SSA value keeps its own slot (no register reuse), so
// the reverse pass reads operands where the forward pass left them.  Per
// slot (3 x uint4):
//   s0.x  handler | single-use A << 6 | single-use B << 7 | dst SSA << 8
//   s0.y  A SSA (0 if absent)
//   s0.z  B SSA; for a register-literal min/max its min/max ordinal
//   s0.w  f32 literal; for a two-register min/max its min/max ordinal
//   s1    dst SSA, min/max ordinal (TSI_NONE unless a min/max), A SSA, B SSA
//         (TSI_NONE if absent; a padding slot: 0, TSI_NONE, TSI_NONE, TSI_NONE)
//   s2    contribution record of A, of B (TSI_NONE: the operand has one
//         user, which writes its sensitivity directly); first record and
//         record count of dst (count 0: dst has at most one user)
// A value with several users gets one contribution record per user, last
// user first, and sums them in that order when the reverse pass reaches it:
// the order of the sequential reverse pass (compute.wgsl:3786), whatever
// bundles the users fall in.
struct WideTape {
  static constexpr uint32_t kWidth = 256;  // threads of the evaluating block
  std::vector<uint32_t> slots;    // 12 words per slot
  std::vector<uint32_t> bundles;  // 2 words per bundle: first slot, slot count (padding included)
  std::vector<uint32_t> narrow_mm;  // per narrow instruction: min/max ordinal or TSI_NONE
  uint32_t arg_gbase[4] = {TSI_NONE, TSI_NONE, TSI_NONE, TSI_NONE};  // records of x, y, z, t
  uint32_t arg_gcount[4] = {0, 0, 0, 0};
  uint32_t ncontrib = 0;          // contribution records per cell
  uint32_t nvalues = 0;           // SSA values (the 4 arguments included)
  uint32_t nbundles = 0;
};

bool compile_wide(const std::vector<IrInstr> &ins, const PackedTape &narrow, WideTape &out, tsi_status &status,
                  std::string &why);

// Maps (op, op_top) to a handler and allocates registers by linear scan
// over SSA last uses.  Fails with TSI_ERR_TAPE_TOO_WIDE beyond 256 live
// values and TSI_ERR_INVALID_ARGUMENT for tapes shorter than the 4 ARGs.
bool compile_tape(const std::vector<IrInstr> &ins, PackedTape &out, tsi_status &status,
                  std::string &why);

}  // namespace tsi
