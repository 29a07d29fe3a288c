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

// Maps (op, op_top) to a handler and allocates registers by linear scan
// over SSA last uses.  Fails with TSI_ERR_TAPE_TOO_WIDE beyond 256 live
// values and TSI_ERR_INVALID_ARGUMENT for tapes shorter than the 4 ARGs.
bool compile_tape(const std::vector<IrInstr> &ins, PackedTape &out, tsi_status &status,
                  std::string &why);

}  // namespace tsi
