// ir_lower.h — host-side tape lowering: LLVM IR subset -> tape instructions.
//
// Behavioural restatement of src/ir.rs:190-366 (parseLLVMIR, IR::new,
// Instruction::to_gpu) in C++, with 32-bit register indices instead of the
// u16 fields of ir.rs:76-84 so tapes beyond 65535 slots still lower.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "tsi.h"

namespace tsi {

struct IrArg {
  bool is_reg = false;
  uint32_t reg = 0;
  float lit = 0.0f;
  bool operator==(const IrArg &o) const {
    return is_reg == o.is_reg && (is_reg ? reg == o.reg : lit == o.lit);
  }
};

// ir.rs:76-84
struct IrInstr {
  uint32_t index = 0;
  uint32_t op = TSI_OP_NOP;
  uint32_t uses = 0;  // only the count of ir.rs's `uses: Vec<u16>` is ever read
  IrArg larg, rarg;
  float val[2] = {0.0f, 0.0f};
  float sens[2] = {0.0f, 0.0f};
};

// Parse error with the 1-based line of the function body that failed.
struct IrError {
  int line = 0;
  std::string message;
};

// IR::new (ir.rs:334-366) on `text`: four ARG slots with the root box and
// [time,time], then the parsed body, then the dummy use of ir.rs:355.
bool ir_new(const std::string &text, float time, const float root_lo[3], const float root_hi[3],
            std::vector<IrInstr> &out, IrError &err);

// Instruction::to_gpu (ir.rs:140-181), truncating fields to 16 bits as the
// reference does.
tsi_gpu_instruction ir_to_gpu(const IrInstr &in);

// Inverse of ir_to_gpu for uploaded tapes; validates register indices.
bool ir_from_gpu(const tsi_gpu_instruction *g, uint32_t n, std::vector<IrInstr> &out,
                 tsi_status &status, std::string &why);

}  // namespace tsi
