// Device-side interpreter ("VM") for short streams (see vm.cu): straight-line
// segments, and whole programs with their if/while control flow.
#pragma once

#include <cstdint>

#include "device.h"

namespace bsz {

// One instruction, 16 bytes.
//
// Segment mode: operands and destinations are value locations: v >= 0 is
// slot v of the slot file (v * n_words words in), v < 0 is entry -1 - v of
// the external pointer table (bound inputs, constants, and buffers that
// outlive the segment).
//
// Program mode adds control flow and device-side state: every stream value
// is a slot with a tail bit (tails[slot]); ints live in 64-bit registers;
// per-class op counters reproduce the dynamic op count and op mix.
enum VmCode : uint8_t {
  kVmNot = 0, kVmAnd, kVmOr, kVmXor, kVmAndNot, kVmAdd, kVmShl, kVmShr, kVmPop,
  // program mode only
  kVmCopy,     // dst <- a (words and tail)
  kVmFill,     // dst <- constant `fill`: 0 ZERO, 1 the N-bit mask (ONES operand), 2 all ones, tail 1
  kVmLoad,     // dst <- ext[a] (words), tail = fill
  kVmStore,    // ext[dst] <- slot a (words)
  kVmJz,       // if slot a is zero (no stored bit and tail 0): jump to instruction b
  kVmJmp,      // jump to instruction b
  kVmPopI,     // ireg[dst] <- popcount(slot a); error 1 if tail(a) = 1
  kVmIConst,   // ireg[dst] <- (uint32)a | (int64)b << 32
  kVmIAdd, kVmISub, kVmIMul,   // ireg[dst] <- ireg[a] op ireg[b]
  kVmTick,     // ireg[dst] += 1; error 2 if it exceeds 10000 (while-loop limit)
  kVmErr       // error a
};

// Error codes written by program mode; the host raises the reference
// interpreter's messages for 1-3.  kVmErrBudget: the program executed more
// than kVmMaxExecuted instructions (nested while loops multiply their
// 10,000-iteration limits); the host then runs it with the host-driven walk
// instead, which is exact because program mode writes only its own slots and
// output buffers.
enum VmError : uint32_t { kVmOk = 0, kVmErrNegPop = 1, kVmErrWhile = 2, kVmErrNegShift = 3, kVmErrBudget = 4 };
constexpr int64_t kVmMaxExecuted = int64_t(1) << 27;

// Op-count classes (VmOp::cls): 0 = not counted.
enum VmClass : uint8_t {
  kClsNone = 0, kClsNot, kClsAnd, kClsOr, kClsXor, kClsAdd, kClsShl, kClsShr, kClsPop, kClsCount
};

struct VmOp {
  uint8_t code;
  uint8_t fill;     // Shr (segment mode): bits shifted in from above are ones; Fill/Load: see codes
  uint8_t cls;      // program mode: op-count class
  uint8_t pad;
  int32_t dst;      // Pop: popcount slot index; PopI/IConst/I*: int register
  int32_t a;
  int32_t b;        // Shl / Shr: shift amount (clamped to 64 * n_words); Jz/Jmp: target
};
static_assert(sizeof(VmOp) == 16, "VmOp is 16 bytes");

struct VmLaunch {
  const VmOp* ops;
  int64_t n_ops;
  const uint64_t* const* ext;
  uint64_t* file;            // global slot file (unused when it fits in shared memory)
  int64_t n_slots;
  int64_t nw;
  uint64_t last_mask;
  unsigned long long* pops;
};

// Program-mode state block in device memory (zeroed before the launch, read
// back after it):
// [err u32, pad u32][counters u64 x kClsCount][iregs i64 x n_iregs][tails u8 x n_slots]
struct VmProgLaunch {
  VmLaunch base;             // ops, ext, file, n_slots, nw, last_mask (pops unused)
  uint8_t* state;
  int64_t n_iregs;
};

inline size_t vm_state_bytes(int64_t n_iregs, int64_t n_slots) {
  return 8 + 8 * static_cast<size_t>(kClsCount) + 8 * static_cast<size_t>(n_iregs) +
         static_cast<size_t>(n_slots);
}

// Largest stream the automatic policy runs on the VM.
constexpr int64_t kVmMaxWords = 8192;

// Runs the instruction list with one CTA on the context's stream.  `file`
// may be null when n_slots * nw words fit in shared memory.
void launch_vm(Device& dev, const VmLaunch& L);
void launch_vm_program(Device& dev, const VmProgLaunch& L);
// Bytes of shared memory the VM would use for a slot file (0 = global).
int64_t vm_smem_bytes(int64_t n_slots, int64_t nw);

}  // namespace bsz
