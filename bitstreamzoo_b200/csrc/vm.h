// Device-side segment interpreter ("VM") for short streams (see vm.cu).
#pragma once

#include <cstdint>

#include "device.h"

namespace bsz {

// One instruction, 16 bytes.  Operands and destinations are value
// locations: v >= 0 is slot v of the segment's slot file (v * n_words words
// in), v < 0 is entry -1 - v of the external pointer table (bound inputs,
// constants, and buffers that outlive the segment).
enum VmCode : uint8_t {
  kVmNot = 0, kVmAnd, kVmOr, kVmXor, kVmAndNot, kVmAdd, kVmShl, kVmShr, kVmPop
};

struct VmOp {
  uint8_t code;
  uint8_t fill;     // Shr: bits shifted in from above are ones
  uint16_t pad;
  int32_t dst;      // Pop: popcount slot index
  int32_t a;
  int32_t b;        // Shl / Shr: shift amount (clamped to 64 * n_words)
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

// Largest stream the automatic policy runs on the VM.
constexpr int64_t kVmMaxWords = 8192;

// Runs the instruction list with one CTA on the context's stream.  `file`
// may be null when n_slots * nw words fit in shared memory.
void launch_vm(Device& dev, const VmLaunch& L);
// Bytes of shared memory the VM would use for a slot file (0 = global).
int64_t vm_smem_bytes(int64_t n_slots, int64_t nw);

}  // namespace bsz
