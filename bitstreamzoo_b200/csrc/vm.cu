// Device-side interpreter for short streams.
//
// At small N the per-op form is launch-bound (a few microseconds per DSL
// operation whatever the stream length; the reference pays the same, plus a
// cudaMalloc per result), and compiling a fused kernel per segment costs far
// more than the segment's work.  The VM runs a whole segment -- possibly
// millions of operations of an unrolled loop nest -- as one launch of one
// CTA that walks a 16-byte instruction list:
//
//   * thread t owns words t, t + T, t + 2T, ... of every value (T = CTA size,
//     a multiple of 32, at most 1024), so pointwise operations need no
//     synchronisation beyond program order;
//   * temporaries live in a slot file, in shared memory when it fits (a
//     host-side linear scan keeps it to the segment's peak live count);
//     inputs, constants and values that outlive the segment are reached
//     through an external pointer table;
//   * ADD resolves carries per step of T words with warp ballots ((G|P) + G
//     + carry-in gives every lane's carry, bit 32 the carry out) and a
//     composition of the warps' (generate, propagate) pairs in shared memory;
//   * shifts read neighbouring words written by other threads, so every
//     instruction ends with a CTA barrier (a warp barrier when T = 32);
//   * POPCOUNT sums all stored words (unmasked, like the per-op kernel) and
//     adds one atomic per warp into its slot.
//
// Program mode (k_vm_program, compiled by vmprog.cpp) runs a whole program
// with its if/while control flow in the same way; see below.
//
// Every instruction has the exact semantics of the per-op kernel for the
// same node (masking of ~, + and << at the last word; >> filling with the
// operand's tail), so results are bit-identical to the plain form.
#include "vm.h"

#include <algorithm>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

namespace bsz {
namespace {

constexpr int64_t kVmSmemLimit = 200 * 1024;

struct VmArgs {
  const VmOp* ops;
  int64_t n_ops;
  const uint64_t* const* ext;
  uint64_t* file;
  int64_t nw;
  uint64_t last_mask;
  unsigned long long* pops;
};

__device__ __forceinline__ VmOp load_op(const VmOp* p) {
  const int4 v = __ldg(reinterpret_cast<const int4*>(p));
  VmOp o;
  o.code = static_cast<uint8_t>(v.x & 0xff);
  o.fill = static_cast<uint8_t>((v.x >> 8) & 0xff);
  o.cls = static_cast<uint8_t>((v.x >> 16) & 0xff);
  o.pad = 0;
  o.dst = v.y;
  o.a = v.z;
  o.b = v.w;
  return o;
}

// ---- per-instruction stream operations, shared by both modes -------------
// Thread tid of T owns words tid, tid + T, ...  Callers put a barrier
// between instructions.

__device__ __forceinline__ void vm_not(uint64_t* D, const uint64_t* A, int64_t nw, uint64_t lm, int tid, int T) {
  for (int64_t w = tid; w < nw; w += T) {
    uint64_t r = ~A[w];
    if (w == nw - 1) r &= lm;
    D[w] = r;
  }
}

__device__ __forceinline__ void vm_bitwise(uint8_t code, uint64_t* D, const uint64_t* A, const uint64_t* B,
                                           int64_t nw, int tid, int T) {
  for (int64_t w = tid; w < nw; w += T) {
    const uint64_t x = A[w], y = B[w];
    D[w] = code == kVmAnd ? (x & y) : code == kVmOr ? (x | y) : code == kVmXor ? (x ^ y) : (x & ~y);
  }
}

__device__ __forceinline__ void vm_shl(uint64_t* D, const uint64_t* A, int32_t k, int64_t nw, uint64_t lm,
                                       int tid, int T) {
  const int64_t ws = k >> 6;
  const int bs = k & 63;
  for (int64_t w = tid; w < nw; w += T) {
    const int64_t lo = w - ws;
    const uint64_t x = lo >= 0 ? A[lo] : 0;
    const uint64_t y = (bs && lo >= 1) ? A[lo - 1] : 0;
    uint64_t r = bs ? ((x << bs) | (y >> (64 - bs))) : x;
    if (w == nw - 1) r &= lm;
    D[w] = r;
  }
}

__device__ __forceinline__ void vm_shr(uint64_t* D, const uint64_t* A, int32_t k, uint64_t fill, int64_t nw,
                                       int tid, int T) {
  const int64_t ws = k >> 6;
  const int bs = k & 63;
  for (int64_t w = tid; w < nw; w += T) {
    const int64_t lo = w + ws;
    const uint64_t x = lo < nw ? A[lo] : fill;
    const uint64_t y = bs ? (lo + 1 < nw ? A[lo + 1] : fill) : 0;
    D[w] = bs ? ((x >> bs) | (y << (64 - bs))) : x;
  }
}

// Carries per step of T words: two ballots per warp, then the warps'
// (generate, propagate) pairs composed through shared memory.  Each thread
// reads only its own words before writing them, so D may alias A or B.
__device__ __forceinline__ void vm_add(uint64_t* D, const uint64_t* A, const uint64_t* B, int64_t nw,
                                       uint64_t lm, int tid, int T, uint32_t* s_g, uint32_t* s_p) {
  const int lane = tid & 31, warp = tid >> 5, n_warps = T >> 5;
  uint32_t carry = 0;
  for (int64_t base = 0; base < nw; base += T) {
    const int64_t w = base + tid;
    const bool in = w < nw;
    const uint64_t x = in ? A[w] : 0, y = in ? B[w] : 0;
    const uint64_t s = x + y;
    const uint32_t G = __ballot_sync(0xffffffffu, s < x);
    const uint32_t P = __ballot_sync(0xffffffffu, in && s == ~uint64_t(0));
    uint32_t cin, cout;
    if (n_warps == 1) {
      cin = carry;
      cout = static_cast<uint32_t>((static_cast<uint64_t>(G | P) + G + cin) >> 32);
    } else {
      if (lane == 0) {
        s_g[warp] = static_cast<uint32_t>((static_cast<uint64_t>(G | P) + G) >> 32);
        s_p[warp] = P == 0xffffffffu;
      }
      __syncthreads();
      cin = carry;
      for (int v = 0; v < warp; ++v) cin = s_g[v] | (s_p[v] & cin);
      cout = carry;
      for (int v = 0; v < n_warps; ++v) cout = s_g[v] | (s_p[v] & cout);
      __syncthreads();
    }
    const uint64_t z = static_cast<uint64_t>(G | P) + G + cin;
    const uint32_t carries = static_cast<uint32_t>(z) ^ P;
    if (in) {
      uint64_t r = s + ((carries >> lane) & 1u);
      if (w == nw - 1) r &= lm;
      D[w] = r;
    }
    carry = cout;
  }
}

// Popcount of all stored words (unmasked, like the per-op kernel), summed
// over the CTA into *out by one atomic per warp.
__device__ __forceinline__ void vm_popcount(unsigned long long* out, const uint64_t* A, int64_t nw, int tid,
                                            int T) {
  unsigned long long c = 0;
  for (int64_t w = tid; w < nw; w += T) c += __popcll(A[w]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((tid & 31) == 0 && c) atomicAdd(out, c);
}

__device__ __forceinline__ void vm_barrier(int T) {
  if (T > 32) __syncthreads();
  else __syncwarp();
}

// ---- segment mode ----------------------------------------------------------

template <bool SMEM>
__global__ void __launch_bounds__(1024) k_vm(VmArgs args) {
  extern __shared__ uint64_t s_file[];
  __shared__ uint32_t s_g[32], s_p[32];
  uint64_t* file = SMEM ? s_file : args.file;
  const int T = blockDim.x;
  const int tid = threadIdx.x;
  const int64_t nw = args.nw;
  const uint64_t lm = args.last_mask;
  auto loc = [&](int32_t v) -> uint64_t* {
    return v >= 0 ? file + static_cast<int64_t>(v) * nw : const_cast<uint64_t*>(args.ext[-1 - v]);
  };
  VmOp next = args.n_ops > 0 ? load_op(args.ops) : VmOp{};
  for (int64_t i = 0; i < args.n_ops; ++i) {
    const VmOp op = next;
    if (i + 1 < args.n_ops) next = load_op(args.ops + i + 1);
    const uint64_t* A = loc(op.a);
    switch (op.code) {
      case kVmNot: vm_not(loc(op.dst), A, nw, lm, tid, T); break;
      case kVmAnd: case kVmOr: case kVmXor: case kVmAndNot:
        vm_bitwise(op.code, loc(op.dst), A, loc(op.b), nw, tid, T);
        break;
      case kVmShl: vm_shl(loc(op.dst), A, op.b, nw, lm, tid, T); break;
      case kVmShr: vm_shr(loc(op.dst), A, op.b, op.fill ? ~uint64_t(0) : 0, nw, tid, T); break;
      case kVmAdd: vm_add(loc(op.dst), A, loc(op.b), nw, lm, tid, T, s_g, s_p); break;
      case kVmPop: vm_popcount(args.pops + op.dst, A, nw, tid, T); break;
      default: break;
    }
    vm_barrier(T);
  }
}

// ---- program mode ----------------------------------------------------------
// Control flow runs on the device: a condition is a CTA-wide OR of the
// slot's words (plus its tail), taken by every thread alike.  Thread 0
// updates tails, int registers and op counters; the barrier after every
// instruction publishes them.  Errors stop the program with a code the host
// turns into the reference's message.

struct VmProgArgs {
  VmArgs base;
  uint8_t* state;
  int64_t n_iregs;
};

template <bool SMEM>
__global__ void __launch_bounds__(1024) k_vm_program(VmProgArgs P) {
  extern __shared__ uint64_t s_file[];
  __shared__ uint32_t s_g[32], s_p[32];
  __shared__ uint32_t s_err;
  __shared__ unsigned long long s_pop;
  const VmArgs& args = P.base;
  uint64_t* file = SMEM ? s_file : args.file;
  const int T = blockDim.x;
  const int tid = threadIdx.x;
  const int64_t nw = args.nw;
  const uint64_t lm = args.last_mask;
  uint32_t* g_err = reinterpret_cast<uint32_t*>(P.state);
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(P.state + 8);
  long long* iregs = reinterpret_cast<long long*>(P.state + 8 + 8 * kClsCount);
  uint8_t* tails = P.state + 8 + 8 * kClsCount + 8 * P.n_iregs;
  if (tid == 0) {
    s_err = 0;
    s_pop = 0;
  }
  __syncthreads();
  auto slot = [&](int32_t v) -> uint64_t* { return file + static_cast<int64_t>(v) * nw; };
  int64_t pc = 0, executed = 0;
  while (pc < args.n_ops) {
    if (++executed > kVmMaxExecuted) {   // uniform: every thread leaves here
      if (tid == 0) *g_err = kVmErrBudget;
      return;
    }
    const VmOp op = load_op(args.ops + pc);
    ++pc;
    switch (op.code) {
      case kVmNot:
        vm_not(slot(op.dst), slot(op.a), nw, lm, tid, T);
        if (tid == 0) tails[op.dst] = 0;
        break;
      case kVmAnd: case kVmOr: case kVmXor: case kVmAndNot: {
        const uint8_t ta = tails[op.a], tb = tails[op.b];
        vm_bitwise(op.code, slot(op.dst), slot(op.a), slot(op.b), nw, tid, T);
        if (tid == 0)
          tails[op.dst] = op.code == kVmAnd ? (ta & tb) : op.code == kVmOr ? (ta | tb)
                          : op.code == kVmXor ? (ta ^ tb) : (ta & (tb ^ 1));
        break;
      }
      case kVmShl:
        vm_shl(slot(op.dst), slot(op.a), op.b, nw, lm, tid, T);
        if (tid == 0) tails[op.dst] = 0;
        break;
      case kVmShr: {
        const uint8_t ta = tails[op.a];
        vm_shr(slot(op.dst), slot(op.a), op.b, ta ? ~uint64_t(0) : 0, nw, tid, T);
        if (tid == 0) tails[op.dst] = ta;
        break;
      }
      case kVmAdd:
        vm_add(slot(op.dst), slot(op.a), slot(op.b), nw, lm, tid, T, s_g, s_p);
        if (tid == 0) tails[op.dst] = 0;
        break;
      case kVmCopy: {
        const uint64_t* A = slot(op.a);
        uint64_t* D = slot(op.dst);
        const uint8_t ta = tails[op.a];
        if (D != A)
          for (int64_t w = tid; w < nw; w += T) D[w] = A[w];
        if (tid == 0) tails[op.dst] = ta;
        break;
      }
      case kVmFill: {
        uint64_t* D = slot(op.dst);
        const uint64_t v = op.fill ? ~uint64_t(0) : 0;
        for (int64_t w = tid; w < nw; w += T) D[w] = (op.fill == 1 && w == nw - 1) ? (v & lm) : v;
        if (tid == 0) tails[op.dst] = op.fill == 2 ? 1 : 0;
        break;
      }
      case kVmLoad: {
        const uint64_t* A = args.ext[op.a];
        uint64_t* D = slot(op.dst);
        for (int64_t w = tid; w < nw; w += T) D[w] = A[w];
        if (tid == 0) tails[op.dst] = op.fill;
        break;
      }
      case kVmStore: {
        const uint64_t* A = slot(op.a);
        uint64_t* D = const_cast<uint64_t*>(args.ext[op.dst]);
        for (int64_t w = tid; w < nw; w += T) D[w] = A[w];
        break;
      }
      case kVmJz: {
        const uint64_t* A = slot(op.a);
        int any = 0;
        for (int64_t w = tid; w < nw; w += T) any |= A[w] != 0;
        const int nz = __syncthreads_or(any) || tails[op.a];
        if (!nz) pc = op.b;
        break;
      }
      case kVmJmp:
        pc = op.b;
        break;
      case kVmPopI: {
        if (tails[op.a]) {
          if (tid == 0) s_err = kVmErrNegPop;
          break;
        }
        vm_popcount(&s_pop, slot(op.a), nw, tid, T);
        __syncthreads();
        if (tid == 0) {
          iregs[op.dst] = static_cast<long long>(s_pop);
          s_pop = 0;
        }
        break;
      }
      case kVmIConst:
        if (tid == 0)
          iregs[op.dst] = static_cast<long long>(static_cast<uint64_t>(static_cast<uint32_t>(op.a)) |
                                                 (static_cast<uint64_t>(static_cast<uint32_t>(op.b)) << 32));
        break;
      case kVmIAdd: case kVmISub: case kVmIMul:
        if (tid == 0) {
          // two's-complement wrap, like the int64 host arithmetic
          const unsigned long long x = static_cast<unsigned long long>(iregs[op.a]);
          const unsigned long long y = static_cast<unsigned long long>(iregs[op.b]);
          iregs[op.dst] = static_cast<long long>(op.code == kVmIAdd ? x + y : op.code == kVmISub ? x - y : x * y);
        }
        break;
      case kVmTick:
        if (tid == 0) {
          const long long t = ++iregs[op.dst];
          if (t > 10000) s_err = kVmErrWhile;
        }
        break;
      case kVmErr:
        if (tid == 0) s_err = static_cast<uint32_t>(op.a);
        break;
      default:
        break;
    }
    if (op.cls && tid == 0 && s_err == 0) ++counters[op.cls];
    __syncthreads();
    if (s_err) break;
  }
  if (tid == 0) *g_err = s_err;
}

int vm_threads(int64_t nw) {
  const int64_t t = ((nw + 31) / 32) * 32;
  return static_cast<int>(std::max<int64_t>(32, std::min<int64_t>(1024, t)));
}

// Once per device: the opt-in shared-memory size of the slot-file kernels.
void set_smem_attr() {
  static std::mutex mu;
  static std::set<int> done;
  int d = 0;
  cudaGetDevice(&d);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(d)) return;
  cudaFuncSetAttribute(k_vm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kVmSmemLimit));
  cudaFuncSetAttribute(k_vm_program<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(kVmSmemLimit));
  done.insert(d);
}

void check_vm_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw CudaError(std::string(what) + " launch failed: " + cudaGetErrorString(e));
}

}  // namespace

int64_t vm_smem_bytes(int64_t n_slots, int64_t nw) {
  const int64_t b = std::max<int64_t>(1, n_slots) * nw * 8;
  return b <= kVmSmemLimit ? b : 0;
}

void launch_vm(Device& dev, const VmLaunch& L) {
  if (L.n_ops <= 0) return;
  VmArgs a{L.ops, L.n_ops, L.ext, L.file, L.nw, L.last_mask, L.pops};
  const int threads = vm_threads(L.nw);
  const int64_t smem = vm_smem_bytes(L.n_slots, L.nw);
  set_smem_attr();
  ProfScope prof(dev, "k_vm");
  if (smem > 0) {
    k_vm<true><<<1, threads, static_cast<size_t>(smem), dev.stream()>>>(a);
  } else {
    if (!L.file && L.n_slots > 0) throw std::invalid_argument("vm: slot file does not fit in shared memory");
    k_vm<false><<<1, threads, 0, dev.stream()>>>(a);
  }
  check_vm_launch("vm");
  ++dev.n_launches;
}

void launch_vm_program(Device& dev, const VmProgLaunch& L) {
  const VmLaunch& B = L.base;
  if (B.n_ops <= 0) return;
  VmProgArgs a{{B.ops, B.n_ops, B.ext, B.file, B.nw, B.last_mask, nullptr}, L.state, L.n_iregs};
  const int threads = vm_threads(B.nw);
  const int64_t smem = vm_smem_bytes(B.n_slots, B.nw);
  set_smem_attr();
  ProfScope prof(dev, "k_vm_program");
  if (smem > 0) {
    k_vm_program<true><<<1, threads, static_cast<size_t>(smem), dev.stream()>>>(a);
  } else {
    if (!B.file && B.n_slots > 0) throw std::invalid_argument("vm: slot file does not fit in shared memory");
    k_vm_program<false><<<1, threads, 0, dev.stream()>>>(a);
  }
  check_vm_launch("vm program");
  ++dev.n_launches;
}

}  // namespace bsz
