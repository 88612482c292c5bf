// Device-side segment interpreter for short streams.
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
// Every instruction has the exact semantics of the per-op kernel for the
// same node (masking of ~, + and << at the last word; >> filling with the
// operand's tail), so results are bit-identical to the plain form.
#include "vm.h"

#include <algorithm>
#include <mutex>
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
  o.pad = 0;
  o.dst = v.y;
  o.a = v.z;
  o.b = v.w;
  return o;
}

template <bool SMEM>
__global__ void __launch_bounds__(1024) k_vm(VmArgs args) {
  extern __shared__ uint64_t s_file[];
  __shared__ uint32_t s_g[32], s_p[32];
  uint64_t* file = SMEM ? s_file : args.file;
  const int T = blockDim.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, n_warps = T >> 5;
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
      case kVmNot: {
        uint64_t* D = loc(op.dst);
        for (int64_t w = tid; w < nw; w += T) {
          uint64_t r = ~A[w];
          if (w == nw - 1) r &= lm;
          D[w] = r;
        }
        break;
      }
      case kVmAnd: case kVmOr: case kVmXor: case kVmAndNot: {
        uint64_t* D = loc(op.dst);
        const uint64_t* B = loc(op.b);
        for (int64_t w = tid; w < nw; w += T) {
          const uint64_t x = A[w], y = B[w];
          D[w] = op.code == kVmAnd ? (x & y) : op.code == kVmOr ? (x | y) : op.code == kVmXor ? (x ^ y) : (x & ~y);
        }
        break;
      }
      case kVmShl: {
        uint64_t* D = loc(op.dst);
        const int64_t ws = op.b >> 6;
        const int bs = op.b & 63;
        for (int64_t w = tid; w < nw; w += T) {
          const int64_t lo = w - ws;
          const uint64_t x = lo >= 0 ? A[lo] : 0;
          const uint64_t y = (bs && lo >= 1) ? A[lo - 1] : 0;
          uint64_t r = bs ? ((x << bs) | (y >> (64 - bs))) : x;
          if (w == nw - 1) r &= lm;
          D[w] = r;
        }
        break;
      }
      case kVmShr: {
        uint64_t* D = loc(op.dst);
        const int64_t ws = op.b >> 6;
        const int bs = op.b & 63;
        const uint64_t fill = op.fill ? ~uint64_t(0) : 0;
        for (int64_t w = tid; w < nw; w += T) {
          const int64_t lo = w + ws;
          const uint64_t x = lo < nw ? A[lo] : fill;
          const uint64_t y = bs ? (lo + 1 < nw ? A[lo + 1] : fill) : 0;
          D[w] = bs ? ((x >> bs) | (y << (64 - bs))) : x;
        }
        break;
      }
      case kVmAdd: {
        uint64_t* D = loc(op.dst);
        const uint64_t* B = loc(op.b);
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
        break;
      }
      case kVmPop: {
        unsigned long long c = 0;
        for (int64_t w = tid; w < nw; w += T) c += __popcll(A[w]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0 && c) atomicAdd(args.pops + op.dst, c);
        break;
      }
      default:
        break;
    }
    if (n_warps > 1) __syncthreads();
    else __syncwarp();
  }
}

int vm_threads(int64_t nw) {
  const int64_t t = ((nw + 31) / 32) * 32;
  return static_cast<int>(std::max<int64_t>(32, std::min<int64_t>(1024, t)));
}

std::once_flag g_smem_attr;

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
  std::call_once(g_smem_attr, [] {
    cudaFuncSetAttribute(k_vm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kVmSmemLimit));
  });
  ProfScope prof(dev, "k_vm");
  if (smem > 0) {
    k_vm<true><<<1, threads, static_cast<size_t>(smem), dev.stream()>>>(a);
  } else {
    if (!L.file && L.n_slots > 0) throw std::invalid_argument("vm: slot file does not fit in shared memory");
    k_vm<false><<<1, threads, 0, dev.stream()>>>(a);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw CudaError(std::string("vm launch failed: ") + cudaGetErrorString(e));
  ++dev.n_launches;
}

}  // namespace bsz
