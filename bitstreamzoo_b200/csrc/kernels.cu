// Plain per-op kernels for sm_100a: one launch per DSL operation.
//
// Layout: a stream is n little-endian uint64 words (bit i -> word i/64).
// Every kernel here is HBM-bound integer work, so the design goals are
// coalesced 128-bit accesses, enough bytes in flight per SM (several
// independent 16-byte loads per thread), grids sized in multiples of the SM
// count, and no extra passes over HBM:
//   AND/OR/XOR/ANDNOT/NOT   16 B vector loads, 4 in flight per thread
//   SHL/SHR                 one output word per lane, the neighbour word
//                           comes from L1 (both loads are warp-coalesced)
//   ADD                     single pass: 4-word blocks per lane (256-bit
//                           accesses), per-warp ballot carry resolution
//                           + decoupled look-back across CTAs (24 B/word,
//                           the reference's CUB scan path moves ~120 B/word)
//   POPCOUNT / ANY          one pass, one atomic per CTA, no host sync
#include "device.h"

#include <algorithm>

namespace bsz {
namespace {

constexpr int kThreads = 256;
constexpr int kUnroll = 4;

int grid_for(const Device& dev, int64_t work_items, int per_block) {
  int64_t want = (work_items + per_block - 1) / per_block;
  int64_t cap = static_cast<int64_t>(dev.sm_count()) * 8;
  return static_cast<int>(std::max<int64_t>(1, std::min(want, cap)));
}

void check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw CudaError(std::string("kernel launch failed: ") + cudaGetErrorString(e));
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <int OP>
__device__ __forceinline__ uint64_t apply_op(uint64_t x, uint64_t y) {
  if constexpr (OP == kAnd) return x & y;
  if constexpr (OP == kOr) return x | y;
  if constexpr (OP == kXor) return x ^ y;
  return x & ~y;
}

// OP in {And, Or, Xor, AndNot}; OP == 4 means NOT (b unused).
template <int OP>
__device__ __forceinline__ uint64_t apply_any(uint64_t x, uint64_t y) {
  if constexpr (OP == 4) return ~x;
  else return apply_op<OP>(x, y);
}

// Words [0, 2*nvec) in 16-byte pairs; words [2*nvec, n) (one or two words,
// the second of which is the last word and gets last_mask) by one thread.
template <int OP>
__global__ void __launch_bounds__(kThreads)
k_map_vec(uint64_t* __restrict__ d, const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
          int64_t n, uint64_t last_mask) {
  const int64_t nvec = (n - 1) / 2;
  const ulonglong2* A = reinterpret_cast<const ulonglong2*>(a);
  const ulonglong2* B = reinterpret_cast<const ulonglong2*>(b);
  ulonglong2* D = reinterpret_cast<ulonglong2*>(d);
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads * kUnroll;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * kThreads * kUnroll + threadIdx.x;
       base < nvec; base += step) {
    ulonglong2 x[kUnroll], y[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      int64_t i = base + u * kThreads;
      if (i < nvec) {
        x[u] = A[i];
        if constexpr (OP != 4) y[u] = B[i];
        else y[u] = x[u];
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      int64_t i = base + u * kThreads;
      if (i < nvec) {
        ulonglong2 r;
        r.x = apply_any<OP>(x[u].x, y[u].x);
        r.y = apply_any<OP>(x[u].y, y[u].y);
        D[i] = r;
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int64_t w = 2 * nvec; w < n; ++w) {
      uint64_t r = apply_any<OP>(a[w], OP != 4 ? b[w] : 0);
      if (w == n - 1) r &= last_mask;
      d[w] = r;
    }
  }
}

template <int OP>
__global__ void __launch_bounds__(kThreads)
k_map_scalar(uint64_t* d, const uint64_t* a, const uint64_t* b, int64_t n, uint64_t last_mask) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; w < n; w += step) {
    uint64_t r = apply_any<OP>(a[w], OP != 4 ? b[w] : 0);
    if (w == n - 1) r &= last_mask;
    d[w] = r;
  }
}

template <int OP>
void launch_map(Device& dev, uint64_t* d, const uint64_t* a, const uint64_t* b, int64_t n,
                uint64_t last_mask) {
  if (n <= 0) return;
  static const char* names[] = {"k_and", "k_or", "k_xor", "k_andnot", "k_not"};
  ProfScope prof(dev, names[OP]);
  const bool vec = aligned16(d) && aligned16(a) && (OP == 4 || aligned16(b));
  if (vec) {
    int64_t nvec = (n - 1) / 2;
    int grid = grid_for(dev, std::max<int64_t>(nvec, 1), kThreads * kUnroll);
    k_map_vec<OP><<<grid, kThreads, 0, dev.stream()>>>(d, a, b, n, last_mask);
  } else {
    int grid = grid_for(dev, n, kThreads);
    k_map_scalar<OP><<<grid, kThreads, 0, dev.stream()>>>(d, a, b, n, last_mask);
  }
  check_launch();
  ++dev.n_launches;
}

// ---- shifts --------------------------------------------------------------
// Left shift by k = 64*ws + bs (toward higher bit positions):
//   r[w] = (a[w-ws] << bs) | (a[w-ws-1] >> (64-bs)), zeros below, masked.
__global__ void __launch_bounds__(kThreads)
k_shl(uint64_t* __restrict__ d, const uint64_t* __restrict__ a, int64_t ws, int bs, int64_t n,
      uint64_t last_mask) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads * kUnroll;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * kThreads * kUnroll + threadIdx.x;
       base < n; base += step) {
    uint64_t x[kUnroll], y[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      int64_t w = base + u * kThreads;
      int64_t lo = w - ws;
      x[u] = (w < n && lo >= 0) ? a[lo] : 0;
      y[u] = (w < n && lo >= 1 && bs) ? a[lo - 1] : 0;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      int64_t w = base + u * kThreads;
      if (w < n) {
        uint64_t r = bs ? ((x[u] << bs) | (y[u] >> (64 - bs))) : x[u];
        if (w == n - 1) r &= last_mask;
        d[w] = r;
      }
    }
  }
}

// Right shift: r[w] = (a[w+ws] >> bs) | (a[w+ws+1] << (64-bs)); words past the
// end read ``fill`` (the stream's tail: all-zero or all-one).
__global__ void __launch_bounds__(kThreads)
k_shr(uint64_t* __restrict__ d, const uint64_t* __restrict__ a, int64_t ws, int bs, int64_t n,
      uint64_t fill) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads * kUnroll;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * kThreads * kUnroll + threadIdx.x;
       base < n; base += step) {
    uint64_t x[kUnroll], y[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      int64_t w = base + u * kThreads;
      int64_t lo = w + ws;
      x[u] = (w < n) ? (lo < n ? a[lo] : fill) : 0;
      y[u] = (w < n && bs) ? (lo + 1 < n ? a[lo + 1] : fill) : 0;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      int64_t w = base + u * kThreads;
      if (w < n) d[w] = bs ? ((x[u] >> bs) | (y[u] << (64 - bs))) : x[u];
    }
  }
}

// ---- add: single-pass carry scan ----------------------------------------
// The tile of the decoupled look-back is one WARP's: kAddSteps consecutive
// 128-word steps (kAddTile words).  In a step, lane l owns the 4-word block
// at 4l: one 32-byte sector, a 256-bit load or store per lane, so every warp
// access is one contiguous kilobyte.  A CTA draws one ticket for kAddWarps
// consecutive tiles; after that its warps are independent: each publishes its
// aggregate as soon as its loads have landed and resolves its carry in by
// look-back with no CTA barrier, so a warp waiting on its predecessor holds
// up nobody else on the SM.
//
// Carry resolution inside a step: per block, generate g (the block sum with
// no carry in overflowed) and propagate p (a ^ b is all ones over the block:
// then, and only then, the carry out equals the carry in).  The carries into
// the 32 blocks are the internal carries of the 32-bit addition
// (G|P) + G + cin: carry into lane i = bit i of ((G|P)+G+cin) ^ P, carry out
// = bit 32.  Across steps the (g, p) pairs compose; across tiles the status
// word is flag | g | p<<1, with bounded spins.  dst may be a or b exactly
// (each word is read before it is written, by the one thread that writes
// it); partial overlaps are not allowed.
constexpr int kAddWarps = 8;   // warps per CTA (independent tiles)
constexpr int kAddSteps = 4;
constexpr int64_t kAddTile = kAddSteps * 128;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr int kSpinLimit = 1 << 22;

// Test hook: a tile that never publishes its status, and a shorter spin
// limit, so a test can make a look-back wait run out (its successor then
// reports kErrLookbackTimeout).  Off (-1, kSpinLimit) unless a test sets it.
int64_t g_add_silent_tile = -1;
int g_add_spin_limit = kSpinLimit;

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) {
  *reinterpret_cast<volatile uint32_t*>(p) = v;
}

// 4 words at word index w (w % 4 == 0): one 256-bit load when the block is
// whole and the pointer 32-byte aligned, else word by word (zero past n).
// Plain (coherent) loads: dst may alias the operand.
template <bool VEC>
__device__ __forceinline__ void load4(const uint64_t* p, int64_t w, int64_t n, uint64_t r[4]) {
  if (VEC && w + 3 < n) {
    asm volatile("ld.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(r[0]), "=l"(r[1]), "=l"(r[2]), "=l"(r[3])
                 : "l"(p + w));
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) r[i] = (w + i < n) ? p[w + i] : 0;
  }
}

template <bool VEC>
__device__ __forceinline__ void store4(uint64_t* p, int64_t w, int64_t n, const uint64_t r[4]) {
  if (VEC && w + 3 < n) {
    asm volatile("st.global.v4.u64 [%0], {%1,%2,%3,%4};" ::"l"(p + w), "l"(r[0]), "l"(r[1]), "l"(r[2]),
                 "l"(r[3])
                 : "memory");
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (w + i < n) p[w + i] = r[i];
  }
}

#define BSZ_LO(x) static_cast<uint32_t>(x)
#define BSZ_HI(x) static_cast<uint32_t>((x) >> 32)

// s = a + b over a 256-bit block (no carry in); returns the carry out.
__device__ __forceinline__ uint32_t add4(uint64_t s[4], const uint64_t a[4], const uint64_t b[4]) {
  uint32_t r[8], c;
  asm("add.cc.u32 %0, %9, %17;\n\t"
      "addc.cc.u32 %1, %10, %18;\n\t"
      "addc.cc.u32 %2, %11, %19;\n\t"
      "addc.cc.u32 %3, %12, %20;\n\t"
      "addc.cc.u32 %4, %13, %21;\n\t"
      "addc.cc.u32 %5, %14, %22;\n\t"
      "addc.cc.u32 %6, %15, %23;\n\t"
      "addc.cc.u32 %7, %16, %24;\n\t"
      "addc.u32 %8, 0, 0;"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]),
        "=&r"(r[7]), "=&r"(c)
      : "r"(BSZ_LO(a[0])), "r"(BSZ_HI(a[0])), "r"(BSZ_LO(a[1])), "r"(BSZ_HI(a[1])), "r"(BSZ_LO(a[2])),
        "r"(BSZ_HI(a[2])), "r"(BSZ_LO(a[3])), "r"(BSZ_HI(a[3])), "r"(BSZ_LO(b[0])), "r"(BSZ_HI(b[0])),
        "r"(BSZ_LO(b[1])), "r"(BSZ_HI(b[1])), "r"(BSZ_LO(b[2])), "r"(BSZ_HI(b[2])), "r"(BSZ_LO(b[3])),
        "r"(BSZ_HI(b[3])));
#pragma unroll
  for (int i = 0; i < 4; ++i) s[i] = (static_cast<uint64_t>(r[2 * i + 1]) << 32) | r[2 * i];
  return c;
}

// s += c (c in {0, 1}) over a 256-bit block.
__device__ __forceinline__ void inc4(uint64_t s[4], uint32_t c) {
  uint32_t r[8];
  asm("add.cc.u32 %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, 0;\n\t"
      "addc.cc.u32 %2, %10, 0;\n\t"
      "addc.cc.u32 %3, %11, 0;\n\t"
      "addc.cc.u32 %4, %12, 0;\n\t"
      "addc.cc.u32 %5, %13, 0;\n\t"
      "addc.cc.u32 %6, %14, 0;\n\t"
      "addc.u32 %7, %15, 0;"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]),
        "=&r"(r[7])
      : "r"(BSZ_LO(s[0])), "r"(BSZ_HI(s[0])), "r"(BSZ_LO(s[1])), "r"(BSZ_HI(s[1])), "r"(BSZ_LO(s[2])),
        "r"(BSZ_HI(s[2])), "r"(BSZ_LO(s[3])), "r"(BSZ_HI(s[3])), "r"(c));
#pragma unroll
  for (int i = 0; i < 4; ++i) s[i] = (static_cast<uint64_t>(r[2 * i + 1]) << 32) | r[2 * i];
}

template <bool VEC>
__global__ void __launch_bounds__(kAddWarps * 32)
k_add(uint64_t* d, const uint64_t* a, const uint64_t* b, int64_t n, uint64_t last_mask,
      uint32_t* __restrict__ state, uint32_t* __restrict__ err, int64_t silent_tile, int spin_limit) {
  // one ticket per CTA (same-address atomics serialize: one per warp would
  // cost ~5 ns x 2^17 tiles); its warps take the CTA's kAddWarps tiles
  __shared__ uint32_t s_ticket;
  if (threadIdx.x == 0) s_ticket = atomicAdd(&state[0], 1u);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t tile = static_cast<int64_t>(s_ticket) * kAddWarps + (threadIdx.x >> 5);
  const int64_t wbase = tile * kAddTile + 4 * lane;
  if (tile * kAddTile >= n) return;   // a whole warp past the end (grid rounding)
  uint64_t sum[kAddSteps][4];
  uint32_t G[kAddSteps], P[kAddSteps];
  {
    uint64_t x[kAddSteps][4], y[kAddSteps][4];
#pragma unroll
    for (int j = 0; j < kAddSteps; ++j) {
      load4<VEC>(a, wbase + j * 128, n, x[j]);
      load4<VEC>(b, wbase + j * 128, n, y[j]);
    }
#pragma unroll
    for (int j = 0; j < kAddSteps; ++j) {
      const uint32_t g = add4(sum[j], x[j], y[j]);
      const uint64_t q = (x[j][0] ^ y[j][0]) & (x[j][1] ^ y[j][1]) & (x[j][2] ^ y[j][2]) & (x[j][3] ^ y[j][3]);
      G[j] = __ballot_sync(0xffffffffu, g != 0);
      // words past n are zero in both operands, so their blocks never propagate
      P[j] = __ballot_sync(0xffffffffu, q == ~uint64_t(0));
    }
  }
  // the tile's aggregate over its steps (in word order)
  uint32_t tg = 0, tp = 1;
#pragma unroll
  for (int j = 0; j < kAddSteps; ++j) {
    const uint64_t z = static_cast<uint64_t>(G[j] | P[j]) + G[j];
    const uint32_t sg = static_cast<uint32_t>(z >> 32);
    const uint32_t sp = P[j] == 0xffffffffu;
    tg = sg | (sp & tg);
    tp &= sp;
  }
  uint32_t cin = 0;
  if (lane == 0 && tile != silent_tile) {
    uint32_t* status = state + 1;
    if (tile == 0) {
      st_volatile(&status[0], kFlagInc | tg);
    } else {
      st_volatile(&status[tile], kFlagAgg | tg | (tp << 1));
      // walk back: (ag, ap) = composition of the tiles between j and this one
      uint32_t ag = 0, ap = 1;
      int64_t j = tile - 1;
      int spins = 0;
      while (true) {
        const uint32_t v = ld_volatile(&status[j]);
        const uint32_t f = v & kFlagMask;
        if (f == 0) {
          if (++spins > spin_limit) {
            atomicOr(err, kErrLookbackTimeout);
            cin = 0;
            break;
          }
          __nanosleep(32);
          continue;
        }
        if (f == kFlagInc) {
          cin = ag | (ap & (v & 1u));
          break;
        }
        const uint32_t g = v & 1u, p = (v >> 1) & 1u;
        ag = ag | (ap & g);
        ap &= p;
        if (!ap) {   // the carry out of the walked range no longer depends on earlier tiles
          cin = ag;
          break;
        }
        --j;
        spins = 0;
      }
      __threadfence();
      st_volatile(&status[tile], kFlagInc | (tg | (tp & cin)));
    }
  }
  uint32_t c = __shfl_sync(0xffffffffu, cin, 0);
#pragma unroll
  for (int j = 0; j < kAddSteps; ++j) {
    const uint64_t z = static_cast<uint64_t>(G[j] | P[j]) + G[j] + c;
    const uint32_t carries = static_cast<uint32_t>(z) ^ P[j];
    c = static_cast<uint32_t>(z >> 32);
    const int64_t w = wbase + j * 128;
    if (w < n) {
      inc4(sum[j], (carries >> lane) & 1u);
      if (w + 3 >= n - 1) {   // this block holds the last word
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (w + i == n - 1) sum[j][i] &= last_mask;
      }
      store4<VEC>(d, w, n, sum[j]);
    }
  }
}

#undef BSZ_LO
#undef BSZ_HI

// ---- reductions ------------------------------------------------------------
__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kThreads)
k_popcount(const uint64_t* __restrict__ a, int64_t n, unsigned long long* __restrict__ slot,
           int vec) {
  __shared__ uint64_t s_part[kThreads / 32];
  uint64_t c = 0;
  if (vec) {
    const int64_t npairs = n / 2;
    const ulonglong2* A = reinterpret_cast<const ulonglong2*>(a);
    const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads * kUnroll;
    for (int64_t base = static_cast<int64_t>(blockIdx.x) * kThreads * kUnroll + threadIdx.x;
         base < npairs; base += step) {
      ulonglong2 x[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        int64_t i = base + u * kThreads;
        x[u] = i < npairs ? A[i] : make_ulonglong2(0, 0);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) c += __popcll(x[u].x) + __popcll(x[u].y);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) c += __popcll(a[n - 1]);
  } else {
    const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads;
    for (int64_t w = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; w < n; w += step)
      c += __popcll(a[w]);
  }
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint64_t v = threadIdx.x < kThreads / 32 ? s_part[threadIdx.x] : 0;
    v = warp_sum(v);
    if (threadIdx.x == 0 && v) atomicAdd(slot, static_cast<unsigned long long>(v));
  }
}

__global__ void __launch_bounds__(kThreads)
k_any(const uint64_t* __restrict__ a, int64_t n, unsigned int* __restrict__ flag) {
  uint64_t acc = 0;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; w < n; w += step)
    acc |= a[w];
  if (__any_sync(0xffffffffu, acc != 0) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

__global__ void __launch_bounds__(kThreads)
k_fill(uint64_t* __restrict__ d, int64_t n, uint64_t value, uint64_t last_value) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; w < n; w += step)
    d[w] = (w == n - 1) ? last_value : value;
}

}  // namespace

void launch_bitwise(Device& dev, int op, uint64_t* d, const uint64_t* a, const uint64_t* b,
                    int64_t n) {
  switch (op) {
    case kAnd: launch_map<kAnd>(dev, d, a, b, n, ~uint64_t(0)); break;
    case kOr: launch_map<kOr>(dev, d, a, b, n, ~uint64_t(0)); break;
    case kXor: launch_map<kXor>(dev, d, a, b, n, ~uint64_t(0)); break;
    case kAndNot: launch_map<kAndNot>(dev, d, a, b, n, ~uint64_t(0)); break;
    default: throw std::invalid_argument("launch_bitwise: bad op");
  }
}

void launch_not(Device& dev, uint64_t* d, const uint64_t* a, int64_t n, uint64_t last_mask) {
  launch_map<4>(dev, d, a, nullptr, n, last_mask);
}

void launch_shl(Device& dev, uint64_t* d, const uint64_t* a, int64_t k, int64_t n,
                uint64_t last_mask) {
  if (n <= 0) return;
  int64_t ws = std::min<int64_t>(k / 64, n + 1);
  int bs = static_cast<int>(k % 64);
  int grid = grid_for(dev, n, kThreads * kUnroll);
  ProfScope prof(dev, "k_shl");
  k_shl<<<grid, kThreads, 0, dev.stream()>>>(d, a, ws, bs, n, last_mask);
  check_launch();
  ++dev.n_launches;
}

void launch_shr(Device& dev, uint64_t* d, const uint64_t* a, int64_t k, int64_t n, uint64_t fill) {
  if (n <= 0) return;
  int64_t ws = std::min<int64_t>(k / 64, n + 1);
  int bs = static_cast<int>(k % 64);
  int grid = grid_for(dev, n, kThreads * kUnroll);
  ProfScope prof(dev, "k_shr");
  k_shr<<<grid, kThreads, 0, dev.stream()>>>(d, a, ws, bs, n, fill);
  check_launch();
  ++dev.n_launches;
}

int64_t add_state_words(int64_t n) { return 1 + (n + kAddTile - 1) / kAddTile; }

static bool aligned32(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31) == 0; }

static void launch_add_kernel(cudaStream_t stream, uint64_t* d, const uint64_t* a, const uint64_t* b,
                              int64_t n, uint64_t last_mask, uint32_t* state, uint32_t* err) {
  const int64_t tiles = (n + kAddTile - 1) / kAddTile;
  if (tiles > 0x7fffffff) throw std::invalid_argument("launch_add: stream too long");
  const bool vec = aligned32(d) && aligned32(a) && aligned32(b);
  auto k = vec ? k_add<true> : k_add<false>;
  // one warp per tile (each warp draws its own ticket)
  const int64_t blocks = (tiles + kAddWarps - 1) / kAddWarps;
  if (blocks > 0x7fffffff) throw std::invalid_argument("launch_add: stream too long");
  k<<<static_cast<unsigned>(blocks), kAddWarps * 32, 0, stream>>>(d, a, b, n, last_mask, state, err,
                                                                  g_add_silent_tile, g_add_spin_limit);
  check_launch();
}

void launch_add_with_state(Device& dev, uint64_t* d, const uint64_t* a, const uint64_t* b,
                           int64_t n, uint64_t last_mask, uint32_t* state) {
  if (n <= 0) return;
  ProfScope prof(dev, "k_add");
  launch_add_kernel(dev.stream(), d, a, b, n, last_mask, state, dev.error_word());
  ++dev.n_launches;
}

void launch_add_on_stream(cudaStream_t stream, uint64_t* d, const uint64_t* a, const uint64_t* b,
                          int64_t n, uint64_t last_mask, uint32_t* state, uint32_t* err) {
  if (n <= 0) return;
  launch_add_kernel(stream, d, a, b, n, last_mask, state, err);
}

void set_add_lookback_test_hook(int64_t silent_tile, int spin_limit) {
  g_add_silent_tile = silent_tile;
  g_add_spin_limit = spin_limit > 0 ? spin_limit : kSpinLimit;
}

void launch_add(Device& dev, uint64_t* d, const uint64_t* a, const uint64_t* b, int64_t n,
                uint64_t last_mask) {
  if (n <= 0) return;
  uint32_t* state = dev.scan_state(add_state_words(n));
  launch_add_with_state(dev, d, a, b, n, last_mask, state);
}

void launch_popcount(Device& dev, const uint64_t* a, int64_t n, unsigned long long* slot) {
  if (n <= 0) return;
  int vec = aligned16(a) ? 1 : 0;
  int grid = grid_for(dev, vec ? std::max<int64_t>(n / 2, 1) : n, kThreads * (vec ? kUnroll : 1));
  ProfScope prof(dev, "k_popcount");
  k_popcount<<<grid, kThreads, 0, dev.stream()>>>(a, n, slot, vec);
  check_launch();
  ++dev.n_launches;
}

void launch_any(Device& dev, const uint64_t* a, int64_t n, unsigned int* flag) {
  if (n <= 0) return;
  int grid = grid_for(dev, n, kThreads * 4);
  ProfScope prof(dev, "k_any");
  k_any<<<grid, kThreads, 0, dev.stream()>>>(a, n, flag);
  check_launch();
  ++dev.n_launches;
}

void launch_fill(Device& dev, uint64_t* d, int64_t n, uint64_t value, uint64_t last_value) {
  if (n <= 0) return;
  int grid = grid_for(dev, n, kThreads * 4);
  ProfScope prof(dev, "k_fill");
  k_fill<<<grid, kThreads, 0, dev.stream()>>>(d, n, value, last_value);
  check_launch();
  ++dev.n_launches;
}

void launch_copy(Device& dev, uint64_t* d, const uint64_t* a, int64_t n) {
  if (n <= 0 || d == a) return;
  BSZ_CUDA(cudaMemcpyAsync(d, a, static_cast<size_t>(n) * 8, cudaMemcpyDeviceToDevice, dev.stream()));
}

}  // namespace bsz
