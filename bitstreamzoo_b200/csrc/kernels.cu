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
// The tile is one WARP's: kAddSteps consecutive 32-word steps (kAddTile
// words; lane = word in a step, so every load and store is a coalesced
// 256-byte warp access, kAddSteps of each in flight per operand).  A CTA
// draws one ticket for kAddWarps consecutive tiles (same-address atomics
// serialize, so one per warp would cost ~5 ns x 2^17 tiles); after that its
// warps are independent.
//
// Carry into a tile.  The word just before the tile decides it whenever that
// word does not propagate (a ^ b != ~0: then its carry out is its own
// overflow, whatever comes in), so almost every tile reads that one word and
// needs nothing from any other tile.  Only a tile whose preceding word
// propagates resolves its carry in by decoupled look-back: it publishes its
// aggregate, walks back over its predecessors' status words (flag | g |
// p<<1; bounded spins, a wait that runs out sets kErrLookbackTimeout) and
// publishes its inclusive carry out.  Every tile publishes its inclusive
// carry out as soon as it is known, so a look-back stops at the first tile
// before the propagate run.  The ticket order makes every predecessor a tile
// that has started, so a wait always ends.
//
// dst may be a or b exactly (each word is read before it is written, by the
// one thread that writes it); then the word before a tile may already hold
// its sum, so that call resolves every carry in by look-back (in_place).
// Partial overlaps are not allowed.
//
// Carry resolution inside a step: per word, generate g (the sum with no
// carry in overflowed) and propagate p (a ^ b is all ones: then, and only
// then, the carry out equals the carry in).  The carries into the 32 lanes
// are the internal carries of the 32-bit addition (G|P) + G + cin: carry
// into lane i = bit i of ((G|P)+G+cin) ^ P, carry out = bit 32.  Across
// steps the (g, p) pairs compose.
constexpr int kAddWarps = 8;   // warps per CTA (independent tiles)
constexpr int kAddSteps = 8;   // 256-word tiles; 16-step tiles need ~150 registers (one CTA per SM)
constexpr int kAddMinBlocks = 2;
constexpr int64_t kAddTile = kAddSteps * 32;
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

// Decoupled look-back for `tile` (> 0) with aggregate (tg, tp): returns the
// carry into the tile and publishes the tile's inclusive carry out.
__device__ __forceinline__ uint32_t add_lookback(uint32_t* status, int64_t tile, uint32_t tg, uint32_t tp,
                                                 uint32_t* err, int spin_limit) {
  st_volatile(&status[tile], kFlagAgg | tg | (tp << 1));
  uint32_t ag = 0, ap = 1, cin = 0;
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
  st_volatile(&status[tile], kFlagInc | (tg | (tp & cin)));
  return cin;
}

__global__ void __launch_bounds__(kAddWarps * 32, kAddMinBlocks)
k_add(uint64_t* d, const uint64_t* a, const uint64_t* b, int64_t n, uint64_t last_mask,
      uint32_t* __restrict__ state, uint32_t* __restrict__ err, int in_place, int64_t silent_tile,
      int spin_limit) {
  __shared__ uint32_t s_ticket;
  if (threadIdx.x == 0) s_ticket = atomicAdd(&state[0], 1u);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t tile = static_cast<int64_t>(s_ticket) * kAddWarps + (threadIdx.x >> 5);
  const int64_t base = tile * kAddTile;
  if (base >= n) return;   // a whole warp past the end (grid rounding)
  // the word before the tile (not in place: nobody writes it during the call)
  uint64_t ha = 0, hb = 0;
  if (lane == 0 && tile > 0 && !in_place) {
    ha = a[base - 1];
    hb = b[base - 1];
  }
  uint64_t x[kAddSteps], y[kAddSteps];
#pragma unroll
  for (int j = 0; j < kAddSteps; ++j) {
    const int64_t w = base + lane + j * 32;
    x[j] = 0;
    y[j] = 0;
    if (w < n) {
      x[j] = a[w];
      y[j] = b[w];
    }
  }
  uint32_t G[kAddSteps], P[kAddSteps];
#pragma unroll
  for (int j = 0; j < kAddSteps; ++j) {
    const uint64_t sj = x[j] + y[j];
    G[j] = __ballot_sync(0xffffffffu, sj < x[j]);
    // words past n are zero in both operands, so they never propagate
    P[j] = __ballot_sync(0xffffffffu, (x[j] ^ y[j]) == ~uint64_t(0));
    x[j] = sj;
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
    } else if (!in_place && (ha ^ hb) != ~uint64_t(0)) {
      cin = (ha + hb) < ha;   // the preceding word's own overflow is its carry out
      st_volatile(&status[tile], kFlagInc | (tg | (tp & cin)));
    } else {
      cin = add_lookback(status, tile, tg, tp, err, spin_limit);
    }
  }
  uint32_t c = __shfl_sync(0xffffffffu, cin, 0);
#pragma unroll
  for (int j = 0; j < kAddSteps; ++j) {
    const uint64_t z = static_cast<uint64_t>(G[j] | P[j]) + G[j] + c;
    const uint32_t carries = static_cast<uint32_t>(z) ^ P[j];
    c = static_cast<uint32_t>(z >> 32);
    const int64_t w = base + lane + j * 32;
    if (w < n) {
      uint64_t r = x[j] + ((carries >> lane) & 1u);
      if (w == n - 1) r &= last_mask;
      d[w] = r;
    }
  }
}


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

static void launch_add_kernel(cudaStream_t stream, uint64_t* d, const uint64_t* a, const uint64_t* b,
                              int64_t n, uint64_t last_mask, uint32_t* state, uint32_t* err) {
  const int64_t tiles = (n + kAddTile - 1) / kAddTile;
  if (tiles > 0x7fffffff) throw std::invalid_argument("launch_add: stream too long");
  const int in_place = (d == a || d == b) ? 1 : 0;
  // one warp per tile, one ticket per CTA of kAddWarps tiles
  const int64_t blocks = (tiles + kAddWarps - 1) / kAddWarps;
  if (blocks > 0x7fffffff) throw std::invalid_argument("launch_add: stream too long");
  k_add<<<static_cast<unsigned>(blocks), kAddWarps * 32, 0, stream>>>(d, a, b, n, last_mask, state, err, in_place,
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
