// Byte -> basis-bit transposition ("serial to parallel") on the device.
//
// Replaces payload_to_basis_bits / payload_to_basis_bits_fast
// (benchmark/apps/regex/src/run.py:164-187): basis stream i holds, at bit j,
// bit i of byte j.  With streams stored as little-endian uint64 words, word w
// of stream i is built from the 64 bytes [64w, 64w+64): one thread per output
// word loads those 64 bytes (four 16-byte loads when the source is aligned)
// and transposes them in registers:
//
//   1. each 8-byte group x_q (bytes 8q..8q+7) is an 8x8 bit matrix (row =
//      byte, column = bit); three masked delta swaps (block sizes 1, 2, 4)
//      transpose it, so byte i of the result holds bit i of the 8 bytes;
//   2. the eight results form an 8x8 byte matrix (row q, column i); three
//      block swaps (32-, 16-, 8-bit halves) transpose it, so word i holds
//      byte i of every group, i.e. bits 64w..64w+63 of basis stream i.
//
// HBM-bound: n bytes in, n bytes out (eight streams of n bits), each warp
// storing 8 coalesced 256-byte rows.  Bytes past n read as zero, so every
// stream's bits at and above n are clean.
#include "device.h"
#include "s2p.h"

#include <algorithm>
#include <stdexcept>
#include <string>

namespace bsz {

namespace {

constexpr int kS2PThreads = 256;

struct BasisOut {
  uint64_t* p[8];
};

// VEC: the byte source is 16-byte aligned, so whole 64-byte groups load as
// four uint4; the group that holds the last byte (and any unaligned source)
// loads byte by byte.
template <bool VEC>
__global__ void __launch_bounds__(kS2PThreads)
k_s2p(const uint8_t* __restrict__ bytes, int64_t n_bytes, int64_t nw, BasisOut out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kS2PThreads;
  const int64_t full = n_bytes / 64;   // words whose 64 bytes all exist
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * kS2PThreads + threadIdx.x; w < nw; w += stride) {
    uint64_t x[8];
    if (VEC && w < full) {
      const uint4* src = reinterpret_cast<const uint4*>(bytes + w * 64);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint4 v = __ldg(src + k);
        x[2 * k] = static_cast<uint64_t>(v.x) | (static_cast<uint64_t>(v.y) << 32);
        x[2 * k + 1] = static_cast<uint64_t>(v.z) | (static_cast<uint64_t>(v.w) << 32);
      }
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint64_t v = 0;
        for (int k = 0; k < 8; ++k) {
          const int64_t j = w * 64 + q * 8 + k;
          if (j < n_bytes) v |= static_cast<uint64_t>(bytes[j]) << (8 * k);
        }
        x[q] = v;
      }
    }
    s2p_transpose64(x);
#pragma unroll
    for (int i = 0; i < 8; ++i) out.p[i][w] = x[i];
  }
}

}  // namespace

void launch_s2p(Device& dev, const uint8_t* bytes, int64_t n_bytes, uint64_t* const* out) {
  if (n_bytes <= 0) return;
  const int64_t nw = (n_bytes + 63) / 64;
  BasisOut o;
  for (int i = 0; i < 8; ++i) {
    if (!out[i]) throw std::invalid_argument("s2p: output stream " + std::to_string(i) + " is null");
    o.p[i] = out[i];
  }
  const int64_t want = (nw + kS2PThreads - 1) / kS2PThreads;
  const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(dev.sm_count()) * 8)));
  ProfScope prof(dev, "k_s2p");
  if ((reinterpret_cast<uintptr_t>(bytes) & 15) == 0)
    k_s2p<true><<<blocks, kS2PThreads, 0, dev.stream()>>>(bytes, n_bytes, nw, o);
  else
    k_s2p<false><<<blocks, kS2PThreads, 0, dev.stream()>>>(bytes, n_bytes, nw, o);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw CudaError(std::string("s2p launch failed: ") + cudaGetErrorString(e));
  ++dev.n_launches;
}

}  // namespace bsz
