// Register transposition of 64 bytes into 8 basis-bit words (s2p.cu).
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

#ifdef __CUDA_ARCH__
#define BSZ_UNROLL _Pragma("unroll")
#else
#define BSZ_UNROLL
#endif

namespace bsz {

// Transposes the 64 bytes in x[0..7] (x[q] = bytes 8q..8q+7) into the eight
// basis words: afterwards x[i] bit (8q + k) = bit i of byte (8q + k).
__host__ __device__ __forceinline__ void s2p_transpose64(uint64_t x[8]) {
BSZ_UNROLL
  for (int q = 0; q < 8; ++q) {
    uint64_t v = x[q], t;
    // bit (8r + c) <-> bit (8c + r)
    t = (v ^ (v >> 7)) & 0x00AA00AA00AA00AAull;
    v ^= t ^ (t << 7);
    t = (v ^ (v >> 14)) & 0x0000CCCC0000CCCCull;
    v ^= t ^ (t << 14);
    t = (v ^ (v >> 28)) & 0x00000000F0F0F0F0ull;
    v ^= t ^ (t << 28);
    x[q] = v;
  }
  // byte matrix transpose: row q, column i -> row i, column q
BSZ_UNROLL
  for (int q = 0; q < 4; ++q) {
    const uint64_t a = x[q], b = x[q + 4];
    x[q] = (a & 0x00000000FFFFFFFFull) | (b << 32);
    x[q + 4] = (a >> 32) | (b & 0xFFFFFFFF00000000ull);
  }
BSZ_UNROLL
  for (int h = 0; h < 4; ++h) {
    const int q = (h & 1) | ((h & 2) << 1);   // 0, 1, 4, 5
    const uint64_t a = x[q], b = x[q + 2];
    constexpr uint64_t m = 0x0000FFFF0000FFFFull;
    x[q] = (a & m) | ((b & m) << 16);
    x[q + 2] = ((a >> 16) & m) | (b & ~m);
  }
BSZ_UNROLL
  for (int h = 0; h < 4; ++h) {
    const int q = 2 * h;
    const uint64_t a = x[q], b = x[q + 1];
    constexpr uint64_t m = 0x00FF00FF00FF00FFull;
    x[q] = (a & m) | ((b & m) << 8);
    x[q + 1] = ((a >> 8) & m) | (b & ~m);
  }
}

}  // namespace bsz
