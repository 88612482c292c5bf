/*
 * CPU oracle, word level.  TEST INFRASTRUCTURE ONLY: used by tests/, by
 * __graft_entry__.smoke() and by the CPU-baseline legs of bench.py as the
 * checker / CPU port.  The product (libbsz) never links or calls it.
 *
 * A stream of bitlength N is stored as n = ceil(N/64) little-endian uint64
 * words (bit i -> word i/64, bit i%64).  Beyond the stored words a stream
 * carries a "tail" bit: every bit >= 64*n equals it (Python's negative ints).
 *
 * The arithmetic restates the reference's scalar CPU data plane and its
 * normative Python semantics:
 *   - pointwise ops          simulator/csim/src/bitstream_ops.cpp:68-110
 *   - ripple-carry add       simulator/csim/src/bitstream_ops.cpp:59-66
 *   - cross-word shifts      simulator/csim/src/bitstream_ops.cpp:112-160
 *   - bounded popcount       simulator/csim/src/cpu_backend.h:111-120
 *   - masking of ~ + <<      simulator/pythonsim/interpreter.py:176-210
 * Shifts and ~ clear the bits at and above N, as Python masks them; >> fills
 * from the tail, as Python's arithmetic right shift of a negative int does.
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline uint64_t last_mask(int64_t nbits) {
    int r = (int)(nbits & 63);
    return r ? ((UINT64_C(1) << r) - 1) : ~UINT64_C(0);
}

/* Clear bits >= nbits of an n-word stream (Python's "& mask"). */
void o_mask(uint64_t *d, int64_t n, int64_t nbits) {
    if (n <= 0 || nbits <= 0) return;
    int64_t lw = (nbits + 63) / 64;
    if (lw > n) return;
    d[lw - 1] &= last_mask(nbits);
    for (int64_t i = lw; i < n; ++i) d[i] = 0;
}

void o_and(uint64_t *d, const uint64_t *a, const uint64_t *b, int64_t n) {
    #pragma omp parallel for schedule(static) if (n > (1 << 16))
    for (int64_t i = 0; i < n; ++i) d[i] = a[i] & b[i];
}

void o_or(uint64_t *d, const uint64_t *a, const uint64_t *b, int64_t n) {
    #pragma omp parallel for schedule(static) if (n > (1 << 16))
    for (int64_t i = 0; i < n; ++i) d[i] = a[i] | b[i];
}

void o_xor(uint64_t *d, const uint64_t *a, const uint64_t *b, int64_t n) {
    #pragma omp parallel for schedule(static) if (n > (1 << 16))
    for (int64_t i = 0; i < n; ++i) d[i] = a[i] ^ b[i];
}

/* ~a masked to nbits */
void o_not(uint64_t *d, const uint64_t *a, int64_t n, int64_t nbits) {
    #pragma omp parallel for schedule(static) if (n > (1 << 16))
    for (int64_t i = 0; i < n; ++i) d[i] = ~a[i];
    o_mask(d, n, nbits);
}

/* (a + b) mod 2^nbits, ripple carry through a 128-bit accumulator. */
void o_add(uint64_t *d, const uint64_t *a, const uint64_t *b, int64_t n, int64_t nbits) {
    unsigned __int128 carry = 0;
    for (int64_t i = 0; i < n; ++i) {
        unsigned __int128 t = (unsigned __int128)a[i] + b[i] + carry;
        d[i] = (uint64_t)t;
        carry = t >> 64;
    }
    o_mask(d, n, nbits);
}

/* (a << k) masked to nbits; bits below k are zero.  d may alias a. */
void o_shl(uint64_t *d, const uint64_t *a, int64_t k, int64_t n, int64_t nbits) {
    int64_t ws = k / 64;
    int bs = (int)(k % 64);
    for (int64_t i = n - 1; i >= 0; --i) {
        int64_t lo = i - ws, hi = lo - 1;
        uint64_t wl = (lo >= 0 && lo < n) ? a[lo] : 0;
        uint64_t wh = (hi >= 0 && hi < n) ? a[hi] : 0;
        d[i] = bs ? ((wl << bs) | (wh >> (64 - bs))) : wl;
    }
    o_mask(d, n, nbits);
}

/* a >> k; bits read beyond the stored words come from the tail.  d may alias a. */
void o_shr(uint64_t *d, const uint64_t *a, int64_t k, int64_t n, int tail) {
    uint64_t fill = tail ? ~UINT64_C(0) : 0;
    int64_t ws = k / 64;
    int bs = (int)(k % 64);
    for (int64_t i = 0; i < n; ++i) {
        int64_t lo = i + ws, hi = lo + 1;
        uint64_t wl = (lo < n) ? a[lo] : fill;
        uint64_t wh = (hi < n) ? a[hi] : fill;
        d[i] = bs ? ((wl >> bs) | (wh << (64 - bs))) : wl;
    }
}

int64_t o_popcount(const uint64_t *a, int64_t n) {
    int64_t c = 0;
    #pragma omp parallel for reduction(+:c) schedule(static) if (n > (1 << 16))
    for (int64_t i = 0; i < n; ++i) c += __builtin_popcountll(a[i]);
    return c;
}

int o_any(const uint64_t *a, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (a[i]) return 1;
    return 0;
}

/*
 * Straight-line op-list evaluator over a register file of n-word streams,
 * the oracle used for large straight-line programs (the Python big-int
 * oracle is used for everything with control flow and for small sizes).
 *
 * ops: 5 int64 per op {code, dst, a, b, imm}
 *   code 0 COPY   dst = a
 *        1 NOT    dst = ~a (masked)
 *        2 AND    3 OR    4 XOR
 *        5 ADD    dst = a + b (masked)
 *        6 SHL    dst = a << imm (masked)
 *        7 SHR    dst = a >> imm, tail of a given by b (0/1)
 *        8 POP    pops[imm] = popcount(a)
 *        9 ZERO   dst = 0           10 ONES dst = N-bit mask
 *       11 ALL1   dst = all ones (the copy of ONES; tail handled by caller)
 * regs: array of register base pointers.
 * Returns 0, or -1 on an unknown op code.
 */
int o_run_ops(const int64_t *ops, int64_t n_ops, uint64_t **regs, int64_t n,
              int64_t nbits, int64_t *pops) {
    for (int64_t j = 0; j < n_ops; ++j) {
        const int64_t *o = ops + 5 * j;
        uint64_t *d = regs[o[1]];
        const uint64_t *a = o[2] >= 0 ? regs[o[2]] : NULL;
        const uint64_t *b = (o[3] >= 0 && o[0] != 7) ? regs[o[3]] : NULL;
        switch (o[0]) {
        case 0: if (d != a) memcpy(d, a, (size_t)n * 8); break;
        case 1: o_not(d, a, n, nbits); break;
        case 2: o_and(d, a, b, n); break;
        case 3: o_or(d, a, b, n); break;
        case 4: o_xor(d, a, b, n); break;
        case 5: o_add(d, a, b, n, nbits); break;
        case 6: o_shl(d, a, o[4], n, nbits); break;
        case 7: o_shr(d, a, o[4], n, (int)o[3]); break;
        case 8: pops[o[4]] = o_popcount(a, n); break;
        case 9: memset(d, 0, (size_t)n * 8); break;
        case 10: memset(d, 0xFF, (size_t)n * 8); o_mask(d, n, nbits); break;
        case 11: memset(d, 0xFF, (size_t)n * 8); break;
        default: return -1;
        }
    }
    return 0;
}

int o_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
