"""CPU restatement of the regex app's byte -> basis-bit transposition.

TEST INFRASTRUCTURE ONLY: the checker for the device S2P kernel, never
called by the product path.

Follows ``payload_to_basis_bits`` (benchmark/apps/regex/src/run.py:164-173):
basis stream i has bit j set exactly when bit i of byte j is set.  Two
restatements: ``basis_ints`` is the reference's loop over Python ints (small
inputs only); ``basis_words`` does the same per bit plane with numpy
(``payload_to_basis_bits_fast``, run.py:176-187) and returns each stream as
little-endian uint64 words, ceil(n/64) of them, zero above bit n.
"""

from __future__ import annotations

import numpy as np


def basis_ints(payload: bytes) -> list[int]:
    out = []
    for i in range(8):
        v = 0
        for j, byte in enumerate(payload):
            if (byte >> i) & 1:
                v |= 1 << j
        out.append(v)
    return out


def basis_words(payload) -> list[np.ndarray]:
    arr = np.frombuffer(bytes(payload), dtype=np.uint8) if not isinstance(payload, np.ndarray) else payload
    n = arr.size
    nw = (n + 63) // 64
    out = []
    for i in range(8):
        bits = ((arr >> i) & 1).astype(np.uint8)
        packed = np.packbits(bits, bitorder="little")
        buf = np.zeros(nw * 8, dtype=np.uint8)
        buf[: packed.size] = packed
        out.append(buf.view("<u8").astype(np.uint64))
    return out
