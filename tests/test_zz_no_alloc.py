"""bsz_add_noalloc: stream addition for callers that cannot allocate GPU memory.

A serving process whose memory pool already holds nearly all of HBM, or a host
application that passes in its own buffers and owns every allocation, cannot
let a library call cudaMalloc behind its back.  bsz_add_noalloc keeps its
carry look-back scratch in a fixed device array instead.  This test calls it
through the C ABI twice in a row (a long stream, then a shorter one, so stale
scratch from the first call would show up in the second) and checks each
result against the existing bsz_op_add entry point.  The arithmetic is
integer, so the tolerance is zero: the words must be identical.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import bitstreamzoo_b200 as bz  # noqa: E402
from bitstreamzoo_b200 import _lib  # noqa: E402


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    # mostly-ones second operand: carries run across many 2048-word tiles
    b = np.full(n, np.uint64(2**64 - 1), dtype=np.uint64)
    zeros = rng.integers(0, n, size=max(1, n // 5000))
    b[zeros] = rng.integers(0, 2**64, size=zeros.size, dtype=np.uint64)
    a[: min(n, 3000)] = np.uint64(2**64 - 1)   # one long propagate run from word 0
    b[0] = np.uint64(1)
    return (torch.from_numpy(a.view(np.int64)).cuda(), torch.from_numpy(b.view(np.int64)).cuda())


@pytest.mark.gpu
def test_noalloc_add_matches_op_add_on_two_calls():
    lib = _lib.load()
    ctx = bz.Context(0)
    for call, (n, nbits) in enumerate([((1 << 20) + 3, 64 * ((1 << 20) + 3) - 7),
                                       ((1 << 15) + 1, 64 * ((1 << 15) + 1))]):
        a, b = _inputs(n, seed=call)
        ref = torch.empty(n, dtype=torch.int64, device="cuda")
        out = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        ctx.op("add", ref.data_ptr(), a.data_ptr(), b.data_ptr(), n, nbits)
        ctx.sync()
        rc = lib.bsz_add_noalloc(out.data_ptr(), a.data_ptr(), b.data_ptr(), n, nbits, None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), f"call {call}: first mismatch at word " \
            f"{int((out != ref).nonzero()[0])}"


@pytest.mark.gpu
def test_noalloc_add_rejects_streams_beyond_its_scratch():
    lib = _lib.load()
    too_long = (1 << 26) + 1
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = lib.bsz_add_noalloc(dummy, dummy, dummy, too_long, 64 * too_long, None)
    assert rc != 0
    assert "exceeds the maximum" in _lib.last_error()
