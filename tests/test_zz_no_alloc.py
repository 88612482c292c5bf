"""bsz_add_noalloc: stream addition for callers that cannot allocate GPU memory.

A serving process whose memory pool already holds nearly all of HBM, or a host
application that passes in its own buffers and owns every allocation, cannot
let a library call cudaMalloc behind its back.  bsz_add_noalloc keeps its
carry look-back scratch in a fixed device array instead.  These tests call it
through the C ABI twice in a row (a long stream, then a shorter one, so stale
scratch from the first call would show up in the second) and check each
result against the word-level C oracle and against the existing bsz_op_add
entry point; they also check that, after the one set-up call, further calls
leave the device's free memory unchanged.  The arithmetic is integer, so the
tolerance is zero: the words must be identical.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import bitstreamzoo_b200 as bz  # noqa: E402
from bitstreamzoo_b200 import _lib  # noqa: E402
from oracle import cwords  # noqa: E402


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    # mostly-ones second operand: carries run across many tiles
    b = np.full(n, np.uint64(2**64 - 1), dtype=np.uint64)
    zeros = rng.integers(0, n, size=max(1, n // 5000))
    b[zeros] = rng.integers(0, 2**64, size=zeros.size, dtype=np.uint64)
    a[: min(n, 3000)] = np.uint64(2**64 - 1)   # one long propagate run from word 0
    b[0] = np.uint64(1)
    return a, b


def _dev(x):
    return torch.from_numpy(x.view(np.int64).copy()).cuda()


@pytest.mark.gpu
def test_noalloc_add_matches_oracle_and_op_add_on_two_calls():
    lib = _lib.load()
    ctx = bz.Context(0)
    for call, (n, nbits) in enumerate([((1 << 20) + 3, 64 * ((1 << 20) + 3) - 7),
                                       ((1 << 15) + 1, 64 * ((1 << 15) + 1))]):
        a, b = _inputs(n, seed=call)
        da, db = _dev(a), _dev(b)
        ref = torch.empty(n, dtype=torch.int64, device="cuda")
        out = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        ctx.op("add", ref.data_ptr(), da.data_ptr(), db.data_ptr(), n, nbits)
        ctx.sync()
        rc = lib.bsz_add_noalloc(out.data_ptr(), da.data_ptr(), db.data_ptr(), n, nbits, None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint64)
        want = cwords.add(a, b, nbits)
        assert np.array_equal(got, want), f"call {call}: first mismatch with the oracle at word " \
            f"{int(np.argmax(got != want))}"
        assert torch.equal(out, ref), f"call {call}: differs from bsz_op_add"
    ctx.close()


@pytest.mark.gpu
def test_noalloc_add_allocates_nothing_after_setup():
    lib = _lib.load()
    n = (1 << 18) + 9
    a, b = _inputs(n, seed=5)
    da, db = _dev(a), _dev(b)
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    assert lib.bsz_add_noalloc(None, None, None, 0, 0, None) == 0, _lib.last_error()   # set-up only
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert lib.bsz_add_noalloc(out.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n, None) == 0
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    # in place: dst = a
    assert lib.bsz_add_noalloc(da.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(da.cpu().numpy().view(np.uint64), cwords.add(a, b, 64 * n))


@pytest.mark.gpu
def test_noalloc_add_rejects_streams_beyond_its_scratch():
    lib = _lib.load()
    too_long = (1 << 26) + 1
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = lib.bsz_add_noalloc(dummy, dummy, dummy, too_long, 64 * too_long, None)
    assert rc != 0
    assert "exceeds the maximum" in _lib.last_error()


@pytest.mark.gpu
def test_noalloc_add_reports_a_lookback_timeout():
    """A look-back wait that runs out (a tile that never publishes its
    status, through the library's test hook; b = ~a so every tile must look
    back) makes the call return nonzero with the timeout message; the next
    call is exact."""
    lib = _lib.load()
    n = 4 * 4096
    rng = np.random.default_rng(41)
    a = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    b = ~a
    da, db = _dev(a), _dev(b)
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    lib.bsz_debug_add_lookback_hook(1, 1000)
    try:
        rc = lib.bsz_add_noalloc(out.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n, None)
        assert rc != 0
        assert "timed out" in _lib.last_error()
    finally:
        lib.bsz_debug_add_lookback_hook(-1, 0)
    assert lib.bsz_add_noalloc(out.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), cwords.add(a, b, 64 * n))
