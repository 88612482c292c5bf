"""Per-operator CUDA kernels (the bsz_op_* C ABI, the reference CudaBackend
op_* data plane) against the word-level C oracle, on device buffers, at the
sizes, shift amounts and carry patterns of the reference's native tests
(test_ops.cpp:114-421, test_kernels.cu:82-557) plus multi-tile sizes."""

import numpy as np
import pytest

from oracle import cwords

torch = pytest.importorskip("torch")

SIZES = [1, 2, 3, 7, 8, 15, 16, 100, 1000, 2047, 2048, 2049, 4097, 65536 + 5, 1 << 20]
SHIFTS = [0, 1, 31, 63, 64, 65, 127, 128, 200, 1000, 4095, 70000]


def dev(a: np.ndarray):
    return torch.from_numpy(a.view(np.int64).copy()).cuda()


def host(t) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint64)


def rand_words(rng, n):
    return rng.integers(0, 2**64, size=n, dtype=np.uint64)


@pytest.mark.gpu
@pytest.mark.parametrize("n", SIZES)
def test_bitwise_not(ctx, n):
    rng = np.random.default_rng(n)
    a, b = rand_words(rng, n), rand_words(rng, n)
    da, db, dd = dev(a), dev(b), torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    for name, ref in [("and", a & b), ("or", a | b), ("xor", a ^ b), ("andnot", a & ~b)]:
        ctx.op(name, dd.data_ptr(), da.data_ptr(), db.data_ptr(), n)
        ctx.sync()
        assert np.array_equal(host(dd), ref), name
    nbits = 64 * n - 13
    ctx.op("not", dd.data_ptr(), da.data_ptr(), n, nbits)
    ctx.sync()
    ref = ~a
    ref[-1] &= np.uint64((1 << (nbits % 64)) - 1)
    assert np.array_equal(host(dd), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 7, 100, 2049, 65541])
@pytest.mark.parametrize("k", SHIFTS)
def test_shifts(ctx, n, k):
    rng = np.random.default_rng(1000 + n + k)
    a = rand_words(rng, n)
    nbits = 64 * n - 3
    a[-1] &= np.uint64((1 << 61) - 1)
    da, dd = dev(a), torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.op("shl", dd.data_ptr(), da.data_ptr(), k, n, nbits)
    ctx.sync()
    assert np.array_equal(host(dd), cwords.shl(a, k, nbits)), "shl"
    for tail in (0, 1):
        ctx.op("shr", dd.data_ptr(), da.data_ptr(), k, n, tail)
        ctx.sync()
        ref = np.empty_like(a)
        cwords.lib().o_shr(cwords._p(ref), cwords._p(a), k, n, tail)
        assert np.array_equal(host(dd), ref), ("shr", tail)


def _check_add(ctx, a, b, nbits):
    n = a.size
    da, db, dd = dev(a), dev(b), torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.op("add", dd.data_ptr(), da.data_ptr(), db.data_ptr(), n, nbits)
    ctx.sync()
    got = host(dd)
    ref = cwords.add(a, b, nbits)
    assert np.array_equal(got, ref), int(np.argmax(got != ref))
    assert ctx.popcount(dd.data_ptr(), n) == cwords.popcount(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("n", SIZES)
def test_add_random(ctx, n):
    rng = np.random.default_rng(7 * n)
    _check_add(ctx, rand_words(rng, n), rand_words(rng, n), 64 * n)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [8, 512, 2048, 2049, 4096 + 3, 1 << 16, (1 << 20) + 17])
def test_add_carry_chains(ctx, n):
    """All-ones + 1 propagates a carry through every word and every tile."""
    ones = np.full(n, np.uint64(2**64 - 1), dtype=np.uint64)
    one = np.zeros(n, dtype=np.uint64)
    one[0] = 1
    _check_add(ctx, ones, one, 64 * n)
    # propagate runs that start mid-tile and cross many tile boundaries
    rng = np.random.default_rng(n)
    a = rand_words(rng, n)
    b = np.zeros(n, dtype=np.uint64)
    for start in range(3, n, max(1, n // 7)):
        run = min(n - start, 3000)
        a[start:start + run] = np.uint64(2**64 - 1)
        b[start - 1] = np.uint64(2**64 - 1)
        a[start - 1] = np.uint64(1)
    _check_add(ctx, a, b, 64 * n - 1)


@pytest.mark.gpu
def test_add_bernoulli_long_carries(ctx):
    """B all ones except rare zeros (the long-carry stream shape)."""
    n = 1 << 22
    rng = np.random.default_rng(5)
    a = rand_words(rng, n)
    z = np.full(n, np.uint64(2**64 - 1), dtype=np.uint64)
    for _ in range(20):
        z &= rand_words(rng, n)
    b = ~z
    _check_add(ctx, a, b, 64 * n)


@pytest.mark.gpu
@pytest.mark.parametrize("n", SIZES)
def test_popcount_nonzero(ctx, n):
    rng = np.random.default_rng(3 * n)
    a = rand_words(rng, n)
    da = dev(a)
    torch.cuda.synchronize()
    assert ctx.popcount(da.data_ptr(), n) == cwords.popcount(a)
    assert ctx.is_nonzero(da.data_ptr(), n)
    z = dev(np.zeros(n, dtype=np.uint64))
    torch.cuda.synchronize()
    assert not ctx.is_nonzero(z.data_ptr(), n)
    assert ctx.popcount(z.data_ptr(), n) == 0


@pytest.mark.gpu
def test_unaligned_pointers_take_scalar_path(ctx):
    n = 1001
    rng = np.random.default_rng(11)
    a, b = rand_words(rng, n + 1), rand_words(rng, n + 1)
    da, db = dev(a), dev(b)
    dd = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    off = 8  # one word: 8-byte aligned, not 16-byte aligned
    ctx.op("xor", dd.data_ptr() + off, da.data_ptr() + off, db.data_ptr() + off, n)
    ctx.sync()
    assert np.array_equal(host(dd)[1:], (a ^ b)[1:])
    assert ctx.popcount(da.data_ptr() + off, n) == cwords.popcount(a[1:])


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["a", "b"])
def test_add_in_place(ctx, which):
    """dst may be one of the operands: every word is read before it is written."""
    n = 3 * 4096 + 5
    rng = np.random.default_rng(17)
    a, b = rand_words(rng, n), rand_words(rng, n)
    a[100:2000] = np.uint64(2**64 - 1)   # a propagate run across a block boundary
    b[99] = np.uint64(2**64 - 1)
    da, db = dev(a), dev(b)
    torch.cuda.synchronize()
    dst = da if which == "a" else db
    ctx.op("add", dst.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n - 3)
    ctx.sync()
    assert np.array_equal(host(dst), cwords.add(a, b, 64 * n - 3))


@pytest.mark.gpu
def test_add_unaligned_multi_tile(ctx):
    """8-byte-aligned (not 32-byte-aligned) operands take the word-by-word path."""
    n = 2 * 4096 + 77
    rng = np.random.default_rng(23)
    a, b = rand_words(rng, n + 1), rand_words(rng, n + 1)
    a[1:3000] = np.uint64(2**64 - 1)
    b[1] = np.uint64(1)
    da, db = dev(a), dev(b)
    dd = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    off = 8
    ctx.op("add", dd.data_ptr() + off, da.data_ptr() + off, db.data_ptr() + off, n, 64 * n)
    ctx.sync()
    assert np.array_equal(host(dd)[1:], cwords.add(a[1:], b[1:], 64 * n))


@pytest.mark.gpu
def test_add_rejects_bitlength_outside_the_words(ctx):
    from bitstreamzoo_b200 import _lib
    n = 64
    d = torch.zeros(n, dtype=torch.int64, device="cuda")
    for bad in (-1, 64 * n + 1):
        with pytest.raises(_lib.BszError, match="bitlength"):
            ctx.op("add", d.data_ptr(), d.data_ptr(), d.data_ptr(), n, bad)


@pytest.mark.gpu
@pytest.mark.parametrize("in_place", [False, True])
def test_add_carry_ripples_across_many_tiles(ctx, in_place):
    """A carry generated once and propagated over ~30 tiles (a = 0, b = all
    ones), between random words: tiles inside the run cannot resolve their
    carry in locally and take it by look-back."""
    n = 50 * 4096 + 13
    rng = np.random.default_rng(31)
    a, b = rand_words(rng, n), rand_words(rng, n)
    a[1000], b[1000] = np.uint64(2**64 - 1), np.uint64(1)
    a[1001:120001] = np.uint64(0)
    b[1001:120001] = np.uint64(2**64 - 1)
    a[150000:150100] = ~b[150000:150100]   # a short propagate run with whatever comes in
    da, db = dev(a), dev(b)
    dd = da if in_place else torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.op("add", dd.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n - 5)
    ctx.sync()
    assert np.array_equal(host(dd), cwords.add(a, b, 64 * n - 5))


@pytest.mark.gpu
def test_add_lookback_timeout_is_reported(ctx):
    """A look-back wait that runs out (its predecessor tile never publishes,
    through the test hook) ends with an error the host reads; the context
    stays usable and the next add is exact."""
    from bitstreamzoo_b200 import _lib
    lib = _lib.load()
    n = 4 * 4096
    rng = np.random.default_rng(29)
    # b = ~a: every word propagates, so no tile can take its carry in from
    # the words before it and every tile past the first must look back
    a = rand_words(rng, n)
    b = ~a
    da, db, dd = dev(a), dev(b), torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    lib.bsz_debug_add_lookback_hook(1, 1000)
    try:
        ctx.op("add", dd.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n)
        with pytest.raises(_lib.BszError, match="look-back timed out"):
            ctx.sync()
    finally:
        lib.bsz_debug_add_lookback_hook(-1, 0)
    ctx.op("add", dd.data_ptr(), da.data_ptr(), db.data_ptr(), n, 64 * n)
    ctx.sync()
    assert np.array_equal(host(dd), cwords.add(a, b, 64 * n))
