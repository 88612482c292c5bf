"""Device byte -> basis-bit transposition (bsz_s2p) against the oracle's
restatement of payload_to_basis_bits (bit-exact)."""

import numpy as np
import pytest

from oracle import basis

pytestmark = pytest.mark.gpu


def _run_s2p(ctx, payload: np.ndarray, offset: int = 0):
    import torch

    n = payload.size
    nw = (n + 63) // 64
    src = torch.zeros(n + offset + 16, dtype=torch.uint8, device="cuda")
    if n:
        src[offset:offset + n] = torch.from_numpy(payload).cuda()
    # poison the outputs so words the kernel fails to write show up
    outs = [torch.full((max(1, nw),), -1, dtype=torch.int64, device="cuda") for _ in range(8)]
    torch.cuda.synchronize()
    ctx.s2p(src.data_ptr() + offset, n, [o.data_ptr() for o in outs])
    ctx.sync()
    return [o.cpu().numpy().view(np.uint64)[:nw] for o in outs]


@pytest.mark.parametrize("n", [1, 7, 63, 64, 65, 1000, 4096, (1 << 20) + 13])
def test_s2p_matches_oracle(ctx, n):
    rng = np.random.default_rng(n)
    payload = rng.integers(0, 256, n, dtype=np.uint8)
    got = _run_s2p(ctx, payload)
    want = basis.basis_words(payload)
    for i in range(8):
        assert np.array_equal(got[i], want[i]), i


@pytest.mark.parametrize("offset", [1, 3, 8])
def test_s2p_unaligned_source(ctx, offset):
    rng = np.random.default_rng(100 + offset)
    payload = rng.integers(0, 256, 5000, dtype=np.uint8)
    got = _run_s2p(ctx, payload, offset)
    want = basis.basis_words(payload)
    for i in range(8):
        assert np.array_equal(got[i], want[i]), i


def test_s2p_small_against_reference_loop(ctx):
    payload = np.frombuffer(b"The quick brown fox \xff\x00\x80 jumps", dtype=np.uint8)
    got = _run_s2p(ctx, payload)
    want = basis.basis_ints(payload.tobytes())
    for i in range(8):
        assert int.from_bytes(got[i].tobytes(), "little") == want[i]


def test_s2p_zero_bytes_is_a_no_op(ctx):
    ctx.s2p(0, 0, [0] * 8)
    ctx.sync()


def test_s2p_matches_reference_goldens(ctx):
    """bsz_s2p against the reference's own payload_to_basis_bits outputs."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "s2p_golden.json")) as f:
        cases = json.load(f)["cases"]
    for c in cases:
        payload = np.frombuffer(bytes.fromhex(c["payload"]), dtype=np.uint8)
        got = _run_s2p(ctx, payload)
        want = [int(h, 16) for h in c["basis"]]
        assert [int.from_bytes(w.astype("<u8").tobytes(), "little") for w in got] == want, c["name"]
