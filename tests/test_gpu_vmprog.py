"""Whole programs with control flow on the device interpreter (program mode).

Each program runs in VM and auto mode and is compared with the Python oracle
(outputs and op count); the statistics show whether it ran as one device
launch with a single read-back or fell back to the host-driven walk.
"""

import random

import pytest

import bitstreamzoo_b200 as bz
from oracle import pyoracle
import progen

pytestmark = pytest.mark.gpu


def _int_outputs(src):
    return {ln.split()[2] for ln in src.splitlines() if ln.startswith("output int ")}


def run_and_check(ctx, src, nbits, inputs, params=None, arrays=None, modes=(bz.MODE_VM, bz.MODE_AUTO)):
    want, ops, mix = pyoracle.run_source(src, nbits, inputs, params, arrays)
    mask = (1 << nbits) - 1
    ints = _int_outputs(src)
    stats = {}
    for mode in modes:
        r = ctx.run(src, nbits, inputs, params, arrays, mode=mode)
        for name, v in want.items():
            if name in ints:
                assert r.int(name) == v, (mode, name)
            elif isinstance(v, dict):
                for i, x in v.items():
                    assert r.stream_int(name, i) & mask == x & mask, (mode, name, i)
            else:
                assert r.stream_int(name) & mask == v & mask, (mode, name)
        assert r.stats["op_count"] == ops, (mode, r.stats["op_count"], ops)
        stats[mode] = r.stats
    return stats, mix


REGEX_LIKE = """input stream b[8]
output stream m0
output stream m1
output int n0
stream nb0 = ~b[0]
stream t1 = b[1] & nb0
stream a1 = t1 << 1
stream t2 = a1 & b[2]
stream z = ZERO
m0 = z
if (t2) {
  stream a2 = t2 << 1
  stream t3 = a2 & b[3]
  m0 = t3
}
stream cc = b[4] | b[5]
stream mm = b[6] & cc
stream v_test = mm
stream v_acc = mm
stream v_pend = mm
while (v_test) {
  stream q = cc & v_pend
  stream adv = q << 1
  stream x1 = adv & cc
  stream x2 = x1 + cc
  stream x3 = x2 ^ cc
  stream x4 = x3 | adv
  stream nacc = ~v_acc
  stream np = x4 & nacc
  v_pend = np
  stream acc2 = v_acc | x4
  v_acc = acc2
  v_test = v_pend
}
m1 = v_acc
n0 = popcount(m1)
"""


@pytest.mark.parametrize("nbits", [1, 50, 64, 777, 4096 + 3, 64 * 1500])
def test_regex_like_program_one_launch(ctx, nbits):
    rnd = random.Random(nbits)
    arrays = {"b": {i: progen.rand_stream(rnd, nbits) for i in range(8)}}
    stats, _ = run_and_check(ctx, REGEX_LIKE, nbits, {}, None, arrays)
    st = stats[bz.MODE_VM]
    assert st["n_vm_launches"] == 1
    assert st["n_syncs"] <= 2


def test_branch_not_taken_hides_errors(ctx):
    # popcount of a negative value inside a branch that is not taken: no error
    src = """input stream a
output int c
output stream r
stream z = ZERO
stream neg = ONES
r = a
if (z) {
  c = popcount(neg)
}
c = popcount(r)
"""
    stats, _ = run_and_check(ctx, src, 100, {"a": 12345})
    assert stats[bz.MODE_VM]["n_vm_launches"] == 1


def test_taken_branch_raises_reference_errors(ctx):
    src = """input stream a
output int c
stream neg = ONES
if (a) {
  c = popcount(neg)
}
"""
    for mode in (bz.MODE_VM, bz.MODE_AUTO, bz.MODE_PLAIN):
        with pytest.raises(bz.BszError, match="popcount on negative value"):
            ctx.run(src, 64, {"a": 1}, mode=mode)
    loop = """input stream a
output stream r
stream t = a
while (t) {
  r = t
}
"""
    for mode in (bz.MODE_VM, bz.MODE_PLAIN):
        with pytest.raises(bz.BszError, match="while loop exceeded 10000 iterations"):
            ctx.run(loop, 64, {"a": 1}, mode=mode)


def test_device_ints_loops_and_arrays(ctx):
    src = """input stream a
input stream b
output stream o[3]
output int k
output int s
k = 0
o[0] = a
o[1] = b
o[2] = ZERO
stream t = a & b
if (t) {
  k = popcount(t)
  for i in 0..3 {
    stream u = o[i] << 1
    o[i] = u ^ b
  }
  k = k * 2 + i
}
s = popcount(a) + k
"""
    for seed in range(4):
        rnd = random.Random(seed)
        nbits = rnd.choice([70, 300, 2000])
        a = rnd.getrandbits(nbits)
        b = rnd.getrandbits(nbits) if seed % 2 else (~a) & ((1 << nbits) - 1)
        stats, _ = run_and_check(ctx, src, nbits, {"a": a, "b": b})
        assert stats[bz.MODE_VM]["n_vm_launches"] == 1


def test_conditionally_defined_read_falls_back(ctx):
    # `x` exists only if the branch ran: the program needs the host walk
    src = """input stream a
output stream r
if (a) {
  stream x = a << 2
}
r = x
"""
    for mode in (bz.MODE_VM, bz.MODE_AUTO):
        r = ctx.run(src, 64, {"a": 3}, mode=mode)
        assert r.stream_int("r") == 12
    with pytest.raises(bz.BszError):
        ctx.run(src, 64, {"a": 0}, mode=bz.MODE_VM)


@pytest.mark.parametrize("nbits", [1, 65, 700])
def test_random_programs_with_control_flow(ctx, nbits):
    mask = (1 << nbits) - 1
    n_checked = n_device = 0
    for seed in range(25):
        rng = random.Random(7000 + nbits * 31 + seed)
        src, meta = progen.random_program(rng, n_stmts=45)
        inputs = {n: progen.rand_stream(rng, nbits) for n in meta["inputs"]}
        arrays = {"arr_in": {i: progen.rand_stream(rng, nbits) for i in range(4)}}
        try:
            want, ops, _ = pyoracle.run_source(src, nbits, inputs, meta["params"], arrays)
        except Exception:  # the reference raises: so must we
            for mode in (bz.MODE_VM, bz.MODE_AUTO):
                with pytest.raises(bz.BszError):
                    ctx.run(src, nbits, inputs, meta["params"], arrays, mode=mode)
            continue
        n_checked += 1
        for mode in (bz.MODE_VM, bz.MODE_AUTO):
            r = ctx.run(src, nbits, inputs, meta["params"], arrays, mode=mode)
            assert r.stream_int("out0") & mask == want["out0"] & mask, (seed, mode)
            assert r.stream_int("out1") & mask == want["out1"] & mask, (seed, mode)
            for j in range(3):
                assert r.stream_int("outa", j) & mask == want["outa"].get(j, 0) & mask, (seed, mode, j)
            assert r.int("cnt") == want["cnt"], (seed, mode)
            assert r.stats["op_count"] == ops, (seed, mode)
            if mode == bz.MODE_VM and r.stats["n_vm_launches"] == 1 and r.stats["n_segments"] == 1:
                n_device += 1
    assert n_checked >= 10
    assert n_device >= 1
