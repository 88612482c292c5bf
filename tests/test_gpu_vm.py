"""Device interpreter (VM) and automatic mode against the word-level oracle.

Covers one-warp streams (up to 32 words), multi-warp streams whose carries
cross warps and steps of the CTA (B nearly all ones, so carry runs span the
whole stream), a slot file too large for shared memory (global slot file),
and a loop nest unrolled to hundreds of thousands of operations, which the
automatic flush cuts into several segments."""

import random

import numpy as np
import pytest

import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import workloads as wl
from oracle import cwords, pyoracle
import progen

pytestmark = pytest.mark.gpu


def _mask(nbits):
    r = nbits % 64
    return ((1 << r) - 1) if r else (1 << 64) - 1


def check(ctx, src, nbits, inputs, modes=(bz.MODE_VM, bz.MODE_AUTO)):
    prog = pyoracle.parse(src)
    ref_out, ref_pops = cwords.run_straight_line(prog, nbits, inputs)
    stats = {}
    for mode in modes:
        r = ctx.run(src, nbits, inputs, mode=mode)
        for name, words in ref_out.items():
            got = r.stream(name)
            exp = words.copy()
            exp[-1] &= np.uint64(_mask(nbits))
            if not np.array_equal(got, exp):
                bad = int(np.argmax(got != exp))
                raise AssertionError(f"mode {mode} output {name}: first bad word {bad} of {got.size}")
        for name, v in ref_pops.items():
            assert r.int(name) == v, (mode, name)
        stats[mode] = r.stats
    return stats


@pytest.mark.parametrize("nbits", [1, 63, 64, 65, 1000, 2047, 2048 + 7, 64 * 700 + 9])
def test_random_programs(ctx, nbits):
    """Random programs with control flow and arrays: VM and auto vs the
    Python oracle (unmasked words compared under the stream mask)."""
    mask = (1 << nbits) - 1
    n_checked = 0
    for seed in range(10):
        rng = random.Random(nbits * 100 + seed)
        src, meta = progen.random_program(rng, n_stmts=40)
        inputs = {n: progen.rand_stream(rng, nbits) for n in meta["inputs"]}
        arrays = {"arr_in": {i: progen.rand_stream(rng, nbits) for i in range(4)}}
        try:
            want, ops, _ = pyoracle.run_source(src, nbits, inputs, meta["params"], arrays)
        except Exception:
            continue
        n_checked += 1
        for mode in (bz.MODE_VM, bz.MODE_AUTO):
            r = ctx.run(src, nbits, inputs, meta["params"], arrays, mode=mode)
            assert r.stream_int("out0") & mask == want["out0"] & mask, (seed, mode)
            assert r.stream_int("out1") & mask == want["out1"] & mask, (seed, mode)
            for j in range(3):
                assert r.stream_int("outa", j) & mask == want["outa"].get(j, 0) & mask, (seed, mode, j)
            assert r.int("cnt") == want["cnt"], (seed, mode)
            assert r.stats["op_count"] == ops
    assert n_checked >= 5


@pytest.mark.parametrize("nbits", [(1 << 17) + 13, 32 * 64 * 5 + 1, 1 << 19])
def test_long_carries_across_warps(ctx, nbits):
    inputs = wl.long_streams_inputs(nbits, seed=nbits)
    check(ctx, wl.long_streams_src(), nbits, inputs)


def test_matchstar_multi_warp(ctx):
    nbits = 300_001
    check(ctx, wl.MATCHSTAR_SRC, nbits, wl.matchstar_inputs(nbits, seed=5))


def test_global_slot_file(ctx):
    # 8192 words per value: more than a handful of live temporaries exceed
    # the shared-memory slot file, so the VM keeps them in global memory.
    nbits = 8192 * 64
    src = wl.regex_dag_src(n_ops=300, seed=12)
    rng = np.random.default_rng(12)
    inputs = {f"b{i}": rng.integers(0, 2**63, 8192, dtype=np.uint64) * 2 + rng.integers(0, 2, 8192, dtype=np.uint64)
              for i in range(8)}
    check(ctx, src, nbits, inputs, modes=(bz.MODE_VM,))


def test_unrolled_loop_nest(ctx):
    # ~2.4 million DSL operations at 100 bits: several automatic flushes,
    # each one VM launch; compared with the plain per-op form on the GPU.
    src = """input stream a
input stream b
output stream x
output int c
stream x = a
stream t = a
for i in 0..400 {
  for j in 0..1000 {
    t = x + b
    x = t ^ a
    t = x << 1
    x = t | b
    t = ~x
    x = t & a
  }
}
c = popcount(x)
"""
    nbits = 100
    rnd = random.Random(9)
    inputs = {"a": rnd.getrandbits(nbits), "b": rnd.getrandbits(nbits)}
    rv = ctx.run(src, nbits, inputs, mode=bz.MODE_VM)
    assert rv.stats["op_count"] == 400 * 1000 * 6 + 1
    assert rv.stats["n_vm_launches"] >= 2
    assert rv.stats["n_kernel_launches"] < 100
    m = (1 << nbits) - 1
    a, b = inputs["a"], inputs["b"]
    x = a
    for _ in range(400 * 1000):
        x = (((((x + b) & m) ^ a) << 1) & m) | b
        x = ~x & m & a
    assert rv.stream_int("x") == x
    assert rv.int("c") == bin(x).count("1")


def test_auto_mode_case_json_matches_plain(ctx):
    src = wl.regex_dag_src(n_ops=120, seed=4)
    rnd = random.Random(4)
    nbits = 777
    payload = {"inputs": {f"b{i}": hex(rnd.getrandbits(nbits)) for i in range(8)}, "n_vectors": nbits}
    a = ctx.run_case_json(src, json_input=payload, mode="auto")
    p = ctx.run_case_json(src, json_input=payload, mode="plain")
    assert a["outputs"] == p["outputs"]
    assert a["op_count"] == p["op_count"]
    assert a["executor"] == "b200-auto"
