"""Walk cache: a straight-line program run again with the same bit length,
mode and bindings restores its statement walk (the DAG and the variable
state) from the program instead of walking the statements again; the device
work runs in full on every run.

Every run here is checked against the oracle: repeated runs of one compiled
program with new data (replayed), runs whose bindings differ (another
parameter value, an unbound input, another bit length: walked again, then
replayed in turn), and programs whose walk cannot be cached (a popcount used
as a shift amount needs the device during the walk).
"""

import random

import numpy as np
import pytest

import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import workloads as wl
from oracle import cwords, pyoracle
import progen


def _mask(nbits):
    r = nbits % 64
    return ((1 << r) - 1) if r else (1 << 64) - 1


def _check_words(r, src, nbits, inputs, tag):
    ref_out, ref_pops = cwords.run_straight_line(pyoracle.parse(src), nbits, inputs)
    for name, words in ref_out.items():
        exp = words.copy()
        exp[-1] &= np.uint64(_mask(nbits))
        got = r.stream(name)
        if not np.array_equal(got, exp):
            bad = int(np.argmax(got != exp))
            raise AssertionError(f"{tag} output {name}: first bad word {bad} of {got.size}")
    for name, v in ref_pops.items():
        assert r.int(name) == v, (tag, name)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,nbits", [(bz.MODE_PLAIN, (1 << 20) + 11), (bz.MODE_FUSED, (1 << 20) + 11),
                                        (bz.MODE_AUTO, (1 << 20) + 11), (bz.MODE_VM, 64 * 4096 + 5),
                                        (bz.MODE_AUTO, 64 * 4096 + 5)])
def test_repeated_runs_replay_the_walk(ctx, mode, nbits):
    src = wl.regex_dag_src(n_ops=300, seed=7)
    prog = ctx.compile(src)
    for i, seed in enumerate((11, 12, 13)):
        inputs = wl.regex_dag_inputs(nbits, seed=seed)
        r = ctx.run(prog, nbits, inputs, mode=mode)
        assert r.stats["walk_replayed"] == (1 if i > 0 else 0), (mode, i)
        _check_words(r, src, nbits, inputs, f"mode {mode} run {i}")
        first_ops = r.stats["op_count"] if i == 0 else first_ops
        assert r.stats["op_count"] == first_ops


@pytest.mark.gpu
def test_bindings_and_length_change_the_key(ctx):
    checked = 0
    for seed in range(10):
        rng = random.Random(100 + seed)
        src, meta = progen.random_program(rng, n_stmts=40, allow_ctrl=False)
        prog = ctx.compile(src)
        nb1 = rng.choice([64 * 2048 + 3, 100000])
        nb2 = nb1 + 64 * 7 + 1
        k0 = meta["params"]["K"]
        # (bit length, params, inputs left unbound, expect replay)
        plan = [(nb1, {"K": k0}, (), False), (nb1, {"K": k0}, (), True),
                (nb1, {"K": k0 + 1}, (), False), (nb1, {"K": k0 + 1}, (), True),
                (nb1, {"K": k0}, ("in1",), False), (nb2, {"K": k0}, (), False),
                (nb1, {"K": k0}, (), True)]
        for mode in (bz.MODE_PLAIN, bz.MODE_FUSED):
            for j, (nbits, params, unbound, replay) in enumerate(plan):
                inputs = {n: progen.rand_stream(rng, nbits) for n in meta["inputs"]}
                arrays = {"arr_in": {i: progen.rand_stream(rng, nbits) for i in range(4)}}
                oracle_in = {n: (0 if n in unbound else v) for n, v in inputs.items()}
                try:
                    want, ops, _ = pyoracle.run_source(src, nbits, oracle_in, params, arrays)
                except Exception:
                    break
                r = prog.run(nbits, mode)
                for k, v in params.items():
                    r.set_param(k, v)
                for k, v in inputs.items():
                    if k not in unbound:
                        r.bind(k, v)
                for k, arr in arrays.items():
                    for i, v in arr.items():
                        r.bind(k, v, index=i)
                r.execute()
                tag = (seed, mode, j)
                assert r.stats["walk_replayed"] == (1 if replay else 0), tag
                mask = (1 << nbits) - 1
                assert r.stream_int("out0") & mask == want["out0"] & mask, tag
                assert r.stream_int("out1") & mask == want["out1"] & mask, tag
                for a in range(3):
                    assert r.stream_int("outa", a) & mask == want["outa"].get(a, 0) & mask, (tag, a)
                assert r.int("cnt") == want["cnt"], tag
                assert r.stats["op_count"] == ops, tag
                checked += 1
    assert checked >= 40


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [bz.MODE_PLAIN, bz.MODE_FUSED, bz.MODE_AUTO])
def test_walk_that_needs_the_device_is_not_cached(ctx, mode):
    # the shift amount is a popcount: the walk flushes to read it
    src = ("input stream a\ninput stream b\noutput stream r\noutput int n\n"
           "int k = popcount(b)\nstream s = a + b\nstream t = s << k\nr = t ^ a\nn = popcount(r)\n")
    nbits = 64 * 3000 + 9
    prog = ctx.compile(src)
    rng = random.Random(5)
    for i in range(3):
        a = progen.rand_stream(rng, nbits)
        b = progen.rand_stream(rng, 40 + 13 * i)    # popcount(b) differs per run
        want, _, _ = pyoracle.run_source(src, nbits, {"a": a, "b": b}, {}, {})
        r = ctx.run(prog, nbits, {"a": a, "b": b}, mode=mode)
        assert r.stats["walk_replayed"] == 0
        mask = (1 << nbits) - 1
        assert r.stream_int("r") & mask == want["r"] & mask, (mode, i)
        assert r.int("n") == want["n"], (mode, i)
