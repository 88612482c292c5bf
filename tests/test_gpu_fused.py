"""Fused (generated persistent kernel) path at sizes where many warps share a
stream, so every warp's start state comes from speculative warm-up.

Each case runs through the C ABI in plain and fused form and is compared
word for word with the word-level C oracle: the long-stream primitives
(add with long carry runs, shifts by 1/63/64/1000), regex-shaped DAGs with
chained additions and shifted temporaries, right shifts (which cut the
segment), and an addition whose carry never resolves (x + ~x), where
speculation cannot be proven and the exact per-op re-run must take over.
"""

import random

import numpy as np
import pytest

import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import workloads as wl
from oracle import cwords, pyoracle
import progen


# fused forms: warp ranges with lane = word, thread-sequential ranges with
# register chunks (4 or 8 words), and thread-sequential ranges through TMA
# boxes (8- and 4-word rows; streams under 2^16 words take the register form
# instead); carry scheme 2 runs every addition with the plain carry-scan
# kernel between the generated parts
FORMS = [(bz.MODE_PLAIN, None), (bz.MODE_FUSED, {"layout": 0}), (bz.MODE_FUSED, {"layout": 1}),
         (bz.MODE_FUSED, {"layout": 2, "chunk_words": 8, "warps": 4, "min_blocks": 1}),
         (bz.MODE_FUSED, {"layout": 2, "chunk_words": 4, "warps": 8, "min_blocks": 1}),
         (bz.MODE_FUSED, {"layout": 2, "chunk_words": 4, "warps": 8, "min_blocks": 1, "shift_mul": 1}),
         (bz.MODE_FUSED, {"layout": 1, "warps": 4, "min_blocks": 1, "shift_mul": 1}),
         (bz.MODE_FUSED, {"layout": 1, "chunk_words": 8, "warps": 4, "min_blocks": 1}),
         (bz.MODE_FUSED, {"layout": 1, "warps": 4, "min_blocks": 1, "cut_adds": 2}),
         (bz.MODE_FUSED, {"layout": 0, "cut_adds": 2}),
         (bz.MODE_FUSED, {"layout": 2, "chunk_words": 4, "warps": 8, "min_blocks": 1, "cut_adds": 2})]


def run_both(ctx, src, nbits, inputs):
    prog = pyoracle.parse(src)
    ref_out, ref_pops = cwords.run_straight_line(prog, nbits, inputs)
    results = {}
    for mode, sched in FORMS:
        r = ctx.run(src, nbits, inputs, mode=mode, schedule=sched)
        for name, words in ref_out.items():
            got = r.stream(name)
            exp = words.copy()
            exp[-1] &= np.uint64(bz_mask(nbits))
            if not np.array_equal(got, exp):
                bad = int(np.argmax(got != exp))
                raise AssertionError(f"mode {mode} {sched} output {name}: first bad word {bad} of {got.size}")
        for name, v in ref_pops.items():
            assert r.int(name) == v, (mode, sched, name)
        results[(mode, tuple(sorted((sched or {}).items())))] = r.stats
    return results


def bz_mask(nbits):
    r = nbits % 64
    return ((1 << r) - 1) if r else (1 << 64) - 1


@pytest.mark.gpu
@pytest.mark.parametrize("nbits", [(1 << 22) + 37, 1 << 24])
def test_long_streams(ctx, nbits):
    inputs = wl.long_streams_inputs(nbits, seed=nbits)
    st = run_both(ctx, wl.long_streams_src(), nbits, inputs)
    for key, v in st.items():
        if key[0] == bz.MODE_FUSED:
            assert v["n_fused_launches"] >= 1, key


@pytest.mark.gpu
def test_matchstar(ctx):
    nbits = (1 << 22) + 5
    inputs = wl.matchstar_inputs(nbits, seed=3)
    run_both(ctx, wl.MATCHSTAR_SRC, nbits, inputs)


@pytest.mark.gpu
@pytest.mark.parametrize("n_ops,seed,nbits", [(300, 1, (1 << 20) + 64 * 3 + 11), (300, 2, (1 << 20) + 64 * 3 + 11),
                                              (2000, 3, (1 << 20) + 64 * 3 + 11), (2000, 4, (1 << 23) + 5),
                                              (2000, 5, 1 << 24)])
def test_regex_dag(ctx, n_ops, seed, nbits):
    src = wl.regex_dag_src(n_ops=n_ops, seed=seed)
    inputs = wl.regex_dag_inputs(nbits, seed=seed)
    run_both(ctx, src, nbits, inputs)


@pytest.mark.gpu
def test_chained_adds_and_shifted_temporaries(ctx):
    src = ("input stream a\ninput stream b\ninput stream c\noutput stream r\noutput stream q\n"
           "output int n\n"
           "stream s1 = a + b\nstream t1 = s1 << 1\nstream s2 = t1 + c\nstream t2 = s2 << 700\n"
           "stream m = t2 & a\nstream s3 = m + s2\nstream t3 = s3 << 64\nr = t3 ^ s1\n"
           "stream u = s3 >> 3\nstream v = u + a\nq = v << 5\nn = popcount(q)\n")
    nbits = (1 << 21) + 17
    rng = np.random.default_rng(9)
    inputs = {k: wl.random_words(rng, nbits) for k in "abc"}
    run_both(ctx, src, nbits, inputs)


@pytest.mark.gpu
def test_unresolvable_carry_falls_back_exactly(ctx):
    src = ("input stream x\ninput stream z\noutput stream r\noutput int n\n"
           "stream y = ~x\nstream s = x + y\nstream t = s << 1\nr = t + z\nn = popcount(r)\n")
    nbits = 1 << 22
    rng = np.random.default_rng(4)
    inputs = {"x": wl.random_words(rng, nbits), "z": wl.random_words(rng, nbits)}
    st = run_both(ctx, src, nbits, inputs)
    for key, v in st.items():
        if key[0] == bz.MODE_FUSED:
            if dict(key[1]).get("cut_adds") == 2:
                assert v["n_fused_fallbacks"] == 0, key   # the look-back scan needs no speculation
            else:
                assert v["n_fused_fallbacks"] >= 1, key


@pytest.mark.gpu
def test_random_straight_line_programs_fused_matches_plain_and_oracle(ctx):
    for seed in range(12):
        rng = random.Random(seed)
        nbits = rng.choice([64 * 2048 + 3, 64 * 4096, 100000])
        src, meta = progen.random_program(rng, n_stmts=40, allow_ctrl=False)
        inputs = {n: progen.rand_stream(rng, nbits) for n in meta["inputs"]}
        arrays = {"arr_in": {i: progen.rand_stream(rng, nbits) for i in range(4)}}
        try:
            want, ops, _ = pyoracle.run_source(src, nbits, inputs, meta["params"], arrays)
        except Exception:
            continue
        mask = (1 << nbits) - 1
        for mode, sched in FORMS:
            r = ctx.run(src, nbits, inputs, meta["params"], arrays, mode=mode, schedule=sched)
            assert r.stream_int("out0") & mask == want["out0"] & mask, (seed, mode)
            assert r.stream_int("out1") & mask == want["out1"] & mask, (seed, mode)
            for j in range(3):
                exp = want["outa"].get(j, 0) & mask
                assert r.stream_int("outa", j) & mask == exp, (seed, mode, j)
            assert r.int("cnt") == want["cnt"], (seed, mode)
            assert r.stats["op_count"] == ops


@pytest.mark.gpu
def test_outputs_folded_to_constants_or_inputs(ctx):
    """Folding can reduce an output to ZERO (a ^ a) or to an input; every form
    must still store it and count its popcount."""
    src = ("input stream a\ninput stream b\noutput stream z\noutput stream y\noutput stream w\n"
           "output int nz\noutput int ny\noutput int nw\n"
           "stream t = a ^ a\nz = t & b\ny = a\nstream s = a + b\nw = s << 1\n"
           "nz = popcount(z)\nny = popcount(y)\nnw = popcount(w)\n")
    nbits = (1 << 22) + 64 * 5
    rng = np.random.default_rng(12)
    inputs = {k: wl.random_words(rng, nbits) for k in "ab"}
    run_both(ctx, src, nbits, inputs)


@pytest.mark.gpu
def test_async_runs_overlap_and_stay_exact(ctx):
    """bsz_execute_async / bsz_run_wait: two runs enqueued back to back (the
    second launched before the first is waited on) give the same streams and
    popcounts as a synchronous run, and a run whose speculation cannot be
    proven (x + ~x) is re-run exactly when it is waited on, even with the
    next run already enqueued behind it."""
    nbits = (1 << 22) + 5
    rng = np.random.default_rng(8)
    src = ("input stream x\ninput stream z\noutput stream r\noutput int n\n"
           "stream y = ~x\nstream s = x + y\nstream t = s << 1\nr = t + z\nn = popcount(r)\n")
    inputs = {"x": wl.random_words(rng, nbits), "z": wl.random_words(rng, nbits)}
    prog = ctx.compile(src)
    for sched in ({"layout": 0}, {"layout": 1, "warps": 4, "min_blocks": 1}):
        want = ctx.run(prog, nbits, inputs, mode=bz.MODE_PLAIN)
        want_r, want_n = want.stream("r"), want.int("n")
        runs = []
        for _ in range(3):
            r = prog.run(nbits, bz.MODE_FUSED)
            r.set_schedule(sched)
            for k, v in inputs.items():
                r.bind(k, v)
            r.launch()
            runs.append(r)
        for r in runs:
            st = r.wait()
            assert st["n_fused_fallbacks"] >= 1, sched
            assert np.array_equal(r.stream("r"), want_r), sched
            assert r.int("n") == want_n, sched
    # a run that needs no re-run, read without an explicit wait
    src2 = ("input stream a\ninput stream b\noutput stream c\noutput int m\n"
            "stream s = a + b\nstream t = a << 3\nc = s ^ t\nm = popcount(c)\n")
    ins2 = {"a": wl.random_words(rng, nbits), "b": wl.random_words(rng, nbits)}
    p2 = ctx.compile(src2)
    want = ctx.run(p2, nbits, ins2, mode=bz.MODE_PLAIN)
    r1, r2 = p2.run(nbits, bz.MODE_FUSED), p2.run(nbits, bz.MODE_FUSED)
    for r in (r1, r2):
        for k, v in ins2.items():
            r.bind(k, v)
        r.launch()
    assert r2.int("m") == want.int("m")
    assert np.array_equal(r1.stream("c"), want.stream("c"))


@pytest.mark.gpu
def test_segment_whose_speculation_failed_switches_to_lookback_adds(ctx):
    """After a segment's speculative carry state could not be proven once,
    the next run of the same segment and schedule takes its additions through
    the look-back carry scan: no re-run, the same exact result."""
    nbits = (1 << 21) + 9
    rng = np.random.default_rng(12)
    src = ("input stream x\ninput stream z\noutput stream r\noutput int n\n"
           "stream y = ~x\nstream s = x + y\nstream t = s << 3\nr = t + z\nn = popcount(r)\n")
    inputs = {"x": wl.random_words(rng, nbits), "z": wl.random_words(rng, nbits)}
    want = ctx.run(src, nbits, inputs, mode=bz.MODE_PLAIN)
    sched = {"layout": 1, "warps": 8, "min_blocks": 1}
    first = ctx.run(src, nbits, inputs, mode=bz.MODE_FUSED, schedule=sched)
    second = ctx.run(src, nbits, inputs, mode=bz.MODE_FUSED, schedule=sched)
    assert first.stats["n_fused_fallbacks"] >= 1
    assert second.stats["n_fused_fallbacks"] == 0
    for r in (first, second):
        assert np.array_equal(r.stream("r"), want.stream("r"))
        assert r.int("n") == want.int("n")
