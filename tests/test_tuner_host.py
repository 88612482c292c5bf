"""Host-side checks of the autotuner and the cost model's reference math (no GPU)."""

import math
import random

import numpy as np
import pytest

from bitstreamzoo_b200 import DEFAULT_SCHEDULE, tuner
from bitstreamzoo_b200.workloads import shaped_dag_src

import mlp_ref
from oracle import pyoracle


def test_candidate_space_is_the_product():
    c = tuner.candidate_space()
    n = 1
    for ax in (tuner.CODEGEN_AXES, tuner.LAUNCH_AXES):
        for v in ax.values():
            n *= len(v)
    m = 1
    for v in tuner.SEQ_AXES.values():
        m *= len(v)
    n += m + len(tuner.TMA_CANDIDATES) + len(tuner.CARRY_CANDIDATES)
    assert len(c) == n == len(tuner.CANDIDATES) == 32
    assert sum(1 for s in c if s["layout"] == 1 and s["cut_adds"] == 0) == m
    assert sum(1 for s in c if s["cut_adds"] == 2) == len(tuner.CARRY_CANDIDATES)
    assert len({tuner.schedule_key(s) for s in c}) == n
    for s in c:
        assert set(s) == set(DEFAULT_SCHEDULE)


def test_schedule_encoding():
    e = tuner.encode_schedule(DEFAULT_SCHEDULE)
    assert len(e) == tuner.N_SCHEDULE_FEATURES
    assert e[0] == 2.0 and e[4] == 1.0 and e[5] == 0.0
    assert e[6] == math.log2(32 * 4 * 4)
    # warp form: no thread-form knobs, speculative carries
    assert e[7:] == [0.0, 0.0, 0.0, 0.0, 0.0, 0.0]
    # register form with 8-word chunks and look-back additions
    r = tuner.encode_schedule(dict(DEFAULT_SCHEDULE, layout=1, chunk_words=8, cut_adds=2, min_blocks=1))
    assert r[5] == 0.0 and r[7] == 1.0 and r[8] == 0.0 and r[9] == 3.0 and r[12] == 1.0
    # TMA form, 3 stages, materialized additions
    t = tuner.encode_schedule(dict(DEFAULT_SCHEDULE, layout=2, stages=3, cut_adds=1))
    assert t[5] == 1.0 and t[7] == 1.0 and t[8] == 1.0 and t[9] == 2.0 and t[10] == 3.0 and t[12] == 0.0


def test_every_candidate_has_a_distinct_encoding():
    rows = {tuple(tuner.encode_schedule(s)) for s in tuner.CANDIDATES}
    assert len(rows) == len(tuner.CANDIDATES)


def test_regret():
    times = {(1,): 2.0, (2,): 1.0, (3,): 1.5}
    assert tuner.regret(times, (2,)) == 0.0
    assert tuner.regret(times, (1,)) == 1.0


def test_tuning_suite_is_seeded_and_valid():
    a = tuner.tuning_suite(6, 4)
    b = tuner.tuning_suite(6, 4)
    assert a == b
    rnd = random.Random(3)
    for src in a[0] + a[1][:2]:
        ins = {f"b{i}": rnd.getrandbits(200) for i in range(8)}
        out, _, _ = pyoracle.run_source(src, 200, ins)
        assert {"o0", "p0"} <= set(out)


def test_shaped_dag_window_limits_operands():
    src = shaped_dag_src(200, seed=5, window=4, p_shr=0.1, max_shift=9)
    defined = []
    for line in src.splitlines():
        if line.startswith("stream v"):
            lhs, rhs = line[len("stream "):].split(" = ")
            operands = [t for t in rhs.replace("~", " ").split() if t[0] in "vb"]
            for o in operands:
                if o.startswith("v"):
                    assert o in defined[-4:]
            defined.append(lhs)
    assert len(defined) == 200


def test_reference_mlp_gradients_match_finite_differences():
    """Pins the float64 reference that the GPU gradient test compares against."""
    rng = np.random.default_rng(0)
    dims = mlp_ref.dims_of(5, 7, 2)
    npar = sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    p = rng.normal(0, 0.5, npar)
    x = rng.normal(0, 1, (11, 5))
    y = rng.normal(0, 1, 11)
    loss, g = mlp_ref.loss_and_grad(p, dims, x, y)
    h = 1e-6
    for i in rng.choice(npar, 25, replace=False):
        e = np.zeros(npar)
        e[i] = h
        fd = (mlp_ref.loss_and_grad(p + e, dims, x, y)[0] - mlp_ref.loss_and_grad(p - e, dims, x, y)[0]) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-5, abs=1e-8)
