"""GPU tests of the cost model's CUDA kernels, the DAG features, schedule
parity and the autotuner.

MLP kernels (tiled FP32 GEMM, bias/ReLU epilogue, MSE, column sums, Adam) are
checked against the float64 numpy restatement in ``mlp_ref`` with FP32
tolerances: forward rtol 1e-4 / atol 1e-5, gradients within 1e-4 of the
gradient norm, Adam within 1e-6 absolute."""

import math

import numpy as np
import pytest

import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import tuner
from bitstreamzoo_b200.workloads import regex_dag_src, shaped_dag_src

import mlp_ref

pytestmark = pytest.mark.gpu


def _model(ctx, in_dim=20, hidden=64, layers=3, seed=7):
    m = tuner.CostModel(ctx, in_dim, hidden=hidden, layers=layers, seed=seed)
    return m, mlp_ref.dims_of(in_dim, hidden, layers)


def test_mlp_forward_matches_numpy(ctx):
    m, dims = _model(ctx)
    rng = np.random.default_rng(1)
    x = rng.normal(0, 1, (300, 20)).astype(np.float32)
    p = m.params()
    assert p.size == m.n_params == sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    ref = mlp_ref.forward(p, dims, x)[-1][:, 0]
    got = m.raw_predict(x)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("n", [1, 37, 256, 1000])
def test_mlp_gradients_match_numpy(ctx, n):
    m, dims = _model(ctx, in_dim=13, hidden=48, layers=2)
    rng = np.random.default_rng(n)
    # non-zero biases so every term of the bias gradients is exercised
    p = m.params()
    p += rng.normal(0, 0.05, p.size).astype(np.float32)
    m.set_params(p)
    x = rng.normal(0, 1, (n, 13)).astype(np.float32)
    y = rng.normal(0, 1, n).astype(np.float32)
    loss, g = m.raw_gradients(x, y)
    rloss, rg = mlp_ref.loss_and_grad(p, dims, x.astype(np.float64), y.astype(np.float64))
    assert loss == pytest.approx(rloss, rel=1e-4)
    err = np.linalg.norm(g - rg) / max(np.linalg.norm(rg), 1e-12)
    assert err < 1e-4, err


@pytest.mark.parametrize("wd", [0.0, 0.05])
def test_mlp_adam_steps_match_numpy(ctx, wd):
    m, dims = _model(ctx, in_dim=6, hidden=32, layers=2)
    m.set_weight_decay(wd)
    rng = np.random.default_rng(3)
    p = m.params().astype(np.float64)
    mom = np.zeros_like(p)
    vel = np.zeros_like(p)
    for step in range(1, 4):
        x = rng.normal(0, 1, (64, 6)).astype(np.float32)
        y = rng.normal(0, 1, 64).astype(np.float32)
        _, g = mlp_ref.loss_and_grad(p, dims, x.astype(np.float64), y.astype(np.float64))
        p, mom, vel = mlp_ref.adam_step(p, g, mom, vel, step, 1e-3, wd=wd)
        m.raw_train_step(x, y, 1e-3)
        np.testing.assert_allclose(m.params(), p, atol=2e-6, rtol=0)


def test_mlp_training_fits_a_smooth_function(ctx):
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (4000, 8)).astype(np.float32)
    f = np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * np.abs(X[:, 3])
    m = tuner.CostModel(ctx, 8, seed=11)
    losses = m.fit(X, np.exp(f), steps=800, lr=2e-3)
    assert np.mean(losses[-50:]) < 0.1 * np.mean(losses[:20])
    pred = np.log(m.predict_ms(X[:500]))
    assert np.corrcoef(pred, f[:500])[0, 1] > 0.97


def test_program_features_of_a_known_program(ctx):
    src = ("input stream a\ninput stream b\noutput stream o\noutput int c\n"
           "stream t = a + b\no = t << 3\nc = popcount(o)\n")
    f = tuner.program_features(ctx.compile(src))
    assert len(f) == 15
    assert f[0] == pytest.approx(math.log2(3))          # two ops
    assert f[5] == pytest.approx(0.5)                   # half are adds
    assert f[3] == pytest.approx(0.5)                   # half shift a temporary
    assert f[7] == pytest.approx(math.log2(3))          # depth 2
    assert f[8] == pytest.approx(1.0)                   # one add on the path
    assert f[10] == pytest.approx(math.log2(3))         # two inputs
    assert f[14] == pytest.approx(math.log2(3))         # two values live at once


def test_every_candidate_schedule_is_bit_exact(ctx):
    """All schedules in the search space give the plain backend's results."""
    src = regex_dag_src(n_ops=300, seed=99)
    nbits = (1 << 20) + 37
    rng = np.random.default_rng(9)
    nw = (nbits + 63) // 64
    ins = {}
    for i in range(8):
        w = rng.integers(0, 2**63, nw, dtype=np.uint64) * 2 + rng.integers(0, 2, nw, dtype=np.uint64)
        w[-1] &= np.uint64((1 << 37) - 1)
        ins[f"b{i}"] = w
    prog = ctx.compile(src)
    r = prog.run(nbits, bz.MODE_PLAIN)
    for k, v in ins.items():
        r.bind(k, v)
    r.execute()
    want = {f"o{j}": r.stream(f"o{j}") for j in range(4)}
    want_i = {f"p{j}": r.int(f"p{j}") for j in range(4)}
    # the candidate space, plus the uncapped grid (ctas_per_sm = -1: one
    # minimum-length range per warp) at two range lengths
    extra = [dict(bz.DEFAULT_SCHEDULE, ctas_per_sm=-1, range_steps=rs, prefetch=pf)
             for rs in (1, 64) for pf in (0, 1)]
    for s in list(tuner.CANDIDATES) + extra:
        f = prog.run(nbits, bz.MODE_FUSED)
        f.set_schedule(s)
        for k, v in ins.items():
            f.bind(k, v)
        f.execute()
        for k, v in want.items():
            assert np.array_equal(f.stream(k), v), (s, k)
        assert {k: f.int(k) for k in want_i} == want_i, s


def test_autotuner_sweep_and_cache(ctx, tmp_path):
    torch = pytest.importorskip("torch")
    src = shaped_dag_src(120, seed=4, window=8, p_add=0.1, max_shift=7)
    prog = ctx.compile(src)
    nbits = 1 << 22
    bufs, inputs = tuner._device_inputs(nbits, 8, 1)
    cands = tuner.candidate_space({"warps": (4, 8), "min_blocks": (4,), "prefetch": (0, 1), "cut_adds": (0,)},
                                  {"ctas_per_sm": (0,), "range_steps": (64,)}, seq={})
    path = str(tmp_path / "tune.json")
    at = tuner.Autotuner(ctx, cands, cache_path=path, reps=2)
    times = at.sweep(prog, src, nbits, inputs)
    assert len(times) == 4 and all(t > 0 for t in times.values())
    best = at.best(prog, src, nbits, inputs)
    assert tuner.schedule_key(best) == min(times, key=times.get)
    again = tuner.Autotuner(ctx, cands, cache_path=path)
    assert again.sweep(prog, src, nbits, inputs) == times
    del bufs, torch


def test_tuning_study_end_to_end(ctx):
    pytest.importorskip("torch")
    train, test = tuner.tuning_suite(n_train=4, n_test=2, seed=31)
    cands = tuner.candidate_space({"warps": (4, 8), "min_blocks": (4,), "prefetch": (0, 1), "cut_adds": (0, 1, 2)},
                                  {"ctas_per_sm": (0,), "range_steps": (64,)}, seq={})
    rep = tuner.study(ctx, train, test[:1], sizes=(1 << 21, 1 << 23), candidates=cands, sample_frac=0.5,
                      reps=2, steps=300)
    assert rep["loss_last"] < rep["loss_first"]
    assert len(rep["rows"]) == 2
    for r in rep["rows"]:
        assert 0 <= r["regret_top4"] <= r["regret_top1"] + 1e-12
        assert r["regret_default"] >= 0
        assert math.isfinite(r["best_ms"]) and r["best_ms"] > 0
    choice = rep["model"].choose(ctx.compile(test[0]), 1 << 23, cands)
    assert tuner.schedule_key(choice) in {tuner.schedule_key(s) for s in cands}


def test_shipped_cost_model_picks_from_the_space(ctx):
    m = tuner.CostModel.load_default(ctx)
    assert m is not None, "bitstreamzoo_b200/data/cost_model.npz is missing"
    prog = ctx.compile(regex_dag_src(n_ops=300, seed=5))
    keys = {tuner.schedule_key(s) for s in tuner.CANDIDATES}
    for nbits in (1 << 20, 1 << 26):
        assert tuner.schedule_key(m.choose(prog, nbits)) in keys


def test_cost_model_beats_default_and_random_pick_on_held_out_programs(ctx):
    """What the trained network gains over going without it: on programs it
    has not seen, its top-1 schedule is closer to the exhaustive best than
    the default schedule and than a random pick from the space (mean regret
    over held-out programs x lengths)."""
    pytest.importorskip("torch")
    train, test = tuner.tuning_suite(n_train=24, n_test=10, seed=53, max_ops=1500)
    rep = tuner.study(ctx, train, test, sizes=(1 << 22, 1 << 24), sample_frac=0.5, reps=2, steps=800,
                      precompile_threads=8)
    top1, dflt, rnd = (rep[k]["mean"] for k in ("regret_top1", "regret_default", "regret_random"))
    assert top1 < dflt, (top1, dflt)
    assert top1 < rnd, (top1, rnd)
