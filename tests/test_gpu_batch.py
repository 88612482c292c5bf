"""Batched uneven instances: one graph-captured persistent launch runs many
instances of several programs with different stream lengths; every instance
must match its own CPU oracle run word for word (outputs) and exactly (ints).
"""

import numpy as np
import pytest

import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import workloads as wl
from oracle import cwords, pyoracle

torch = pytest.importorskip("torch")


def _run_batch(ctx, srcs, plan, seed, schedule=None, replays=2):
    progs = [ctx.compile(s) for s in srcs]
    parsed = [pyoracle.parse(s) for s in srcs]
    rng = np.random.default_rng(seed)
    keep, instances, host = [], [], []
    for dag, bits in plan:
        p = parsed[dag]
        nw = wl.n_words(bits)
        ins = {name: wl.random_words(rng, bits) for name in p["inputs"]}
        din = [torch.from_numpy(ins[name].view(np.int64)).cuda() for name in p["inputs"]]
        dout = [torch.full((nw,), -1, dtype=torch.int64, device="cuda") for _ in p["outputs"]]
        keep += din + dout
        instances.append((dag, bits, [t.data_ptr() for t in din], [t.data_ptr() for t in dout]))
        host.append((ins, dout))
    torch.cuda.synchronize()
    b = bz.Batch(ctx, progs, instances, schedule)
    for _ in range(replays):
        b.launch()
        st = b.finish()
    for i, (dag, bits) in enumerate(plan):
        p = parsed[dag]
        ins, dout = host[i]
        ref_out, ref_pops = cwords.run_straight_line(p, bits, ins)
        mask_last = np.uint64(((1 << (bits % 64)) - 1) if bits % 64 else (1 << 64) - 1)
        for j, name in enumerate(p["outputs"]):
            exp = ref_out[name].copy()
            exp[-1] &= mask_last
            got = dout[j].cpu().numpy().view(np.uint64)
            assert np.array_equal(got, exp), f"instance {i} (dag {dag}, {bits} bits) output {name}"
        ints = b.ints(i)
        assert ints == [ref_pops[n] for n in p["output_ints"]], f"instance {i}"
    return b, st


@pytest.mark.gpu
def test_batched_uneven_regex_dags(ctx):
    srcs, plan = wl.batched_plan(n_instances=96, n_dags=16, lo_log2=12, hi_log2=18, ops=300, seed=5)
    b, st = _run_batch(ctx, srcs, plan, seed=1)
    assert b.items >= len(plan)
    assert st["n_fused_launches"] == 2


@pytest.mark.gpu
def test_batched_mixed_programs_and_ragged_lengths(ctx):
    srcs = [wl.long_streams_src(), wl.MATCHSTAR_SRC, wl.regex_dag_src(300, seed=11)]
    plan = [(k % 3, bits) for k, bits in enumerate([1, 63, 64, 65, 4095, 4096, 100003, 1 << 20,
                                                     (1 << 21) + 7, 777, 2 ** 17 + 1, 5])]
    _run_batch(ctx, srcs, plan, seed=2)


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [{"warps": 2, "range_steps": 32, "prefetch": 0},
                                      {"warps": 8, "range_steps": 256, "min_blocks": 2},
                                      {"layout": 1, "warps": 4, "min_blocks": 1},
                                      {"layout": 1, "warps": 8, "min_blocks": 1},
                                      {"layout": 1, "chunk_words": 8, "warps": 4, "min_blocks": 1}])
def test_batched_schedules(ctx, schedule):
    srcs, plan = wl.batched_plan(n_instances=40, n_dags=4, lo_log2=12, hi_log2=20, ops=200, seed=9)
    _run_batch(ctx, srcs, plan, seed=3, schedule=schedule)


@pytest.mark.gpu
def test_batch_rejects_programs_with_control_flow(ctx):
    src = "input stream a\noutput stream r\nr = a\nif (a) {\n r = ~a\n}\n"
    p = ctx.compile(src)
    t = torch.zeros(4, dtype=torch.int64, device="cuda")
    with pytest.raises(bz.BszError):
        bz.Batch(ctx, [p], [(0, 200, [t.data_ptr()], [t.data_ptr()])])


@pytest.mark.gpu
def test_batched_thread_sequential_uneven_and_ragged(ctx):
    """The thread-sequential batch form on uneven regex DAG instances and on
    ragged lengths (instances shorter than one lane chunk, masked last words)."""
    srcs, plan = wl.batched_plan(n_instances=64, n_dags=8, lo_log2=6, hi_log2=21, ops=300, seed=15)
    _run_batch(ctx, srcs, plan, seed=4, schedule={"layout": 1, "warps": 4, "min_blocks": 1})
    srcs = [wl.long_streams_src(), wl.MATCHSTAR_SRC, wl.regex_dag_src(300, seed=11)]
    plan = [(k % 3, bits) for k, bits in enumerate([1, 63, 64, 65, 4095, 4096, 100003, 1 << 20,
                                                     (1 << 21) + 7, 777, 2 ** 17 + 1, 5])]
    _run_batch(ctx, srcs, plan, seed=6, schedule={"layout": 1, "warps": 8, "min_blocks": 1})
