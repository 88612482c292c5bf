"""The N > 1 host paths on CPU: two gloo ranks (no GPU).

bench.py runs one replica per GPU and reports the slowest rank's time; its
reference arm runs on rank 0 only and the other ranks exit without work."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.reduce_max(1.0 + 1.5 * rank, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_reduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 2.5, 1: 2.5}


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "bsim")),
                    reason="reference CPU binary not built")
def test_reference_arm_prints_one_line_under_two_ranks():
    port = 29700 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--workload", "matchstar", "--cpu-sample-bits", str(1 << 20)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"


def test_streams_as_locals_keeps_the_operations():
    """The reference runs in bench.py use the program with its output streams
    as locals: the same operations and popcounts, no stream outputs."""
    sys.path.insert(0, ROOT)
    import bench
    from bitstreamzoo_b200 import workloads as wl
    from oracle import pyoracle
    for src, outs in ((wl.long_streams_src(), wl.LONG_OUTPUT_STREAMS),
                      (wl.regex_dag_src(300, seed=3), [f"o{j}" for j in range(4)])):
        loc = bench.streams_as_locals(src, outs)
        assert "output stream" not in loc
        nbits = 3000
        ins = {n: (i * 0x9E3779B97F4A7C15 + 12345) % (1 << nbits) for i, n in
               enumerate(pyoracle.parse(src)["inputs"])}
        full, ops_full, _ = pyoracle.run_source(src, nbits, ins)
        only, ops_loc, _ = pyoracle.run_source(loc, nbits, ins)
        assert ops_full == ops_loc
        assert {k: v for k, v in full.items() if k not in outs} == only
