"""Bit-exact parity at the benchmark configurations' full sizes.

* long_streams at 2^32 bits per stream (the headline workload): all 7
  output streams word for word and all 7 popcounts, against the word-level
  C oracle, for the plain per-op form and both fused forms;
* the 2,000-op regex DAG at 2^29 bits per basis stream: the 4 outputs and
  popcounts, same forms;
* the batched plan in full (4,096 instances of 16 300-op DAGs, 2^12..2^26
  bits): 256 instances, the 16 longest among them, against their own CPU
  oracle runs (outputs and popcounts);
* the reference's own AVX-512 executor (``bsim --backend simd_omp``, built
  from its sources by oracle/Makefile) on 2^24-bit samples of long_streams
  and the regex DAG: its output hex must equal ours.

Sizes are the benchmark's, so these tests take tens of seconds each (input
generation and the oracle run on the host).
"""

import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import workloads as wl
from bitstreamzoo_b200.bsdata import write_bsdata
from conftest import ROOT
from oracle import cwords, pyoracle

torch = pytest.importorskip("torch")

FORMS = [(bz.MODE_PLAIN, None), (bz.MODE_FUSED, {"layout": 0}), (bz.MODE_FUSED, {"layout": 1})]


def _mask_last(nbits):
    return np.uint64(((1 << (nbits % 64)) - 1) if nbits % 64 else (1 << 64) - 1)


def _check_forms(ctx, src, nbits, inputs, out_streams):
    prog = pyoracle.parse(src)
    ref_out, ref_pops = cwords.run_straight_line(prog, nbits, inputs)
    nw = wl.n_words(nbits)
    dev_in = {k: torch.from_numpy(v.view(np.int64)).cuda() for k, v in inputs.items()}
    torch.cuda.synchronize()
    cprog = ctx.compile(src)
    for mode, sched in FORMS:
        r = cprog.run(nbits, mode)
        if sched:
            r.set_schedule(sched)
        for k, t in dev_in.items():
            r.bind(k, ("borrow", t.data_ptr(), nw))
        st = r.execute()
        for name in out_streams:
            got = r.stream(name)
            exp = ref_out[name]
            last_ok = (got[-1] & _mask_last(nbits)) == (exp[-1] & _mask_last(nbits))
            body_ok = np.array_equal(got[:-1], exp[:-1])
            if not (body_ok and last_ok):
                bad = int(np.argmax(got[:-1] != exp[:-1])) if not body_ok else nw - 1
                raise AssertionError(f"mode {mode} {sched} output {name}: first bad word {bad} of {nw}")
            del got
        for name, v in ref_pops.items():
            assert r.int(name) == v, (mode, sched, name)
        del r
    return ref_pops


@pytest.mark.gpu
def test_long_streams_full_size_2e32_bits(ctx):
    nbits = 1 << 32
    inputs = wl.long_streams_inputs(nbits)
    _check_forms(ctx, wl.long_streams_src(), nbits, inputs, wl.LONG_OUTPUT_STREAMS)


@pytest.mark.gpu
def test_regex_dag_full_size_2e29_bits(ctx):
    nbits = 1 << 29
    inputs = wl.regex_dag_inputs(nbits)
    _check_forms(ctx, wl.regex_dag_src(), nbits, inputs, [f"o{j}" for j in range(4)])


@pytest.mark.gpu
def test_batched_full_plan_against_oracle(ctx):
    srcs, plan = wl.batched_plan()   # 4,096 instances, 16 DAGs, 2^12..2^26 bits
    progs = [ctx.compile(s) for s in srcs]
    parsed = [pyoracle.parse(s) for s in srcs]
    g = torch.Generator(device="cuda").manual_seed(77)
    keep, instances, devs = [], [], []
    for dag, bits in plan:
        nw = wl.n_words(bits)
        din = [torch.randint(-2**63, 2**63 - 1, (nw,), dtype=torch.int64, device="cuda", generator=g)
               for _ in range(8)]
        if bits % 64:
            for t in din:
                t[-1:].bitwise_and_((1 << (bits % 64)) - 1)
        dout = [torch.full((nw,), -1, dtype=torch.int64, device="cuda") for _ in range(4)]
        keep += din + dout
        instances.append((dag, bits, [t.data_ptr() for t in din], [t.data_ptr() for t in dout]))
        devs.append((din, dout))
    torch.cuda.synchronize()
    b = bz.Batch(ctx, progs, instances)
    b.launch()
    b.finish()
    longest = sorted(range(len(plan)), key=lambda i: -plan[i][1])[:16]
    others = [int(i) for i in np.random.default_rng(5).permutation(len(plan)) if int(i) not in set(longest)]
    for i in longest + others[:240]:
        dag, bits = plan[i]
        p = parsed[dag]
        din, dout = devs[i]
        ins = {name: din[j].cpu().numpy().view(np.uint64) for j, name in enumerate(p["inputs"])}
        ref_out, ref_pops = cwords.run_straight_line(p, bits, ins)
        for j, name in enumerate(p["outputs"]):
            exp = ref_out[name].copy()
            exp[-1] &= _mask_last(bits)
            got = dout[j].cpu().numpy().view(np.uint64)
            assert np.array_equal(got, exp), f"instance {i} (dag {dag}, {bits} bits) output {name}"
        assert b.ints(i) == [ref_pops[n] for n in p["output_ints"]], f"instance {i}"
    del b


def _bsim_outputs(src, nbits, inputs):
    bsim = os.path.join(ROOT, "oracle", "_ref", "bsim")
    if not os.path.exists(bsim):
        pytest.skip("reference CPU binary not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as td:
        prog = os.path.join(td, "p.bs")
        with open(prog, "w") as f:
            f.write(src)
        data = os.path.join(td, "in.bsdata")
        write_bsdata(data, nbits, inputs)
        env = dict(os.environ, GLIBC_TUNABLES="glibc.cpu.x86_rep_stosb_threshold=2000000000")
        r = subprocess.run([bsim, prog, "--backend", "simd_omp", "--reuse-mem", "--input", data],
                           capture_output=True, text=True, env=env, timeout=600)
        assert r.returncode == 0, r.stderr[-500:]
        return json.loads(r.stdout)


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["long_streams", "regex_dag"])
def test_matches_reference_avx512_bsim_on_2e24_samples(ctx, workload):
    nbits = 1 << 24
    if workload == "long_streams":
        src, inputs = wl.long_streams_src(), wl.long_streams_inputs(nbits, seed=41)
        outs, ints = wl.LONG_OUTPUT_STREAMS, wl.LONG_OUTPUT_INTS
    else:
        src, inputs = wl.regex_dag_src(), wl.regex_dag_inputs(nbits, seed=42)
        outs, ints = [f"o{j}" for j in range(4)], [f"p{j}" for j in range(4)]
    ref = _bsim_outputs(src, nbits, inputs)["outputs"]
    mask = (1 << nbits) - 1
    for mode, sched in FORMS:
        r = ctx.run(src, nbits, inputs, mode=mode, schedule=sched)
        for name in outs:
            assert r.stream_int(name) & mask == int(ref[name], 16), (workload, mode, sched, name)
        for name in ints:
            assert r.int(name) == ref[name], (workload, mode, sched, name)
