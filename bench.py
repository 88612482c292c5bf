#!/usr/bin/env python
"""Benchmark: input GB/s and HBM-roofline fraction of the B200 bitstream
executor, fused vs plain per-op, bit-exact.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload long_streams|regex_dag|matchstar] [--nbits BITS]
                    [--mode fused|plain]

Default workload (the one the headline metric is quoted on): two 2^32-bit
streams per GPU, A + B, A << {1, 63, 64, 1000}, A ^ B, A & ~B and the popcount
of each.  ``regex_dag`` is the 2,000-op regex-shaped DAG over 8 basis streams
of 2^29 bits; ``matchstar`` the 2^24-bit MatchStar primitive.

One step = one pass of the program over one set of input streams.  ``value``
is the input GB/s of the fused form with inputs resident in HBM (device time,
CUDA events on the executor's stream, max over ranks); ``e2e`` is the same
metric through the C ABI with pinned host inputs copied in and every output
stream + popcount copied out inside the timed region.  The default inputs
(1 GiB per rank) are larger than L2, so no L2 flush is needed between steps.

``--impl reference`` times the reference's own CPU executor (bsim, built from
the reference sources by oracle/Makefile, AVX-512 + OpenMP on all host cores)
on a bounded sample of the same workload; rank 0 alone runs it.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="long_streams",
                    choices=["long_streams", "regex_dag", "matchstar", "batched"])
    ap.add_argument("--instances", type=int, default=4096, help="batched: number of instances")
    ap.add_argument("--nbits", type=int, default=0, help="bits per stream (default: the workload's)")
    ap.add_argument("--mode", default="fused", choices=["fused", "plain"])
    ap.add_argument("--cpu-sample-bits", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-op comparison form")
    ap.add_argument("--schedule", default="tuned", choices=["tuned", "model", "model1", "default"],
                    help="fused-kernel schedule: the autotuner's pick (every candidate of the 16-schedule "
                         "space timed before the timed region), the fastest of the shipped cost model's 4 "
                         "best predictions, the model's top-1 pick (no timing), or the default")
    return ap.parse_args()


# ---------------------------------------------------------------- workloads --

class Workload:
    def __init__(self, name: str, nbits: int, seed: int):
        from bitstreamzoo_b200 import workloads as wl
        self.name = name
        self.nbits = nbits
        if name == "long_streams":
            self.src = wl.long_streams_src()
            self.inputs = wl.long_streams_inputs(nbits, seed=seed)
            self.out_streams = list(wl.LONG_OUTPUT_STREAMS)
            self.out_ints = list(wl.LONG_OUTPUT_INTS)
            self.desc = (f"long_streams: two {nbits}-bit streams; A+B, A<<{{1,63,64,1000}}, A^B, A&~B "
                         "+ 7 popcounts")
            self.data = "synthetic (seeded: A ~ Bernoulli(1/2), B all ones with zeros at p=2^-20)"
        elif name == "regex_dag":
            self.src = wl.regex_dag_src(2000, seed=20261206)
            self.inputs = wl.regex_dag_inputs(nbits, seed=seed)
            self.out_streams = [f"o{j}" for j in range(4)]
            self.out_ints = [f"p{j}" for j in range(4)]
            self.desc = (f"regex_dag: seeded 2000-op DAG (55% and/or/xor/andnot, 20% <<1, 10% add, 10% "
                         f"MatchStar, 5% not; uniform operand choice) over 8 basis streams of {nbits} bits")
            self.data = ("synthetic (seeded bytes: 70% a-z, 15% 0-9, 10% punctuation, 5% uniform; "
                         "transposed to basis bits)")
        else:
            self.src = wl.MATCHSTAR_SRC
            self.inputs = wl.matchstar_inputs(nbits, seed=seed)
            self.out_streams = ["r"]
            self.out_ints = ["n"]
            self.desc = f"matchstar: (((M&C)+C)^C)|M + popcount on {nbits}-bit streams"
            self.data = "synthetic (seeded: M ~ Bernoulli(1/64), C ~ Bernoulli(3/4))"
        self.stream_bytes = nbits // 8
        self.in_bytes = len(self.inputs) * self.stream_bytes
        self.out_bytes = len(self.out_streams) * self.stream_bytes + 8 * len(self.out_ints)

    def kernel_bytes(self, kname: str) -> float:
        s = self.stream_bytes
        table = {"k_and": 3 * s, "k_or": 3 * s, "k_xor": 3 * s, "k_andnot": 3 * s, "k_not": 2 * s,
                 "k_shl": 2 * s, "k_shr": 2 * s, "k_add": 3 * s, "k_popcount": s + 8, "k_fill": s,
                 "k_any": s}
        if kname.startswith("fused"):
            return self.in_bytes + self.out_bytes
        return table.get(kname, float("nan"))


def alu_roofline(prog, nbits: int, launch_ms: float, clocks) -> dict:
    """Integer-pipe roofline of a fused launch.  Algorithmic INT32 lane
    operations per 64-bit word of the post-DCE DAG: 2 per AND/OR/XOR/NOT/
    ANDNOT, 4 per shift (two funnel shifts and the neighbour word), 6 per ADD
    (64-bit add, carry-generate compare, carry-in add).  Peak: 148 SMs x 128
    INT32 lanes x the median SM clock seen while timing."""
    from bitstreamzoo_b200 import tuner
    f = tuner.program_features(prog)
    n_ops = round(2 ** f[0] - 1)
    per_word = n_ops * (2 * (f[1] + f[2]) + 4 * (f[3] + f[4] + f[6]) + 6 * f[5])
    words = (nbits + 63) // 64
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = 148 * 128 * mhz * 1e6 / 1e12
    achieved = per_word * words / (launch_ms * 1e-3) / 1e12
    return {"bound": "int32", "dag_ops": n_ops, "int32_ops_per_word": per_word, "achieved": achieved,
            "peak": peak, "unit": "Tops/s", "frac": achieved / peak,
            "peak_source": "nominal 148 SMs x 128 lanes x measured median SM clock"}


DEFAULT_BITS = {"long_streams": 1 << 32, "regex_dag": 1 << 29, "matchstar": 1 << 24}
DEFAULT_CPU_SAMPLE = {"long_streams": 1 << 28, "regex_dag": 1 << 26, "matchstar": 1 << 24}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def reduce_max(x: float, dist, device) -> float:
    """The maximum of x over all ranks (every rank gets it); x itself on one
    rank.  Times are reported as the slowest rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU side --

def cpu_model() -> str:
    """The host CPU's model name (as lscpu reports it), or "unknown"."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(workload: str, nbits: int, reps: int, warm: int = 1):
    """Reference CPU executor (bsim --backend simd_omp, AVX-512 + OpenMP, all
    host threads) on a bounded sample of the workload; falls back to the C
    port of the oracle when the reference binary was not built."""
    from bitstreamzoo_b200.bsdata import write_bsdata
    threads = os.cpu_count() or 1
    w = Workload(workload, nbits, seed=99)
    full = DEFAULT_BITS[workload]
    bsim = os.path.join(ROOT, "oracle", "_ref", "bsim")
    if os.path.exists(bsim):
        with tempfile.TemporaryDirectory() as td:
            prog = os.path.join(td, f"{workload}.bs")
            with open(prog, "w") as f:
                f.write(w.src)
            data = os.path.join(td, "in.bsdata")
            write_bsdata(data, nbits, w.inputs)
            env = dict(os.environ, OMP_NUM_THREADS=str(threads),
                       GLIBC_TUNABLES="glibc.cpu.x86_rep_stosb_threshold=2000000000")

            def run_bsim(backend, n_runs, n_warm):
                times = []
                for i in range(n_warm + n_runs):
                    out = os.path.join(td, "out.json")
                    with open(out, "w") as fo:
                        r = subprocess.run([bsim, prog, "--backend", backend, "--reuse-mem",
                                            "--input", data], stdout=fo, stderr=subprocess.PIPE,
                                           env=env, timeout=900)
                    if r.returncode != 0:
                        raise RuntimeError(r.stderr.decode()[-500:])
                    with open(out, "rb") as fi:
                        head = fi.read(4096).decode(errors="replace")
                    t = float(head.split('"exec_ms":', 1)[1].split(",", 1)[0])
                    if i >= n_warm:
                        times.append(t)
                return statistics.median(times)

            ms = run_bsim("simd_omp", reps, warm)
            # the reference's single-core AVX-512 form, once, beside it
            ms1 = run_bsim("simd", 1, 0)
        return {"value": w.in_bytes / (ms * 1e-3) / 1e9, "unit": "GB/s", "cores": threads,
                "cpu_model": cpu_model(),
                "single_core": {"value": w.in_bytes / (ms1 * 1e-3) / 1e9, "unit": "GB/s", "cores": 1,
                                "backend": "bsim --backend simd", "ms": ms1},
                "kind": "reference", "ms_per_step": ms,
                "sample": (f"{workload} program at {nbits} bits per stream (1/{max(1, full // nbits)} "
                           f"of the {full}-bit workload), bsim --backend simd_omp, "
                           f"OMP_NUM_THREADS={threads}, median exec_ms of {reps} runs")}
    from oracle import cwords, pyoracle
    prog = pyoracle.parse(w.src)
    times = []
    for i in range(warm + reps):
        t0 = time.perf_counter()
        cwords.run_straight_line(prog, nbits, w.inputs)
        if i >= warm:
            times.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.median(times)
    return {"value": w.in_bytes / (ms * 1e-3) / 1e9, "unit": "GB/s",
            "cores": cwords.lib().o_num_threads(), "cpu_model": cpu_model(), "kind": "port", "ms_per_step": ms,
            "sample": f"{workload} at {nbits} bits per stream, oracle C port, median of {len(times)}"}


def metric_name(workload: str) -> str:
    return f"input GB/s ({workload}, bit-exact)"


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, min(args.steps, 5))
    warm = min(1, args.warmup)
    sample = args.cpu_sample_bits or DEFAULT_CPU_SAMPLE[args.workload]
    cb = cpu_baseline(args.workload, sample, steps, warm=warm)
    line = {"metric": metric_name(args.workload), "value": cb["value"], "unit": "GB/s",
            "n_gpus": 0, "steps": steps, "warmup": warm, "ms_per_step": cb["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.workload}; CPU sample of {sample} bits per stream"},
            "cpu_baseline": {k: cb[k] for k in ("kind", "cores", "sample", "value", "unit")},
            "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side --

def run_ours(args, rank, world, local):
    import torch
    import bitstreamzoo_b200 as bz
    from bitstreamzoo_b200 import workloads as wl

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    hbm, hbm_src = peaks()
    nbits = args.nbits or DEFAULT_BITS[args.workload]
    nw = wl.n_words(nbits)
    W = Workload(args.workload, nbits, seed=20261204 + rank)
    ctx = bz.Context(local)
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    prog = ctx.compile(W.src)
    dev_in = {k: torch.from_numpy(v.view(np.int64)).to(dev) for k, v in W.inputs.items()}
    torch.cuda.synchronize()
    mode_of = {"fused": bz.MODE_FUSED, "plain": bz.MODE_PLAIN}

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, dev)

    sched, sched_src = dict(bz.DEFAULT_SCHEDULE), "default"
    if args.schedule == "tuned":
        from bitstreamzoo_b200 import tuner
        ins = {k: (t.data_ptr(), nw) for k, t in dev_in.items()}
        sched = tuner.Autotuner(ctx).best(prog, W.src, nbits, ins)
        sched_src = (f"autotuner: fastest of all {len(tuner.CANDIDATES)} candidates "
                     "(median of 3 device-timed runs each, before the timed region)")
    elif args.schedule in ("model", "model1"):
        from bitstreamzoo_b200 import tuner
        model = tuner.CostModel.load_default(ctx)
        if model is not None and args.schedule == "model1":
            sched, sched_src = model.choose(prog, nbits), "cost model top-1 (no timing)"
        elif model is not None:
            ins = {k: (t.data_ptr(), nw) for k, t in dev_in.items()}
            sched = model.choose(prog, nbits, top_k=4, inputs=ins)
            sched_src = "fastest of the cost model's top 4 (timed before the timed region)"

    def step(mode):
        r = prog.run(nbits, mode)
        if mode == bz.MODE_FUSED:
            r.set_schedule(sched)
        for k, t in dev_in.items():
            r.bind(k, ("borrow", t.data_ptr(), nw))
        st = r.execute()
        pops = {n: r.int(n) for n in W.out_ints}
        del r
        return st, pops

    forms = {}
    order = [args.mode] + ([] if args.no_plain else [m for m in ("fused", "plain") if m != args.mode])
    for name in order:
        mode = mode_of[name]
        try:
            for _ in range(args.warmup):
                st, pops = step(mode)
        except bz.BszError as e:
            forms[name] = {"unavailable": str(e)[:200]}
            continue
        compile_ms = st.get("compile_ms", 0.0)
        barrier()
        ctx.profile(True)
        clocks = Clocks(local)
        clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        launches = fallbacks = 0
        for _ in range(args.steps):
            st, pops = step(mode)
            launches += st["n_kernel_launches"]
            fallbacks += st["n_fused_fallbacks"]
        e1.record(ext)
        e1.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        ck = clocks.stop()
        prof = ctx.profile_report()
        ctx.profile(False)
        ms_max = max_over_ranks(ms)
        forms[name] = {"ms": ms_max, "launches": launches, "fused_fallbacks": fallbacks,
                       "profile": prof, "clocks": ck, "pops": pops,
                       "value": world * W.in_bytes * args.steps / (ms_max * 1e-3) / 1e9,
                       "hbm_frac_step": ((W.in_bytes + W.out_bytes) * args.steps / (ms_max * 1e-3) / 1e9) / hbm}

    # cheap host checks of popcounts the two forms must agree on (and, for the
    # long-stream workload, two that numpy computes exactly)
    if "pops" in forms.get("fused", {}) and "pops" in forms.get("plain", {}):
        forms["fused"]["agrees_with_plain"] = forms["fused"]["pops"] == forms["plain"]["pops"]
    if args.workload == "long_streams":
        ref_px = int(np.bitwise_count(W.inputs["A"] ^ W.inputs["B"]).sum())
        ref_pl64 = int(np.bitwise_count(W.inputs["A"][:-1]).sum())
        for f in forms.values():
            if "pops" in f:
                f["check"] = (f["pops"]["px"] == ref_px and f["pops"]["pl64"] == ref_pl64)

    # end to end through the C ABI: pinned host in, every output out
    e2e = None
    main = forms.get(args.mode, {})
    if not args.no_e2e and "ms" in main:
        mode = mode_of[args.mode]
        pinned_in = {k: torch.from_numpy(v.view(np.int64)).pin_memory() for k, v in W.inputs.items()}
        pinned_out = {n: torch.empty(nw, dtype=torch.int64).pin_memory() for n in W.out_streams}
        in_np = {k: t.numpy().view(np.uint64) for k, t in pinned_in.items()}
        out_np = {n: t.numpy().view(np.uint64) for n, t in pinned_out.items()}

        def e2e_step():
            r = prog.run(nbits, mode)
            for k, a in in_np.items():
                r.bind(k, a)
            r.execute()
            for n in W.out_streams:
                bz._lib.check(r.lib.bsz_get_stream(r.h, n.encode(), -1, out_np[n].ctypes.data, nw))
            vals = [r.int(n) for n in W.out_ints]
            del r
            return vals

        for _ in range(max(1, min(args.warmup, 2))):
            e2e_step()
        barrier()
        k = max(1, min(args.steps, 5))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(ext)
        for _ in range(k):
            e2e_step()
        e1.record(ext)
        e1.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        barrier()
        ms = max_over_ranks(max(e0.elapsed_time(e1), wall))
        e2e = {"value": world * W.in_bytes * k / (ms * 1e-3) / 1e9, "unit": "GB/s",
               "h2d_bytes_per_step": W.in_bytes, "d2h_bytes_per_step": len(W.out_streams) * nw * 8 + 8 * len(W.out_ints),
               "steps": k, "ms_per_step": ms / k}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(args.workload, args.cpu_sample_bits or DEFAULT_CPU_SAMPLE[args.workload], 5)
        except Exception as e:  # noqa: BLE001
            cb = {"unavailable": str(e)[:200]}

    if rank == 0:
        prof = main.get("profile", {})
        roof = None
        if prof:
            kname, kv = max(prof.items(), key=lambda kv: kv[1]["ms"])
            per_launch_ms = kv["ms"] / max(1, kv["launches"])
            bytes_launch = W.kernel_bytes(kname)
            achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
            traffic = None
            tpath = os.path.join(ROOT, "profiles", "traffic.json")
            if os.path.exists(tpath):
                with open(tpath) as f:
                    traffic = json.load(f).get(f"{args.workload}:{kname}")
            roof = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm,
                    "peak_source": hbm_src, "unit": "GB/s", "frac": achieved / hbm,
                    "traffic": traffic, "bytes_per_launch": bytes_launch,
                    "launch_ms": per_launch_ms,
                    "kernel_share": kv["ms"] / max(1e-9, sum(x["ms"] for x in prof.values()))}
            if kname.startswith("fused"):
                roof["alu"] = alu_roofline(prog, nbits, per_launch_ms, main.get("clocks"))
        line = {
            "metric": metric_name(args.workload),
            "value": main.get("value"), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main.get("ms", float("nan")) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": W.data,
            "config": {"workload": W.desc + " (per GPU)", "form": args.mode, "bits_per_stream": nbits,
                       "schedule": sched, "schedule_source": sched_src,
                       "l2": ("inputs larger than L2; no flush needed" if W.in_bytes > (126 << 20)
                              else "inputs fit in L2 (reported, not roofline-judged)"),
                       "parallelism": f"replicas x{world} (independent stream sets)"},
            "hbm_frac_step": main.get("hbm_frac_step"),
            "roofline": roof,
            "cpu_baseline": cb,
            "e2e": e2e,
            "gpu_launches": main.get("launches"),
            "clocks": main.get("clocks"),
            "forms": {k: {kk: vv for kk, vv in v.items() if kk != "pops"} for k, v in forms.items()},
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_batched(args, rank, world, local):
    """Batched uneven instances (one graph-captured persistent launch per
    step): 16 seeded 300-op regex-shaped DAGs, instance lengths log-uniform
    in [2^12, 2^26] bits, 8 inputs ~ Bernoulli(1/2) generated on the device,
    4 outputs + 4 popcounts each.  value = input GB/s over all instances."""
    import torch
    import bitstreamzoo_b200 as bz
    from bitstreamzoo_b200 import workloads as wl

    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    hbm, hbm_src = peaks()
    srcs, plan = wl.batched_plan(n_instances=args.instances, n_dags=16, lo_log2=12, hi_log2=26, ops=300,
                                 seed=20261207 + rank)
    ctx = bz.Context(local)
    progs = [ctx.compile(s) for s in srcs]
    g = torch.Generator(device="cuda").manual_seed(20261208 + rank)
    keep, instances = [], []
    in_bytes = out_bytes = 0
    for dag, bits in plan:
        nw = wl.n_words(bits)
        din = [torch.randint(-2**63, 2**63 - 1, (nw,), dtype=torch.int64, device="cuda", generator=g)
               for _ in range(8)]
        if bits % 64:
            m = (1 << (bits % 64)) - 1
            for t in din:
                t[-1:].bitwise_and_(m)
        dout = [torch.empty(nw, dtype=torch.int64, device="cuda") for _ in range(4)]
        keep += din + dout
        instances.append((dag, bits, [t.data_ptr() for t in din], [t.data_ptr() for t in dout]))
        in_bytes += 8 * bits // 8
        out_bytes += 4 * bits // 8 + 4 * 8
    torch.cuda.synchronize()
    t0 = time.time()
    b = bz.Batch(ctx, progs, instances)
    build_s = time.time() - t0
    ext = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    for _ in range(max(3, args.warmup)):
        b.launch()
        b.finish()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.profile(True)
    clocks = Clocks(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(args.steps):
        b.launch()
    e1.record(ext)
    st = b.finish()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ck = clocks.stop()
    prof = ctx.profile_report()
    ctx.profile(False)
    ms = reduce_max(ms, dist, torch.device("cuda", local))
    # spot check: a few instances against their own single-program runs (fused form)
    rng = np.random.default_rng(rank)
    check = True
    for i in rng.choice(len(plan), size=min(6, len(plan)), replace=False):
        dag, bits, ins, outs = instances[int(i)]
        r = progs[dag].run(bits, bz.MODE_FUSED)
        for j in range(8):
            r.bind(f"b{j}", ("borrow", ins[j], wl.n_words(bits)))
        r.execute()
        check = check and [r.int(f"p{j}") for j in range(4)] == b.ints(int(i))
    per_step = ms / args.steps
    kname, kv = (max(prof.items(), key=lambda kv: kv[1]["ms"]) if prof else ("batch", {"ms": ms, "launches": 1}))
    launch_ms = kv["ms"] / max(1, kv["launches"])
    achieved = (in_bytes + out_bytes) / (launch_ms * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": "input GB/s (batched uneven instances, bit-exact)",
            "value": world * in_bytes * args.steps / (ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded: inputs ~ Bernoulli(1/2) generated on the device)",
            "config": {"workload": f"batched: {len(plan)} instances of 16 seeded 300-op regex-shaped DAGs, "
                                   "lengths log-uniform in [2^12, 2^26] bits, 8 inputs / 4 outputs + 4 popcounts each",
                       "input_bytes": in_bytes, "output_bytes": out_bytes, "work_items": b.items,
                       "build_s": build_s, "l2": "inputs (all instances) far larger than L2",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm,
                         "peak_source": hbm_src, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                         "bytes_per_launch": in_bytes + out_bytes, "launch_ms": launch_ms},
            "cpu_baseline": None, "e2e": None,
            "gpu_launches": args.steps, "clocks": ck, "check": check, "fused_fallbacks": st.get("n_fused_fallbacks"),
        }
        print(json.dumps(line), flush=True)
    del b
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        if args.workload == "batched":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched executor; "
                                  "its CPU path runs one program per process"}), flush=True)
            return
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
