"""Collect the reference's unit fixtures into this directory (test data only).

Run in a container that has the reference tree (its location: --ref, else
$BSZ_REFERENCE_TREE, else the oracle recipe's ``make -s -C oracle print-ref``)
and the reference CPU binary (``make -C oracle ref``):

    python tests/golden/fixtures/collect_fixtures.py [--ref <reference tree>]

What ``benchmark/run_all.py --unit`` runs, per app (benchmark/base.py:537-738,
GenericDomain discovery base.py:864-920): every program ``src/*.bs`` against
every case of ``datasets/tests/tests.json`` that has no ``provenance`` block
(base.py:354-366), where a case is either

* a committed ``.bsdata`` file (with ``expected`` outputs in its header):
  copied here unchanged, or
* a ``generated`` case, whose inputs come from the app's ``run_generated``
  (``src/run.py``) and reach the backend in the stdin-JSON form.  It is run
  here through a recording backend: each call's inputs, with the outputs of
  the reference Python interpreter (the normative semantics) as
  ``expected``, are written as a ``.bsdata`` file with the reference's own
  writer (benchmark/bsdata.py:58-193).  Optional cases whose real-data input
  is absent from the tree are skipped, as the harness skips them, and so are
  generated cases whose file would exceed --max-generated-bytes (2 MB by
  default: the 1M-vector circuit, cipher and gemv cases are 5-40 MB each;
  the manifest lists them under ``skipped``).

Every case also records the reference's dynamic op count: the Python
interpreter's for generated cases, the reference C++ ``bsim``'s for
committed files.  Two more cases exercise the ``iterations``/``feedback``
input form (the harness loop of base.py:43-66), which no unit fixture uses.

Outputs: ``manifest.json`` and one folder per app with its programs and data.
"""

from __future__ import annotations

import argparse
import json
import os
import random
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))


def reference_tree():
    v = os.environ.get("BSZ_REFERENCE_TREE")
    if v:
        return v
    return subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                          capture_output=True, text=True, check=True).stdout.strip()


def bsim_op_counts(bsim, prog_path, data_path):
    """op_count of every case of a .bsdata file, from the reference CPU binary."""
    env = dict(os.environ, OMP_NUM_THREADS="4",
               GLIBC_TUNABLES="glibc.cpu.x86_rep_stosb_threshold=2000000000")
    r = subprocess.run([bsim, prog_path, "--word-bits=64", "--reuse-mem", "--backend", "simd_omp",
                        "--input", data_path], capture_output=True, text=True, env=env, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(f"bsim failed on {data_path}: {r.stderr[-500:]}")
    out = json.loads(r.stdout)
    return [o["op_count"] for o in (out if isinstance(out, list) else [out])]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    ap.add_argument("--max-generated-bytes", type=int, default=2_000_000)
    args = ap.parse_args()
    ref = os.path.abspath(args.ref or reference_tree())
    sys.path.insert(0, ref)
    import importlib

    from benchmark import base                                # noqa: E402  (reference harness)
    from benchmark.bsdata import read_bsdata, write_bsdata   # noqa: E402

    bsim = os.path.join(ROOT, "oracle", "_ref", "bsim")
    if not os.path.exists(bsim):
        raise SystemExit("build the reference CPU binary first: make -C oracle ref")
    apps_dir = os.path.join(ref, "benchmark", "apps")
    for d in os.listdir(HERE):
        p = os.path.join(HERE, d)
        if os.path.isdir(p) and not d.startswith("_"):
            shutil.rmtree(p)
    manifest = []
    skipped = []
    bsim_jobs = []
    for app in sorted(os.listdir(apps_dir)):
        tj = os.path.join(apps_dir, app, "datasets", "tests", "tests.json")
        src_dir = os.path.join(apps_dir, app, "src")
        if not os.path.exists(tj) or not os.path.isdir(src_dir):
            continue
        with open(tj) as f:
            data = json.load(f)
        out_dir = os.path.join(HERE, app)
        os.makedirs(out_dir, exist_ok=True)
        try:
            run_generated = getattr(importlib.import_module(f"benchmark.apps.{app}.src.run"),
                                    "run_generated", None)
        except ImportError:
            run_generated = None
        for pf in sorted(f for f in os.listdir(src_dir) if f.endswith(".bs")):
            pname = pf[:-3]
            shutil.copy(os.path.join(src_dir, pf), os.path.join(out_dir, pf))
            prog = base.BenchmarkDomain.load_bs(os.path.join(src_dir, pf))
            ints = set(prog.program.output_int_names)
            cases = data if isinstance(data, list) else data.get(pname, data.get("_default", []))
            n_gen = 0
            for case in cases:
                if "provenance" in case:
                    continue
                df = case.get("data_file")
                src_path = os.path.join(apps_dir, app, "datasets", "tests", df) if df else None
                if src_path and os.path.exists(src_path) and df.endswith(".bsdata"):
                    dst = os.path.join(out_dir, df)
                    if not os.path.exists(dst):
                        shutil.copy(src_path, dst)
                    fd = read_bsdata(dst)
                    rec = {"app": app, "program": f"{app}/{pf}", "case": case["name"], "kind": "bsdata",
                           "data": f"{app}/{df}", "n_cases": len(fd.get("cases", [fd])), "op_counts": None}
                    manifest.append(rec)
                    bsim_jobs.append(rec)
                elif case.get("category") == "generated" and run_generated is not None:
                    calls = []

                    class Recorder(base.PythonBackend):
                        def run(self, prog_, inputs, params=None, input_arrays=None, bitlength=0,
                                iterations=1, feedback=None, bsdata_path=None):
                            out, ops, ms = super().run(prog_, inputs, params, input_arrays, bitlength,
                                                       iterations, feedback)
                            calls.append((dict(inputs), dict(params or {}), dict(input_arrays or {}),
                                          bitlength, iterations, dict(feedback or {}), out, ops))
                            return out, ops, ms

                    try:
                        run_generated(case, prog, backend=Recorder())
                    except (FileNotFoundError, ImportError, OSError) as e:
                        if case.get("optional"):
                            print(f"skip optional {app}/{pname}/{case['name']}: {e}")
                            continue
                        raise
                    for i, (inp, prm, arrs, nb, it, fb, out, ops) in enumerate(calls):
                        name = f"gen_{pname}_{n_gen}.bsdata"
                        n_gen += 1
                        mask = (1 << nb) - 1 if nb > 0 else None
                        expected = {}
                        for k, v in out.items():
                            if k in ints:
                                expected[k] = int(v)
                            elif isinstance(v, dict):
                                expected[k] = {int(j): (int(x) & mask if mask else int(x)) for j, x in v.items()}
                            else:
                                expected[k] = int(v) & mask if mask else int(v)
                        path = os.path.join(out_dir, name)
                        write_bsdata(path, nb, inputs=inp, params=prm,
                                     input_arrays=arrs, expected=expected, iterations=it, feedback=fb)
                        if os.path.getsize(path) > args.max_generated_bytes:
                            skipped.append({"program": f"{app}/{pf}", "case": case["name"],
                                            "bytes": os.path.getsize(path)})
                            os.remove(path)
                            n_gen -= 1
                            continue
                        manifest.append({"app": app, "program": f"{app}/{pf}",
                                         "case": case["name"] + (f" [call {i}]" if len(calls) > 1 else ""),
                                         "kind": "generated", "data": f"{app}/{name}", "n_cases": 1,
                                         "op_counts": [ops]})
                    print(f"generated {app}/{pname}/{case['name']}: {len(calls)} call(s)", flush=True)
    # iterations / feedback: a small program looped with an output fed back
    fb_dir = os.path.join(HERE, "feedback")
    os.makedirs(fb_dir, exist_ok=True)
    fb_src = ("input stream x\ninput stream y\noutput stream z\noutput int n\n"
              "stream t = x + y\nz = t ^ x\nn = popcount(z)\n")
    with open(os.path.join(fb_dir, "feedback.bs"), "w") as f:
        f.write(fb_src)
    fprog = base.BenchmarkDomain.load_bs(os.path.join(fb_dir, "feedback.bs"))
    rng = random.Random(20261204)
    for nb, it in ((1000, 5), (70000, 3)):
        x, y = rng.getrandbits(nb), rng.getrandbits(nb)
        out, ops, _ = base.PythonBackend().run(fprog, {"x": x, "y": y}, {}, {}, nb, it, {"z": "x"})
        name = f"feedback_{nb}.bsdata"
        write_bsdata(os.path.join(fb_dir, name), nb, inputs={"x": x, "y": y},
                     expected={"z": int(out["z"]) & ((1 << nb) - 1), "n": int(out["n"])},
                     iterations=it, feedback={"z": "x"})
        manifest.append({"app": "feedback", "program": "feedback/feedback.bs",
                         "case": f"{it} iterations, z -> x, {nb} bits", "kind": "feedback",
                         "data": f"feedback/{name}", "n_cases": 1, "op_counts": [ops]})

    def job(rec):
        rec["op_counts"] = bsim_op_counts(bsim, os.path.join(HERE, rec["program"]),
                                          os.path.join(HERE, rec["data"]))
    with ThreadPoolExecutor(max_workers=4) as ex:
        list(ex.map(job, bsim_jobs))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "tests/golden/fixtures/collect_fixtures.py",
                   "harness": "benchmark/base.py:537-738 (run_all.py --unit)", "cases": manifest,
                   "skipped": skipped}, f, indent=1)
    print(f"{len(manifest)} fixture entries")


if __name__ == "__main__":
    main()
