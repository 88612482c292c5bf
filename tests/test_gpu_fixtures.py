"""The reference's unit fixtures through the drop-in binary.

``benchmark/run_all.py --unit --backend cuda`` runs every app program on every
unit fixture through ``bsim_cuda <prog.bs> --word-bits=64 --reuse-mem --input
<file.bsdata>`` (benchmark/base.py:198-254) and compares each case's outputs
with the ``expected`` of the fixture, stream outputs masked to the bitlength
and ints exactly (base.py:437-472); generated cases reach the binary as a JSON
document on stdin (base.py:211-218, 261-275).  This file does the same with
``bitstreamzoo_b200/lib/bsim_cuda`` over the fixtures that
tests/golden/fixtures/collect_fixtures.py copied from the reference (the
committed .bsdata files, the small generated cases with the reference Python
interpreter's outputs, two iterations/feedback cases), and also checks each
case's ``op_count`` against the reference's.  Every fixture runs in the
default (auto) mode; the per-op plain form, 32-bit word mode and the stdin
form run on subsets sized to keep the file within minutes.
"""

import json
import os
import subprocess
from collections import defaultdict

import pytest

from bsdata_io import read_bsdata
from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "fixtures")
EXE = os.path.join(ROOT, "bitstreamzoo_b200", "lib", "bsim_cuda")


def _manifest():
    with open(os.path.join(FIX, "manifest.json")) as f:
        return json.load(f)["cases"]


def _by_program():
    groups = defaultdict(list)
    for rec in _manifest():
        groups[rec["program"]].append(rec)
    return sorted(groups.items())


def _parse_outputs(outputs):
    # the harness's _parse_csim_outputs (base.py:310-330)
    res = {}
    for k, v in outputs.items():
        if isinstance(v, str) and v.startswith("0x"):
            res[k] = int(v, 16)
        elif isinstance(v, dict):
            res[k] = {int(i): (int(x, 16) if isinstance(x, str) and x.startswith("0x") else x) for i, x in v.items()}
        else:
            res[k] = v
    return res


def _check_case(got_outputs, case, int_names):
    """The harness's _check_expected (base.py:437-472); returns a mismatch text or None."""
    got = _parse_outputs(got_outputs)
    nb = case["bitlength"]
    mask = (1 << nb) - 1 if nb > 0 else None
    for k, exp in case["expected"].items():
        if k not in got:
            return f"missing output {k}"
        masked = mask is not None and k not in int_names
        if isinstance(exp, dict):
            act = got[k]
            if not isinstance(act, dict):
                return f"{k}: expected an array"
            for i, e in exp.items():
                a = act.get(i, 0)
                if masked:
                    a, e = a & mask, e & mask
                if a != e:
                    return f"{k}[{i}] differs"
        else:
            a, e = got[k], exp
            if masked:
                a, e = a & mask, e & mask
            if a != e:
                return f"{k} differs"
    return None


def _int_outputs(prog_path):
    names = set()
    with open(prog_path) as f:
        for line in f:
            t = line.split()
            if len(t) >= 3 and t[0] == "output" and t[1] == "int":
                names.add(t[2].split("[")[0])
    return names


def _run(prog, args, stdin=None, timeout=900):
    env = dict(os.environ, GLIBC_TUNABLES="glibc.cpu.x86_rep_stosb_threshold=2000000000")
    r = subprocess.run([EXE, prog, *args], input=stdin, capture_output=True, text=True, timeout=timeout, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout)
    return out if isinstance(out, list) else [out]


def _check_file(prog, rec, extra, int_names):
    data = read_bsdata(os.path.join(FIX, rec["data"]))
    outs = _run(prog, ["--word-bits=64", "--reuse-mem", *extra, "--input", os.path.join(FIX, rec["data"])])
    assert len(outs) == len(data["cases"]), rec["case"]
    for i, (o, c) in enumerate(zip(outs, data["cases"])):
        err = _check_case(o["outputs"], c, int_names)
        assert err is None, f"{rec['program']} / {rec['case']} case {i} ({' '.join(extra) or 'auto'}): {err}"
        if rec.get("op_counts"):
            assert o["op_count"] == rec["op_counts"][i], (rec["case"], i, o["op_count"], rec["op_counts"][i])


PLAIN_MAX_OPS = 3_000_000   # the per-op form of bnn's 27.5 M-op cases takes minutes


@pytest.mark.gpu
@pytest.mark.parametrize("program,recs", _by_program(), ids=[p for p, _ in _by_program()])
def test_unit_fixtures_auto_and_plain(program, recs):
    prog = os.path.join(FIX, program)
    ints = _int_outputs(prog)
    for rec in recs:
        _check_file(prog, rec, [], ints)
        if sum(rec.get("op_counts") or [0]) <= PLAIN_MAX_OPS:
            _check_file(prog, rec, ["--mode=plain"], ints)


@pytest.mark.gpu
@pytest.mark.parametrize("program,recs", _by_program(), ids=[p for p, _ in _by_program()])
def test_unit_fixtures_32bit_words(program, recs):
    """The cuda32 backends (run_all.py:67-72): the first fixture of every program."""
    prog = os.path.join(FIX, program)
    _check_file(prog, recs[0], ["--word-bits=32"], _int_outputs(prog))


def _json_doc(case):
    # the harness's build_input_json (base.py:261-275) with its hex rule for
    # ints above 52 bits or negative
    def val(v):
        return hex(v) if v < 0 or v.bit_length() > 52 else v

    d = {"inputs": {k: val(v) for k, v in case["inputs"].items()}, "params": case["params"],
         "n_vectors": case["bitlength"]}
    if case["input_arrays"]:
        d["input_arrays"] = {k: [val(a.get(i, 0)) for i in range(max(a) + 1 if a else 0)]
                             for k, a in case["input_arrays"].items()}
    if case["iterations"] > 1:
        d["iterations"] = case["iterations"]
    if case["feedback"]:
        d["feedback"] = case["feedback"]
    return json.dumps(d)


@pytest.mark.gpu
def test_generated_fixtures_through_stdin_json():
    """Generated and feedback cases in the stdin form the harness uses for them."""
    recs = [r for r in _manifest() if r["kind"] in ("generated", "feedback")]
    assert recs
    for rec in recs:
        prog = os.path.join(FIX, rec["program"])
        case = read_bsdata(os.path.join(FIX, rec["data"]))["cases"][0]
        out = _run(prog, ["--word-bits=64", "--reuse-mem"], stdin=_json_doc(case))[0]
        err = _check_case(out["outputs"], case, _int_outputs(prog))
        assert err is None, f"{rec['program']} / {rec['case']}: {err}"
        assert out["op_count"] == rec["op_counts"][0]


def test_fixture_manifest_is_complete():
    """Every manifest entry has its program and data file (no GPU needed)."""
    recs = _manifest()
    assert len(recs) >= 120
    for rec in recs:
        assert os.path.exists(os.path.join(FIX, rec["program"])), rec["program"]
        assert os.path.exists(os.path.join(FIX, rec["data"])), rec["data"]
        with open(os.path.join(FIX, rec["data"]), "rb") as f:
            head = f.read(1 << 20)
        header = json.loads(head[:head.index(b"\0")])   # the JSON header only: no stream decoding
        cases = header.get("cases", header.get("layers", [header]))
        assert len(cases) == rec["n_cases"] and all(x.get("expected") for x in cases), rec["data"]
        assert len(rec["op_counts"]) == rec["n_cases"], rec["data"]
