"""Shared pytest configuration: the ``gpu`` marker and fixture helpers."""

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_golden(name):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        return json.load(f)["cases"]


def parse_hex(v):
    return int(v, 16)


def decode_case(rec):
    """Golden record -> (src, nbits, inputs, params, arrays)."""
    inputs = {k: int(v, 16) for k, v in rec["inputs"].items()}
    arrays = {k: {int(i): int(x, 16) for i, x in v.items()} for k, v in rec["input_arrays"].items()}
    return rec["src"], rec["bitlength"], inputs, dict(rec["params"]), arrays


def expected_masked(rec):
    """Expected outputs masked to the bitlength, as the reference harness
    compares them (benchmark/base.py:437-472): streams masked, ints exact."""
    mask = (1 << rec["bitlength"]) - 1
    out = {}
    for k, v in rec["expected"].items():
        if isinstance(v, dict) and "int" in v:
            out[k] = v["int"]
        elif isinstance(v, dict):
            out[k] = {int(i): int(x, 16) & mask for i, x in v.items()}
        else:
            out[k] = int(v, 16) & mask
    return out


def mask_outputs(out, ints, nbits):
    mask = (1 << nbits) - 1
    res = {}
    for k, v in out.items():
        if k in ints:
            res[k] = v
        elif isinstance(v, dict):
            res[k] = {i: x & mask for i, x in v.items()}
        else:
            res[k] = v & mask
    return res


def _reference_tree():
    # the oracle recipe holds the one definition of the reference tree location
    v = os.environ.get("BSZ_REFERENCE_TREE")
    if v:
        return v
    import subprocess
    oracle_dir = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")
    r = subprocess.run(["make", "-s", "-C", oracle_dir, "print-ref"], capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


REFERENCE_TREE = _reference_tree()
has_reference = os.path.isdir(os.path.join(REFERENCE_TREE, "simulator", "pythonsim"))


@pytest.fixture(scope="session")
def ctx():
    import bitstreamzoo_b200 as bz
    c = bz.Context(0)
    yield c
    c.close()


def run_golden_case(ctx, rec, mode):
    """Runs a golden record through the C ABI; returns (masked outputs, op_count)."""
    src, nbits, inputs, params, arrays = decode_case(rec)
    r = ctx.run(src, nbits, inputs, params, arrays, mode=mode)
    got = {}
    mask = (1 << nbits) - 1
    for k, v in rec["expected"].items():
        if isinstance(v, dict) and "int" in v:
            got[k] = r.int(k)
        elif isinstance(v, dict):
            idx = r.array_indices(k) or []
            got[k] = {int(i): (r.stream_int(k, int(i)) & mask if int(i) in idx else 0) for i in v}
        else:
            got[k] = r.stream_int(k) & mask
    return got, r.stats["op_count"], r
