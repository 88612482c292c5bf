"""The oracle is pinned before it is trusted.

* against the golden vectors produced by the reference's own interpreter
  (tests/golden/*.json, made by tests/golden/make_golden.py);
* against the reference interpreter itself on fresh seeded programs, when the
  reference tree is present in this container;
* the word-level C oracle against the same golden vectors.
"""

import os
import random

import numpy as np
import pytest

from conftest import decode_case, expected_masked, has_reference, load_golden, mask_outputs, REFERENCE_TREE
from oracle import cwords, pyoracle
import progen

GROUPS = ["random_programs", "kat_ops", "tail_corners"]


def _all_cases():
    for g in GROUPS:
        for rec in load_golden(g):
            yield g, rec


@pytest.mark.parametrize("group", GROUPS)
def test_pyoracle_matches_golden(group):
    n = 0
    for rec in load_golden(group):
        src, nbits, inputs, params, arrays = decode_case(rec)
        if "error" in rec:
            with pytest.raises(Exception):
                pyoracle.run_source(src, nbits, inputs, params, arrays)
            continue
        out, ops, _ = pyoracle.run_source(src, nbits, inputs, params, arrays)
        ints = {k for k, v in rec["expected"].items() if isinstance(v, dict) and "int" in v}
        assert mask_outputs(out, ints, nbits) == expected_masked(rec), rec["name"]
        assert ops == rec["op_count"], rec["name"]
        n += 1
    assert n > 10


def test_pyoracle_unmasked_values_match_reference_exactly():
    """Unmasked values (negative = tail bit set) agree too, not just in-range bits."""
    for rec in load_golden("tail_corners"):
        if "error" in rec:
            continue
        src, nbits, inputs, params, arrays = decode_case(rec)
        out, _, _ = pyoracle.run_source(src, nbits, inputs, params, arrays)
        for k, v in rec["expected"].items():
            if isinstance(v, str):
                assert out[k] == int(v, 16), rec["name"]


@pytest.mark.skipif(not has_reference, reason="reference tree not present")
def test_pyoracle_matches_reference_interpreter_on_fresh_programs():
    import sys
    sys.path.insert(0, REFERENCE_TREE)
    from simulator.pythonsim import parse as rparse
    from simulator.pythonsim.interpreter import Interpreter
    for seed in range(5000, 5120):
        rng = random.Random(seed)
        nbits = rng.choice([1, 3, 64, 65, 191, 500])
        c = progen.random_case(rng, nbits, n_stmts=30)
        try:
            it = Interpreter(bitlength=nbits)
            ref = it.run(rparse(c["src"]), c["inputs"], c["params"], c["input_arrays"])
            ref_err = None
        except Exception as e:  # noqa: BLE001
            ref_err = e
        if ref_err is not None:
            with pytest.raises(Exception):
                pyoracle.run_source(c["src"], nbits, c["inputs"], c["params"], c["input_arrays"])
            continue
        out, ops, _ = pyoracle.run_source(c["src"], nbits, c["inputs"], c["params"], c["input_arrays"])
        assert out == ref and ops == it.op_count, seed


def test_parse_errors():
    with pytest.raises(pyoracle.OracleThreeAddrError):
        pyoracle.parse("input stream a\noutput stream r\nr = a & a | a\n")
    with pytest.raises(pyoracle.OracleThreeAddrError):
        pyoracle.parse("input stream a\noutput stream r\nif (a & a) {\n r = a\n}\n")
    with pytest.raises(pyoracle.OracleParseError):
        pyoracle.parse("input stream a\noutput stream r\nr = \n")
    with pytest.raises(pyoracle.OracleParseError):
        pyoracle.parse("input stream a\nfor i in 0..3 {\n")


def test_while_limit():
    src = "output int c\nstream o = ONES\nint n = 0\nwhile (o) {\n n = n + 1\n}\nc = n\n"
    with pytest.raises(pyoracle.OracleRuntimeError):
        pyoracle.run_source(src, 8, {})


def test_static_op_count():
    src = ("input stream a\noutput stream r\nparam int K\nstream t = a\n"
           "for i in 0..K {\n t = t << 1\n t = t ^ a\n}\nif (a) {\n r = ~t\n}\n")
    prog = pyoracle.parse(src)
    assert pyoracle.count_static_ops(prog, {"K": 5}) == 11


@pytest.mark.parametrize("k", [0, 1, 31, 63, 64, 65, 127, 128, 200])
def test_c_oracle_matches_golden_shifts(k):
    for rec in load_golden("kat_ops"):
        if rec["name"].startswith(f"op<<{k}_") or rec["name"].startswith(f"op>>{k}_"):
            src, nbits, inputs, params, arrays = decode_case(rec)
            prog = pyoracle.parse(src)
            words = {n: cwords.int_to_words(v, nbits) for n, v in inputs.items()}
            outs, _ = cwords.run_straight_line(prog, nbits, words)
            exp = expected_masked(rec)
            assert cwords.words_to_int(outs["r"]) & ((1 << nbits) - 1) == exp["r"], rec["name"]


def test_c_oracle_matches_golden_ops_and_carries():
    n = 0
    for rec in load_golden("kat_ops"):
        if "<<" in rec["name"] or ">>" in rec["name"]:
            continue
        src, nbits, inputs, params, arrays = decode_case(rec)
        prog = pyoracle.parse(src)
        words = {name: cwords.int_to_words(v, nbits) for name, v in inputs.items()}
        outs, pops = cwords.run_straight_line(prog, nbits, words)
        exp = expected_masked(rec)
        for k, v in exp.items():
            if k in pops:
                assert pops[k] == v, rec["name"]
            else:
                assert cwords.words_to_int(outs[k]) & ((1 << nbits) - 1) == v, rec["name"]
        n += 1
    assert n > 50


def test_c_oracle_random_straight_line_vs_pyoracle():
    rng = random.Random(3)
    for _ in range(40):
        nbits = rng.choice([64, 100, 1000, 4097])
        src, _ = progen.random_program(rng, n_stmts=25, allow_ctrl=False)
        # keep the straight-line subset the word oracle lowers: drop array use
        if "[" in src.split("stream tmp[4]")[1]:
            continue
        prog = pyoracle.parse(src)
        inputs = {f"in{i}": progen.rand_stream(rng, nbits) for i in range(3)}
        try:
            ref, _, _ = pyoracle.run_source(src, nbits, inputs, {"K": 2}, {"arr_in": {}})
        except Exception:
            continue
        words = {k: cwords.int_to_words(v, nbits) for k, v in inputs.items()}
        try:
            outs, _ = cwords.run_straight_line(prog, nbits, words)
        except ValueError:
            continue
        mask = (1 << nbits) - 1
        for k in ("out0", "out1"):
            assert cwords.words_to_int(outs[k]) & mask == ref[k] & mask


def test_basis_restatements_agree():
    from oracle import basis
    rng = np.random.default_rng(17)
    for n in (0, 1, 7, 63, 64, 65, 200, 1000):
        payload = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        ints = basis.basis_ints(payload)
        words = basis.basis_words(payload)
        for i in range(8):
            assert cwords.words_to_int(words[i]) == ints[i]
            assert words[i].size == (n + 63) // 64


def test_basis_oracle_matches_reference_s2p_goldens():
    """oracle/basis.py against payload_to_basis_bits(_fast) of the reference
    (benchmark/apps/regex/src/run.py:164-187), via tests/golden/s2p_golden.json."""
    import json
    from oracle import basis
    with open(os.path.join(os.path.dirname(__file__), "golden", "s2p_golden.json")) as f:
        cases = json.load(f)["cases"]
    assert len(cases) >= 20
    for c in cases:
        payload = bytes.fromhex(c["payload"])
        want = [int(h, 16) for h in c["basis"]]
        words = basis.basis_words(payload)
        got = [int.from_bytes(w.astype("<u8").tobytes(), "little") for w in words]
        assert got == want, c["name"]
        if len(payload) <= 4096:
            assert basis.basis_ints(payload) == want, c["name"]
