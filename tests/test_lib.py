"""CPU-side checks of the native library: it loads, exports every symbol of
include/bsz.h, parses/validates programs like the reference front end, and
the bsim_cuda driver reads .bsdata files (no GPU needed for any of this)."""

import ctypes
import json
import random
import os
import re
import subprocess

import pytest

from conftest import ROOT, load_golden, decode_case
from oracle import pyoracle
import bitstreamzoo_b200 as bz
from bitstreamzoo_b200 import _lib
from bsdata_io import write_bsdata


def header_symbols():
    with open(os.path.join(ROOT, "include", "bsz.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bsz_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)


def test_version():
    assert b"sm_100a" in _lib.load().bsz_version()


def _compile(src):
    lib = _lib.load()
    b = src.encode()
    h = lib.bsz_compile(None, b, len(b))
    err = None if h else _lib.last_error()
    if h:
        lib.bsz_program_free(h)
    return err


def test_parse_errors_match_reference_classes():
    assert _compile("input stream a\noutput stream r\nr = a & a\n") is None
    assert "primary" in _compile("input stream a\noutput stream r\nr = a & a | a\n")
    assert "condition must be a variable" in _compile(
        "input stream a\noutput stream r\nif (a & a) {\n r = a\n}\n")
    assert "expected stream expression" in _compile("input stream a\noutput stream r\nr = \n")
    assert "unexpected character" in _compile("input stream a\nr = a @ a\n")
    assert "popcount arg must be a variable" in _compile("input stream a\noutput int c\nc = popcount(~a)\n")


def test_static_op_count_matches_oracle_on_golden_programs():
    lib = _lib.load()
    n = 0
    for rec in load_golden("random_programs"):
        src, nbits, inputs, params, arrays = decode_case(rec)
        b = src.encode()
        h = lib.bsz_compile(None, b, len(b))
        assert h, _lib.last_error()
        names = (ctypes.c_char_p * max(1, len(params)))(*[k.encode() for k in params])
        vals = (ctypes.c_int64 * max(1, len(params)))(*params.values())
        got = lib.bsz_static_ops(h, names, vals, len(params))
        lib.bsz_program_free(h)
        assert got == pyoracle.count_static_ops(pyoracle.parse(src), params), rec["name"]
        n += 1
    assert n > 100


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(bz.BszError):
        bz.Context(0)


def test_cli_dump_input_reads_bsdata(tmp_path):
    exe = bz.bsim_cuda_path()
    prog = tmp_path / "p.bs"
    prog.write_text("input stream a\ninput stream m[3]\noutput stream r\nr = a\n")
    a = (1 << 200) | 12345
    path = tmp_path / "x.bsdata"
    write_bsdata(str(path), 203, inputs={"a": a, "s": 7}, params={"K": 3},
                 input_arrays={"m": {0: 5, 2: (1 << 150)}})
    out = subprocess.run([exe, str(prog), "--input", str(path), "--dump-input"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout)
    assert d["bitlength"] == 203
    assert int(d["inputs"]["a"], 16) == a
    assert int(d["inputs"]["s"], 16) == 7
    assert d["params"] == {"K": 3}
    assert int(d["input_arrays"]["m"]["2"], 16) == 1 << 150
    assert int(d["input_arrays"]["m"]["1"], 16) == 0


def test_cli_parse_error_exit_code(tmp_path):
    exe = bz.bsim_cuda_path()
    prog = tmp_path / "p.bs"
    prog.write_text("input stream a\noutput stream r\nr = a & a ^ a\n")
    out = subprocess.run([exe, str(prog)], input='{"inputs": {}, "n_vectors": 8}',
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 1
    assert "Parse error" in out.stderr


def test_cli_dump_input_large_stream_hex(tmp_path):
    """A 5 MiB stream through the memory-mapped reader and the table-driven,
    multi-threaded hex encoder (long outputs are split across threads), plus
    a stream whose bytes end mid-word."""
    exe = bz.bsim_cuda_path()
    prog = tmp_path / "p.bs"
    prog.write_text("input stream a\ninput stream b\noutput stream r\nr = a\n")
    nbits = 5 * 8 * (1 << 20) + 21
    rng = random.Random(5)
    a = rng.getrandbits(nbits) | (1 << (nbits - 1))
    b = rng.getrandbits(13 * 8 + 5)
    path = tmp_path / "big.bsdata"
    write_bsdata(str(path), nbits, inputs={"a": a, "b": b})
    out = subprocess.run([exe, str(prog), "--input", str(path), "--dump-input"],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout)
    assert d["inputs"]["a"] == hex(a)
    assert int(d["inputs"]["b"], 16) == b


def test_noalloc_add_rejects_bitlength_outside_its_words():
    # checked before any device call, so this runs without a GPU
    lib = _lib.load()
    dummy = ctypes.c_void_p(16)
    for bad in (-5, 64 * 10 + 1):
        assert lib.bsz_add_noalloc(dummy, dummy, dummy, 10, bad, None) != 0
        assert "bitlength" in _lib.last_error()
