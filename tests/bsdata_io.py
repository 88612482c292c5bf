"""Minimal .bsdata writer for tests (format of benchmark/bsdata.py:1-17):
UTF-8 JSON header, NUL, little-endian packed stream bytes referenced by
{"_bin": [offset, nbytes]} / {"_array_bin": [count, offset, stride]}."""

import json
import math


def write_bsdata(path, bitlength, inputs=None, params=None, input_arrays=None, cases=None,
                 iterations=1, feedback=None):
    parts = []
    off = [0]

    def put(b):
        start = off[0]
        parts.append(b)
        off[0] += len(b)
        return start

    def enc_stream(v, nb):
        nbytes = max(1, math.ceil(nb / 8))
        return (v & ((1 << (8 * nbytes)) - 1)).to_bytes(nbytes, "little"), nbytes

    def enc_case(nb, inp, prm, arrs):
        h = {"bitlength": nb}
        if prm:
            h["params"] = prm
        if inp:
            sec = {}
            for k, v in inp.items():
                if 0 <= v < (1 << 52):
                    sec[k] = v
                else:
                    b, n = enc_stream(v, nb)
                    sec[k] = {"_bin": [put(b), n]}
            h["inputs"] = sec
        if arrs:
            sec = {}
            for k, a in arrs.items():
                count = max(a) + 1 if a else 0
                nbytes = max(1, math.ceil(nb / 8))
                start = off[0]
                for i in range(count):
                    put(enc_stream(a.get(i, 0), nb)[0])
                sec[k] = {"_array_bin": [count, start, nbytes]}
            h["input_arrays"] = sec
        return h

    if cases is not None:
        header = {"format": "bsdata", "version": 1,
                  "cases": [enc_case(c["bitlength"], c.get("inputs"), c.get("params"),
                                     c.get("input_arrays")) for c in cases]}
    else:
        header = {"format": "bsdata", "version": 1}
        header.update(enc_case(bitlength, inputs, params, input_arrays))
        if iterations > 1:
            header["iterations"] = iterations
        if feedback:
            header["feedback"] = feedback
    with open(path, "wb") as f:
        f.write(json.dumps(header, separators=(",", ":")).encode())
        f.write(b"\0")
        for p in parts:
            f.write(p)


def read_bsdata(path):
    """Reads a .bsdata file into {"cases": [case, ...]}, each case a dict with
    bitlength, params, inputs, input_arrays, expected, iterations, feedback;
    streams as Python ints, arrays as {index: value} (the format of
    benchmark/bsdata.py:196-270: _bin, _array_bin, _broadcast_pack markers)."""
    with open(path, "rb") as f:
        raw = f.read()
    sep = raw.index(b"\0")
    header = json.loads(raw[:sep].decode())
    blob = memoryview(raw)[sep + 1:]

    def value(v):
        if isinstance(v, dict):
            if "_bin" in v:
                off, nb = v["_bin"]
                return int.from_bytes(blob[off:off + nb], "little")
            if "_array_bin" in v:
                count, off, stride = v["_array_bin"]
                return {i: int.from_bytes(blob[off + i * stride:off + (i + 1) * stride], "little")
                        for i in range(count)}
            if "_broadcast_pack" in v:
                count, off, nb = v["_broadcast_pack"]
                bits = int.from_bytes(blob[off:off + nb], "little")
                return {i: (-1 if (bits >> i) & 1 else 0) for i in range(count)}
            return {k: value(x) for k, x in v.items()}
        if isinstance(v, list):
            return {i: value(x) for i, x in enumerate(v)}
        return v

    def case(h):
        return {"bitlength": h.get("bitlength", h.get("n_vectors", 0)),
                "params": h.get("params", {}),
                "inputs": {k: value(x) for k, x in h.get("inputs", {}).items()},
                "input_arrays": {k: value(x) for k, x in h.get("input_arrays", {}).items()},
                "expected": {k: value(x) for k, x in h.get("expected", {}).items()},
                "iterations": h.get("iterations", 1), "feedback": h.get("feedback") or {}}

    key = "cases" if "cases" in header else ("layers" if "layers" in header else None)
    return {"cases": [case(h) for h in header[key]] if key else [case(header)]}
