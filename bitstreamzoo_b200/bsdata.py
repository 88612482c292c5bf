""".bsdata writer (the reference's test-data format, benchmark/bsdata.py:1-17).

UTF-8 JSON header + NUL + little-endian packed stream bytes.  Streams go to
the binary section as {"_bin": [offset, nbytes]}; numpy uint64 word arrays
are written without conversion to Python ints, so multi-GB inputs are cheap.
"""

from __future__ import annotations

import json
import math

import numpy as np


def write_bsdata(path: str, bitlength: int, inputs: dict, params: dict | None = None) -> None:
    nbytes = max(1, math.ceil(bitlength / 8))
    header = {"format": "bsdata", "version": 1, "bitlength": bitlength}
    if params:
        header["params"] = params
    sec = {}
    blobs = []
    off = 0
    for name, v in inputs.items():
        if isinstance(v, np.ndarray):
            raw = np.ascontiguousarray(v, dtype=np.uint64).view(np.uint8)[:nbytes]
        else:
            raw = np.frombuffer((int(v) & ((1 << (8 * nbytes)) - 1)).to_bytes(nbytes, "little"),
                                dtype=np.uint8)
        if raw.size < nbytes:
            raw = np.concatenate([raw, np.zeros(nbytes - raw.size, dtype=np.uint8)])
        sec[name] = {"_bin": [off, nbytes]}
        blobs.append(raw)
        off += nbytes
    header["inputs"] = sec
    with open(path, "wb") as f:
        f.write(json.dumps(header, separators=(",", ":")).encode())
        f.write(b"\0")
        for b in blobs:
            b.tofile(f)
