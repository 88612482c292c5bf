"""Golden vectors for the byte -> basis-bit transposition, from the reference.

Run in a container that has the reference tree (its location: --ref, else
$BSZ_REFERENCE_TREE, else ``make -s -C oracle print-ref``):

    python tests/golden/make_s2p_golden.py [--ref <reference tree>]

Imports the regex app's own ``payload_to_basis_bits`` and
``payload_to_basis_bits_fast`` (benchmark/apps/regex/src/run.py:164-187),
runs both on seeded payloads (the regex workload's byte mix, all-0x00/0xFF
runs, every byte value, and ragged lengths around word boundaries) and writes
``s2p_golden.json``: per case the payload (hex) and the 8 basis streams as
hex ints, which both reference functions agree on.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_tree():
    v = os.environ.get("BSZ_REFERENCE_TREE")
    if v:
        return v
    return subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                          capture_output=True, text=True, check=True).stdout.strip()


def payloads():
    sys.path.insert(0, ROOT)
    from bitstreamzoo_b200.workloads import regex_bytes
    rng = np.random.default_rng(20261210)
    out = [("empty", b""), ("one_byte", b"\xa5"), ("all_values", bytes(range(256))),
           ("zeros_1000", bytes(1000)), ("ones_777", b"\xff" * 777)]
    for n in (1, 7, 8, 63, 64, 65, 127, 128, 129, 511, 512, 513, 4095, 4096, 4097, 65537):
        out.append((f"regex_mix_{n}", regex_bytes(n, seed=1000 + n).tobytes()))
    for n in (100, 1000, 10000):
        out.append((f"uniform_{n}", rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    args = ap.parse_args()
    sys.path.insert(0, args.ref or reference_tree())
    from benchmark.apps.regex.src.run import payload_to_basis_bits, payload_to_basis_bits_fast
    cases = []
    for name, p in payloads():
        slow = payload_to_basis_bits(p)
        fast = payload_to_basis_bits_fast(p)
        assert slow == fast, name
        cases.append({"name": name, "payload": p.hex(), "basis": [hex(slow[i]) for i in range(8)]})
    with open(os.path.join(HERE, "s2p_golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_s2p_golden.py",
                   "reference": "benchmark/apps/regex/src/run.py:164-187 (payload_to_basis_bits, _fast)",
                   "cases": cases}, f, separators=(",", ":"))
    print(len(cases), "cases")


if __name__ == "__main__":
    main()
