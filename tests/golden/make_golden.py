"""Generate the committed golden vectors from the reference implementation.

Run in a container that has the reference tree (its location: --ref, else
$BSZ_REFERENCE_TREE, else the oracle recipe's default, ``make -s -C oracle
print-ref``):

    python tests/golden/make_golden.py [--ref <reference tree>]

Every expected value is produced by the reference's normative Python
interpreter (simulator/pythonsim/interpreter.py), imported from the reference
tree.  Where the reference C++ CPU binary has been built by
``make -C oracle ref`` its result is recorded next to it (``bsim_agrees``), so
the fixtures also document where the two reference executors diverge.

Outputs (small JSON files next to this script):
  random_programs.json  seeded random programs covering every DSL form
  kat_ops.json          per-operator known-answer cases (sizes, shift
                        amounts and carry patterns of the reference's native
                        tests test_ops.cpp / test_kernels.cu)
  tail_corners.json     the bits->=N ("tail") corner cases
  configs_small.json    the benchmark workload shapes at reduced sizes
"""

from __future__ import annotations

import argparse
import json
import os
import random
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import progen  # noqa: E402


def to_hex(v: int) -> str:
    return hex(v)


class Ref:
    def __init__(self, ref_root: str):
        sys.path.insert(0, ref_root)
        from simulator.pythonsim import parse  # type: ignore
        from simulator.pythonsim.interpreter import Interpreter  # type: ignore
        self.parse = parse
        self.Interpreter = Interpreter
        bsim = os.path.join(ROOT, "oracle", "_ref", "bsim")
        self.bsim = bsim if os.path.exists(bsim) else None

    def run(self, src, nbits, inputs, params, arrays):
        prog = self.parse(src)
        it = self.Interpreter(bitlength=nbits)
        out = it.run(prog, dict(inputs), dict(params), {k: dict(v) for k, v in arrays.items()})
        ints = set(prog.output_int_names)
        return out, it.op_count, ints

    def run_bsim(self, src, nbits, inputs, params, arrays):
        if self.bsim is None:
            return None
        import tempfile
        with tempfile.NamedTemporaryFile("w", suffix=".bs", delete=False) as f:
            f.write(src)
            path = f.name
        payload = {"inputs": {k: hex(v) for k, v in inputs.items()},
                   "params": params, "n_vectors": nbits,
                   "input_arrays": {k: [hex(v.get(i, 0)) for i in range(max(v) + 1)]
                                    for k, v in arrays.items() if v}}
        try:
            r = subprocess.run([self.bsim, path, "--reuse-mem"], input=json.dumps(payload),
                               capture_output=True, text=True, timeout=60)
        finally:
            os.unlink(path)
        if r.returncode != 0:
            return {"error": r.stderr.strip()[:200]}
        return json.loads(r.stdout)


def case_record(ref: Ref, name, src, nbits, inputs, params=None, arrays=None):
    params = params or {}
    arrays = arrays or {}
    rec = {"name": name, "src": src, "bitlength": nbits,
           "inputs": {k: to_hex(v) for k, v in inputs.items()},
           "params": params,
           "input_arrays": {k: {str(i): to_hex(x) for i, x in v.items()} for k, v in arrays.items()}}
    try:
        out, ops, ints = ref.run(src, nbits, inputs, params, arrays)
    except Exception as e:  # reference raised: record the error class
        rec["error"] = type(e).__name__
        return rec
    exp = {}
    for k, v in out.items():
        if k in ints:
            exp[k] = {"int": v}
        elif isinstance(v, dict):
            exp[k] = {str(i): to_hex(x) for i, x in v.items()}
        else:
            exp[k] = to_hex(v)
    rec["expected"] = exp
    rec["op_count"] = ops
    b = ref.run_bsim(src, nbits, inputs, params, arrays)
    if b is not None:
        rec["bsim_agrees"] = bsim_agrees(b, out, ints, nbits)
    return rec


def bsim_agrees(b, out, ints, nbits) -> bool:
    if "error" in b:
        return False
    mask = (1 << nbits) - 1
    got = b["outputs"]
    for k, v in out.items():
        if k not in got:
            return False
        if k in ints:
            if got[k] != v:
                return False
        elif isinstance(v, dict):
            for i, x in v.items():
                g = int(got[k].get(str(i), "0x0"), 16)
                if (g & mask) != (x & mask):
                    return False
        else:
            if (int(got[k], 16) & mask) != (v & mask):
                return False
    return True


def gen_random(ref: Ref, n_cases: int = 140):
    recs = []
    seed = 1000
    sizes = [1, 5, 63, 64, 65, 100, 127, 128, 129, 200, 640, 1000, 4097]
    errors = 0
    while len(recs) < n_cases:
        rng = random.Random(seed)
        nbits = sizes[seed % len(sizes)]
        c = progen.random_case(rng, nbits, n_stmts=rng.randrange(8, 40))
        rec = case_record(ref, f"random_{seed}", c["src"], nbits, c["inputs"],
                          c["params"], c["input_arrays"])
        seed += 1
        if "error" in rec:
            if errors >= 6:
                continue
            errors += 1
        recs.append(rec)
    return recs


def gen_kats(ref: Ref):
    """Per-operator cases at the sizes / shift amounts / carry patterns of the
    reference's native tests (test_ops.cpp:114-421, test_kernels.cu:82-382)."""
    recs = []
    rng = random.Random(42)
    word_counts = [1, 7, 8, 15, 16, 100]
    ones64 = (1 << 64) - 1
    for nw in word_counts:
        for nbits in (64 * nw, 64 * nw - 17 if nw > 1 else 47):
            a = rng.getrandbits(nbits)
            b = rng.getrandbits(nbits)
            for op in ("&", "|", "^", "+"):
                src = f"input stream a\ninput stream b\noutput stream r\nr = a {op} b\n"
                recs.append(case_record(ref, f"op{op}_n{nbits}", src, nbits, {"a": a, "b": b}))
            src = "input stream a\noutput stream r\nr = ~a\n"
            recs.append(case_record(ref, f"op~_n{nbits}", src, nbits, {"a": a}))
            src = "input stream a\noutput int c\nc = popcount(a)\n"
            recs.append(case_record(ref, f"popcount_n{nbits}", src, nbits, {"a": a}))
            for k in (0, 1, 31, 63, 64, 65, 127, 128, 200):
                for op in ("<<", ">>"):
                    src = f"input stream a\noutput stream r\nr = a {op} {k}\n"
                    recs.append(case_record(ref, f"op{op}{k}_n{nbits}", src, nbits, {"a": a}))
    # carry patterns (test_kernels.cu:254-382): single word, 3-word chain,
    # all-ones chains, multi-block and block-boundary carries
    add_src = "input stream a\ninput stream b\noutput stream r\noutput int c\nr = a + b\nc = popcount(r)\n"

    def words(ws):
        return sum(w << (64 * i) for i, w in enumerate(ws))

    patterns = {
        "single_word": ([5], [7]),
        "carry_one_word": ([ones64, 0], [1, 0]),
        "chain3": ([ones64, ones64, 0], [1, 0, 0]),
        "no_carry": ([1, 2, 3], [4, 5, 6]),
        "all_ones_x8": ([ones64] * 8, [1] + [0] * 7),
        "all_ones_512": ([ones64] * 512, [1] + [0] * 511),
        "all_ones_1029": ([ones64] * 1029, [1] + [0] * 1028),
    }
    for bound in (255, 256, 511, 512, 2047, 2048):
        n = bound + 48
        a = [rng.getrandbits(64) if j % 97 == 0 else 0 for j in range(n)]
        b = [rng.getrandbits(64) if j % 89 == 0 else 0 for j in range(n)]
        a[bound - 1] = ones64
        b[bound - 1] = 1
        for j in range(bound, min(bound + 40, n)):
            a[j] = ones64
            b[j] = 0
        patterns[f"boundary_{bound}"] = (a, b)
    # long propagate runs crossing many tiles, carry generated mid-stream
    a = [ones64] * 3000
    b = [0] * 3000
    b[3] = 1 << 63
    a[3] = 1 << 63
    patterns["propagate_3000"] = (a, b)
    for name, (wa, wb) in patterns.items():
        nbits = 64 * len(wa)
        recs.append(case_record(ref, f"add_{name}", add_src, nbits, {"a": words(wa), "b": words(wb)}))
        recs.append(case_record(ref, f"add_{name}_m5", add_src, nbits - 5,
                                {"a": words(wa) & ((1 << (nbits - 5)) - 1),
                                 "b": words(wb) & ((1 << (nbits - 5)) - 1)}))
    return recs


def gen_tail_corners(ref: Ref):
    """Cases where bits at or above the bitlength are observable."""
    recs = []
    rng = random.Random(7)
    progs = {
        "not_then_shr": "input stream x\noutput stream r\nstream t = ~x\nr = t >> 1\n",
        "ones_copy_shr": "output stream r\nstream o = ONES\nr = o >> 1\n",
        "ones_operand_shr": "output stream r\nr = ONES >> 1\n",
        "ones_xor_ones_if": ("input stream x\noutput stream r\nstream o = ONES\n"
                             "stream z = o ^ ONES\nr = x\nif (z) {\n r = ~x\n}\n"),
        "ones_copy_or_shr": ("input stream x\noutput stream r\nstream o = ONES\n"
                             "stream t = o | x\nr = t >> 3\n"),
        "add_then_shr": "input stream x\ninput stream y\noutput stream r\nstream t = x + y\nr = t >> 2\n",
        "shl_then_shr": "input stream x\noutput stream r\nstream t = x << 5\nr = t >> 7\n",
        "ones_copy_and_popcount": ("input stream x\noutput stream r\noutput int c\nstream o = ONES\n"
                                   "r = o & x\nc = popcount(r)\n"),
        "neg_popcount_raises": "output int c\nstream o = ONES\nc = popcount(o)\n",
        "ones_copy_xor_shr": ("input stream x\noutput stream r\nstream o = ONES\n"
                              "stream t = o ^ x\nr = t >> 9\n"),
        "while_on_negative_bounded": ("output int c\nstream o = ONES\nstream z = o ^ ONES\n"
                                      "int n = 0\nwhile (z) {\n z = z >> 1\n n = n + 1\n}\nc = n\n"),
        "tail_and_masks": ("input stream x\noutput stream r\nstream o = ONES\nstream t = o ^ x\n"
                           "stream u = t & x\nr = u >> 4\n"),
    }
    for nbits in (1, 5, 63, 64, 65, 100, 130):
        for name, src in progs.items():
            x = rng.getrandbits(nbits)
            y = rng.getrandbits(nbits)
            recs.append(case_record(ref, f"{name}_n{nbits}", src, nbits, {"x": x, "y": y}))
    # broadcast arrays: elements are 0 / -1 (benchmark/bsdata.py:89-102)
    src = ("input stream m[4]\ninput stream x\noutput stream r\noutput stream s\n"
           "stream t = m[1] ^ x\nr = t >> 2\ns = m[2] & x\n")
    for nbits in (10, 64, 70):
        x = rng.getrandbits(nbits)
        recs.append(case_record(ref, f"broadcast_n{nbits}", src, nbits, {"x": x}, {},
                                {"m": {0: 0, 1: -1, 2: -1, 3: 0}}))
    return recs


def reference_tree():
    v = os.environ.get("BSZ_REFERENCE_TREE")
    if v:
        return v
    oracle_dir = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle")
    return subprocess.run(["make", "-s", "-C", oracle_dir, "print-ref"], capture_output=True, text=True,
                          check=True).stdout.strip()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    args = ap.parse_args()
    ref = Ref(args.ref or reference_tree())
    groups = {"random_programs": gen_random(ref), "kat_ops": gen_kats(ref),
              "tail_corners": gen_tail_corners(ref)}
    try:
        from configs_small import gen_configs  # type: ignore
        groups["configs_small"] = gen_configs(case_record, ref)
    except ImportError:
        pass
    for name, recs in groups.items():
        path = os.path.join(HERE, f"{name}.json")
        with open(path, "w") as f:
            json.dump({"generator": "tests/golden/make_golden.py",
                       "reference": "simulator/pythonsim/interpreter.py", "cases": recs},
                      f, separators=(",", ":"))
        n_err = sum(1 for r in recs if "error" in r)
        n_dis = sum(1 for r in recs if r.get("bsim_agrees") is False)
        print(f"{name}: {len(recs)} cases ({n_err} reference errors, "
              f"{n_dis} where bsim disagrees), {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
