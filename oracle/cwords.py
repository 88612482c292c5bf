"""ctypes wrapper for oracle/wordops.c (liboracle.so).

TEST INFRASTRUCTURE ONLY (see wordops.c).  Streams are numpy uint64 arrays
of n = ceil(N/64) words.  ``run_ops`` evaluates a straight-line op list with
the word-level C oracle; ``program_to_ops`` lowers a parsed straight-line
program (from oracle/pyoracle.py) to that op list, tracking the tail bits
statically exactly as the Python semantics define them.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OP = {"copy": 0, "~": 1, "&": 2, "|": 3, "^": 4, "+": 5, "<<": 6, ">>": 7,
      "pop": 8, "zero": 9, "ones_op": 10, "ones_all": 11}


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(path)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        i64 = ctypes.c_int64
        L.o_and.argtypes = L.o_or.argtypes = L.o_xor.argtypes = [u64p, u64p, u64p, i64]
        L.o_not.argtypes = [u64p, u64p, i64, i64]
        L.o_add.argtypes = [u64p, u64p, u64p, i64, i64]
        L.o_shl.argtypes = [u64p, u64p, i64, i64, i64]
        L.o_shr.argtypes = [u64p, u64p, i64, i64, ctypes.c_int]
        L.o_popcount.argtypes = [u64p, i64]
        L.o_popcount.restype = i64
        L.o_run_ops.argtypes = [ctypes.POINTER(i64), i64, ctypes.POINTER(u64p), i64, i64,
                                ctypes.POINTER(i64)]
        L.o_run_ops.restype = ctypes.c_int
        L.o_num_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def n_words(nbits: int) -> int:
    return max(1, (nbits + 63) // 64)


def int_to_words(v: int, nbits: int) -> np.ndarray:
    n = n_words(nbits)
    v &= (1 << (64 * n)) - 1
    return np.frombuffer(v.to_bytes(8 * n, "little"), dtype=np.uint64).copy()


def words_to_int(w: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(w, dtype=np.uint64).tobytes(), "little")


def add(a, b, nbits):
    d = np.empty_like(a)
    lib().o_add(_p(d), _p(a), _p(b), a.size, nbits)
    return d


def shl(a, k, nbits):
    d = np.empty_like(a)
    lib().o_shl(_p(d), _p(a), k, a.size, nbits)
    return d


def popcount(a) -> int:
    return int(lib().o_popcount(_p(a), a.size))


def program_to_ops(prog):
    """Lower a straight-line program (no if/while/for/arrays) to op tuples.

    Returns (ops, reg_of_input, out_regs, pop_names, n_regs, tails) where ops
    are (code, dst, a, b, imm) rows for ``o_run_ops``.
    """
    regs: dict[str, int] = {}
    tails: dict[int, int] = {}
    ops = []
    nxt = [0]

    def new_reg():
        r = nxt[0]
        nxt[0] += 1
        return r

    for name in prog["inputs"]:
        regs[name] = new_reg()
        tails[regs[name]] = 0
    pops = []

    def opnd(e):
        if e[0] == "var":
            return regs[e[1]]
        if e[0] == "const":
            r = new_reg()
            ops.append((OP["zero"] if e[1] == "ZERO" else OP["ones_op"], r, -1, -1, 0))
            tails[r] = 0
            return r
        raise ValueError("straight-line lowering supports scalar streams only")

    def lower_rhs(e):
        k = e[0]
        d = new_reg()
        if k == "var":
            ops.append((OP["copy"], d, regs[e[1]], -1, 0)); tails[d] = tails[regs[e[1]]]
        elif k == "const":
            if e[1] == "ZERO":
                ops.append((OP["zero"], d, -1, -1, 0)); tails[d] = 0
            else:
                ops.append((OP["ones_all"], d, -1, -1, 0)); tails[d] = 1
        elif k == "not":
            ops.append((OP["~"], d, opnd(e[1]), -1, 0)); tails[d] = 0
        elif k == "bin":
            a, b = opnd(e[2]), opnd(e[3])
            ops.append((OP[e[1]], d, a, b, 0))
            ta, tb = tails[a], tails[b]
            tails[d] = {"&": ta & tb, "|": ta | tb, "^": ta ^ tb, "+": 0}[e[1]]
        elif k == "shift":
            a = opnd(e[2])
            amt = e[3]
            if amt[0] != "lit":
                raise ValueError("shift amount must be a literal here")
            if e[1] == "<<":
                ops.append((OP["<<"], d, a, -1, amt[1])); tails[d] = 0
            else:
                ops.append((OP[">>"], d, a, tails[a], amt[1])); tails[d] = tails[a]
        else:
            raise ValueError(k)
        return d

    for s in prog["stmts"]:
        k = s[0]
        if k == "local":
            if s[2] is None:
                d = new_reg(); ops.append((OP["zero"], d, -1, -1, 0)); tails[d] = 0
                regs[s[1]] = d
            else:
                regs[s[1]] = lower_rhs(s[2])
        elif k == "assign":
            regs[s[1]] = lower_rhs(s[2])
        elif k in ("idecl", "iassign"):
            e = s[2]
            if e[0] == "lit":
                continue
            if e[0] != "pop":
                raise ValueError("only popcount int expressions are supported here")
            src = regs[e[1][1]]
            ops.append((OP["pop"], src, src, -1, len(pops)))
            pops.append(s[1])
        else:
            raise ValueError(f"statement {k} not straight-line")
    outs = {n: regs[n] for n in prog["outputs"] if n in regs}
    return ops, {n: regs[n] for n in prog["inputs"]}, outs, pops, nxt[0], tails


def compact_registers(ops, in_regs, out_regs, nregs):
    """Drops the ops no output or popcount depends on and renumbers the
    registers (written once each) so that a register's buffer is reused after
    its last read: the register file then holds the peak number of live
    values instead of one buffer per op.  A destination never shares a buffer
    with an operand of its own op.
    Returns (ops, in_regs, out_regs, n_physical)."""
    def reads(o):
        code, d, a, b, _ = o
        r = [a] if a >= 0 else []
        if b >= 0 and code != OP[">>"]:
            r.append(b)
        return r

    # drop ops whose value reaches no output and no popcount
    needed = set(out_regs.values())
    keep = [False] * len(ops)
    for j in range(len(ops) - 1, -1, -1):
        o = ops[j]
        if o[0] == OP["pop"] or o[1] in needed:
            keep[j] = True
            needed.update(reads(o))
    ops = [o for o, k in zip(ops, keep) if k]
    last = {}
    for j, o in enumerate(ops):
        for r in reads(o):
            last[r] = j
    # outputs live to the end; inputs are the caller's arrays (never reused)
    pinned = set(out_regs.values()) | set(in_regs.values())
    phys = {}
    free = []
    nphys = 0

    def alloc():
        nonlocal nphys
        if free:
            return free.pop()
        nphys += 1
        return nphys - 1

    for r in in_regs.values():
        phys[r] = alloc()
    out_ops = []
    for j, o in enumerate(ops):
        code, d, a, b, imm = o
        pa = phys[a] if a >= 0 else -1
        pb = phys[b] if (b >= 0 and code != OP[">>"]) else b
        if code == OP["pop"]:
            out_ops.append((code, pa, pa, -1, imm))
        else:
            phys[d] = alloc()
            out_ops.append((code, phys[d], pa, pb, imm))
        for r in set(reads(o)):
            if last.get(r) == j and r not in pinned:
                free.append(phys[r])
        if code != OP["pop"] and d not in last and d not in pinned:
            free.append(phys[d])   # never read: its buffer is free right away
    return (out_ops, {k: phys[r] for k, r in in_regs.items()}, {k: phys[r] for k, r in out_regs.items()},
            max(1, nphys))


def run_straight_line(prog, nbits, inputs: dict, reuse_inputs=False):
    """Evaluate a straight-line program with the C oracle.

    ``inputs`` maps names to numpy uint64 arrays (n words each).
    Returns (outputs dict name->array, popcounts dict name->int).
    Registers are reused after their last read, so the memory held is the
    peak number of live values times the stream size.
    """
    ops, in_regs, out_regs, pops, nregs, _ = program_to_ops(prog)
    ops, in_regs, out_regs, nregs = compact_registers(ops, in_regs, out_regs, nregs)
    n = n_words(nbits)
    bufs = [None] * nregs
    for name, r in in_regs.items():
        # inputs are never written (every op writes a fresh register)
        bufs[r] = np.ascontiguousarray(inputs[name], dtype=np.uint64)
    for r in range(nregs):
        if bufs[r] is None:
            bufs[r] = np.empty(n, dtype=np.uint64)
    arr = (ctypes.POINTER(ctypes.c_uint64) * nregs)(*[_p(b) for b in bufs])
    flat = np.array(ops, dtype=np.int64).reshape(-1) if ops else np.zeros(5, np.int64)
    popv = np.zeros(max(1, len(pops)), dtype=np.int64)
    rc = lib().o_run_ops(flat.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(ops), arr, n,
                         nbits, popv.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    if rc != 0:
        raise RuntimeError("oracle op list rejected")
    return ({k: bufs[r] for k, r in out_regs.items()},
            {name: int(popv[i]) for i, name in enumerate(pops)})
