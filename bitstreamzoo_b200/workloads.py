"""Seeded synthetic workloads with the benchmark's named shapes.

There is no dataset to download: every workload is generated from a seed,
with the shapes and value distributions of the benchmark configurations.

* ``matchstar``    -- result = (((M & C) + C) ^ C) | M and its popcount;
                      M ~ Bernoulli(1/64), C ~ Bernoulli(0.75); 2^24 bits.
* ``long_streams`` -- A + B, A << k for k in {1, 63, 64, 1000}, A ^ B,
                      A & ~B and the popcount of each on two 2^32-bit
                      streams; A ~ Bernoulli(1/2), B all ones except zeros
                      with probability 2^-20 (carry runs span ~16K words).
* ``regex_dag``    -- a seeded random DAG of generator ops (55% AND/OR/
                      XOR/ANDNOT, 20% shift-by-1, 10% ADD, 10% MatchStar,
                      5% NOT) over 8 basis-bit streams transposed from random
                      bytes (70% a-z, 15% 0-9, 10% ASCII punctuation, 5%
                      uniform 0-255); 4 output streams + their popcounts.

Bernoulli(p) streams with tiny p are drawn exactly by sampling the number of
set bits from Binomial(N, p) and their positions uniformly without
replacement, which has the same distribution as independent bits.
"""

from __future__ import annotations

import numpy as np

# ----------------------------------------------------------------- helpers --


def n_words(nbits: int) -> int:
    return max(1, (nbits + 63) // 64)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def random_words(rng, nbits: int) -> np.ndarray:
    w = rng.integers(0, 2**64, size=n_words(nbits), dtype=np.uint64)
    _mask_tail(w, nbits)
    return w


def _mask_tail(w: np.ndarray, nbits: int):
    r = nbits % 64
    if r:
        w[-1] &= np.uint64((1 << r) - 1)


def sparse_bits(rng, nbits: int, p: float) -> np.ndarray:
    """Bernoulli(p) stream for small p: Binomial count + uniform positions."""
    w = np.zeros(n_words(nbits), dtype=np.uint64)
    k = int(rng.binomial(nbits, p))
    pos = np.unique(rng.integers(0, nbits, size=k, dtype=np.int64))
    while pos.size < k:   # top up duplicates so exactly k distinct bits are set
        extra = rng.integers(0, nbits, size=k - pos.size, dtype=np.int64)
        pos = np.unique(np.concatenate([pos, extra]))
    np.bitwise_or.at(w, pos >> 6, np.left_shift(np.uint64(1), (pos & 63).astype(np.uint64)))
    return w


def bernoulli_words(rng, nbits: int, p_num: int, p_log2: int) -> np.ndarray:
    """Bernoulli(p_num / 2^p_log2) via comparing random integers (exact)."""
    nw = n_words(nbits)
    out = np.zeros(nw, dtype=np.uint64)
    # draw per-bit uniform integers in [0, 2^p_log2) in chunks of words
    chunk = 1 << 16
    for s in range(0, nw, chunk):
        e = min(nw, s + chunk)
        u = rng.integers(0, 1 << p_log2, size=((e - s), 64), dtype=np.uint32 if p_log2 <= 32 else np.uint64)
        bits = (u < p_num).astype(np.uint64)
        out[s:e] = (bits << np.arange(64, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    _mask_tail(out, nbits)
    return out


# --------------------------------------------------------------- matchstar --

MATCHSTAR_SRC = """\
input stream M
input stream C
output stream r
output int n
stream t0 = M & C
stream t1 = t0 + C
stream t2 = t1 ^ C
r = t2 | M
n = popcount(r)
"""


def matchstar_inputs(nbits: int = 1 << 24, seed: int = 20261203) -> dict:
    rng = _rng(seed)
    # M ~ Bernoulli(1/64): AND of 6 uniform words; C ~ Bernoulli(3/4): OR of 2
    m = random_words(rng, nbits)
    for _ in range(5):
        m &= random_words(rng, nbits)
    c = random_words(rng, nbits) | random_words(rng, nbits)
    _mask_tail(c, nbits)
    return {"M": m, "C": c}


# ------------------------------------------------------------ long streams --

LONG_SHIFTS = (1, 63, 64, 1000)


def long_streams_src() -> str:
    lines = ["input stream A", "input stream B", "output stream s"]
    lines += [f"output stream l{k}" for k in LONG_SHIFTS]
    lines += ["output stream x", "output stream an", "output int ps"]
    lines += [f"output int pl{k}" for k in LONG_SHIFTS]
    lines += ["output int px", "output int pan", "s = A + B"]
    lines += [f"l{k} = A << {k}" for k in LONG_SHIFTS]
    lines += ["x = A ^ B", "stream nb = ~B", "an = A & nb", "ps = popcount(s)"]
    lines += [f"pl{k} = popcount(l{k})" for k in LONG_SHIFTS]
    lines += ["px = popcount(x)", "pan = popcount(an)"]
    return "\n".join(lines) + "\n"


LONG_OUTPUT_STREAMS = ["s"] + [f"l{k}" for k in LONG_SHIFTS] + ["x", "an"]
LONG_OUTPUT_INTS = ["ps"] + [f"pl{k}" for k in LONG_SHIFTS] + ["px", "pan"]


def long_streams_inputs(nbits: int = 1 << 32, seed: int = 20261204) -> dict:
    rng = _rng(seed)
    a = random_words(rng, nbits)
    b = ~sparse_bits(rng, nbits, 2.0 ** -20)
    _mask_tail(b, nbits)
    return {"A": a, "B": b}


# --------------------------------------------------------------- regex DAG --

_PUNCT = np.frombuffer(b"!\"#$%&'()*+,-./:;<=>?@[\\]^_`{|}~", dtype=np.uint8)


def regex_bytes(n_bytes: int, seed: int = 20261205) -> np.ndarray:
    rng = _rng(seed)
    cat = rng.integers(0, 100, size=n_bytes, dtype=np.uint8)
    out = np.empty(n_bytes, dtype=np.uint8)
    lower = cat < 70
    digit = (cat >= 70) & (cat < 85)
    punct = (cat >= 85) & (cat < 95)
    other = cat >= 95
    out[lower] = 97 + rng.integers(0, 26, size=int(lower.sum()), dtype=np.uint8)
    out[digit] = 48 + rng.integers(0, 10, size=int(digit.sum()), dtype=np.uint8)
    out[punct] = _PUNCT[rng.integers(0, _PUNCT.size, size=int(punct.sum()))]
    out[other] = rng.integers(0, 256, size=int(other.sum()), dtype=np.uint16).astype(np.uint8)
    return out


def basis_bits(data: np.ndarray) -> list[np.ndarray]:
    """Byte stream -> 8 basis bit streams: stream i bit j = (data[j] >> i) & 1
    (the layout of benchmark/apps/regex/src/run.py:164-187)."""
    n = data.size
    streams = []
    for i in range(8):
        bits = ((data >> i) & 1).astype(np.uint8)
        packed = np.packbits(bits, bitorder="little")
        pad = (-packed.size) % 8
        if pad:
            packed = np.concatenate([packed, np.zeros(pad, dtype=np.uint8)])
        streams.append(packed.view(np.uint64)[: n_words(n)].copy())
    return streams


def regex_dag_src(n_ops: int = 2000, seed: int = 20261206, n_outputs: int = 4) -> str:
    """Seeded random regex-shaped DAG.

    Operand rule: every operand is drawn uniformly from all values defined so
    far (the 8 basis streams and every earlier op result).  Outputs are the
    last ``n_outputs`` values.  Op classes: 13.75% each AND/OR/XOR/ANDNOT,
    20% Advance (<< 1), 10% ADD, 10% MatchStar (4 DSL ops), 5% NOT.
    """
    rng = _rng(seed)
    vals = [f"b{i}" for i in range(8)]
    lines = [f"input stream b{i}" for i in range(8)]
    lines += [f"output stream o{j}" for j in range(n_outputs)]
    lines += [f"output int p{j}" for j in range(n_outputs)]
    body = []
    tmp = [0]

    def t():
        tmp[0] += 1
        return f"v{tmp[0]}"

    def pick():
        return vals[int(rng.integers(0, len(vals)))]

    for _ in range(n_ops):
        u = float(rng.random())
        if u < 0.55:
            kind = int(rng.integers(0, 4))
            a, b = pick(), pick()
            d = t()
            if kind == 3:
                nb = t()
                body.append(f"stream {nb} = ~{b}")
                body.append(f"stream {d} = {a} & {nb}")
            else:
                body.append(f"stream {d} = {a} {'&|^'[kind]} {b}")
        elif u < 0.75:
            d = t()
            body.append(f"stream {d} = {pick()} << 1")
        elif u < 0.85:
            d = t()
            body.append(f"stream {d} = {pick()} + {pick()}")
        elif u < 0.95:
            m, c = pick(), pick()
            x1, x2, x3, d = t(), t(), t(), t()
            body += [f"stream {x1} = {m} & {c}", f"stream {x2} = {x1} + {c}",
                     f"stream {x3} = {x2} ^ {c}", f"stream {d} = {x3} | {m}"]
        else:
            d = t()
            body.append(f"stream {d} = ~{pick()}")
        vals.append(d)
    for j in range(n_outputs):
        body.append(f"o{j} = {vals[-1 - j]}")
        body.append(f"p{j} = popcount(o{j})")
    return "\n".join(lines + body) + "\n"


def batched_plan(n_instances: int = 4096, n_dags: int = 16, lo_log2: int = 12, hi_log2: int = 26,
                 ops: int = 300, seed: int = 20261207):
    """Batched uneven instances: ``n_dags`` seeded regex-shaped DAGs of ``ops``
    generator ops (the regex_dag mix, 8 basis inputs, 4 outputs + popcounts)
    and ``n_instances`` stream lengths drawn log-uniformly from
    [2^lo_log2, 2^hi_log2] bits; instance i runs DAG i mod n_dags.
    Returns (list of program sources, list of (dag, bits))."""
    rng = _rng(seed)
    srcs = [regex_dag_src(n_ops=ops, seed=seed + 1 + k) for k in range(n_dags)]
    logs = rng.uniform(lo_log2, hi_log2, size=n_instances)
    bits = np.maximum(1, np.floor(np.exp2(logs))).astype(np.int64)
    return srcs, [(i % n_dags, int(bits[i])) for i in range(n_instances)]


def shaped_dag_src(n_ops: int, seed: int, window: int = 0, p_bit: float = 0.55, p_shl: float = 0.2,
                   p_add: float = 0.1, p_shr: float = 0.0, max_shift: int = 1, n_inputs: int = 8,
                   n_outputs: int = 4) -> str:
    """Seeded DAG with a chosen shape, for schedule tuning.

    Operands come from the last ``window`` values (0 = all values so far, as
    in :func:`regex_dag_src`): a small window gives deep chains with few live
    temporaries, a large one wide DAGs.  Op classes are drawn with the given
    probabilities (the rest are NOTs); shift distances are uniform in
    [1, max_shift].  Outputs are the last ``n_outputs`` values and their
    popcounts."""
    rng = _rng(seed)
    vals = [f"b{i}" for i in range(n_inputs)]
    lines = [f"input stream b{i}" for i in range(n_inputs)]
    lines += [f"output stream o{j}" for j in range(n_outputs)]
    lines += [f"output int p{j}" for j in range(n_outputs)]
    body = []
    for i in range(n_ops):
        lo = 0 if window <= 0 else max(0, len(vals) - window)

        def pick():
            return vals[int(rng.integers(lo, len(vals)))]

        d = f"v{i}"
        u = float(rng.random())
        if u < p_bit:
            body.append(f"stream {d} = {pick()} {'&|^'[int(rng.integers(0, 3))]} {pick()}")
        elif u < p_bit + p_shl:
            body.append(f"stream {d} = {pick()} << {int(rng.integers(1, max_shift + 1))}")
        elif u < p_bit + p_shl + p_add:
            body.append(f"stream {d} = {pick()} + {pick()}")
        elif u < p_bit + p_shl + p_add + p_shr:
            body.append(f"stream {d} = {pick()} >> {int(rng.integers(1, max_shift + 1))}")
        else:
            body.append(f"stream {d} = ~{pick()}")
        vals.append(d)
    for j in range(n_outputs):
        body.append(f"o{j} = {vals[-1 - j]}")
        body.append(f"p{j} = popcount(o{j})")
    return "\n".join(lines + body) + "\n"


def regex_dag_inputs(nbits: int = 1 << 29, seed: int = 20261205) -> dict:
    streams = basis_bits(regex_bytes(nbits, seed))
    return {f"b{i}": s for i, s in enumerate(streams)}
