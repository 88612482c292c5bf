"""Seeded random DSL programs and inputs for parity tests.

Produces valid 3-address `.bs` programs that exercise every statement form
(stream/array/int declarations, all seven stream operators, ZERO/ONES as
operands and as copies, array element reads and writes, counted loops, `if`
and bounded `while`, popcount into int locals and int outputs) plus inputs of
a given bitlength.  Used by the golden-vector generator and by the tests.
"""

from __future__ import annotations

import random


def rand_stream(rng: random.Random, nbits: int, density: float | None = None) -> int:
    """A random non-negative stream of ``nbits`` bits."""
    if nbits <= 0:
        return 0
    if density is None:
        return rng.getrandbits(nbits)
    v = 0
    for i in range(nbits):
        if rng.random() < density:
            v |= 1 << i
    return v


def random_program(rng: random.Random, n_stmts: int = 30, allow_shr: bool = True,
                   allow_ctrl: bool = True, allow_ones_copy: bool = True,
                   n_inputs: int = 3, max_shift: int = 130) -> tuple[str, dict]:
    """Return (source, meta); meta lists inputs/arrays/params needed."""
    lines: list[str] = []
    inputs = [f"in{i}" for i in range(n_inputs)]
    for name in inputs:
        lines.append(f"input stream {name}")
    lines.append("input stream arr_in[4]")
    lines.append("param int K")
    lines.append("output stream out0")
    lines.append("output stream out1")
    lines.append("output stream outa[3]")
    lines.append("output int cnt")
    lines.append("stream tmp[4]")
    streams = list(inputs)          # names with tail 0 (safe for popcount)
    maybe_neg: set[str] = set()      # names that may hold negative values
    counter = [0]

    def fresh() -> str:
        counter[0] += 1
        return f"t{counter[0]}"

    def operand(safe: bool = False) -> str:
        r = rng.random()
        if r < 0.06 and not safe:
            return rng.choice(["ZERO", "ONES"])
        if r < 0.14:
            return f"arr_in[{rng.randrange(4)}]"
        if r < 0.20:
            return f"tmp[{rng.randrange(4)}]"
        pool = [s for s in streams if not (safe and s in maybe_neg)] or inputs
        return rng.choice(pool)

    def rhs() -> tuple[str, bool]:
        """Returns (expr, may_be_negative)."""
        r = rng.random()
        a = operand()
        neg_a = a in maybe_neg or a == "ONES"
        if r < 0.12:
            return f"~{a}", False
        if r < 0.55:
            op = rng.choice("&|^")
            b = operand()
            neg_b = b in maybe_neg or b == "ONES"
            return f"{a} {op} {b}", (neg_a or neg_b)
        if r < 0.67:
            return f"{a} + {operand()}", False
        if r < 0.82:
            k = rng.choice([0, 1, 2, 31, 63, 64, 65, 100, 127, 128, rng.randrange(max_shift)])
            if rng.random() < 0.2:
                return f"{a} << K", False
            return f"{a} << {k}", False
        if allow_shr and r < 0.92:
            k = rng.choice([0, 1, 5, 63, 64, 65, rng.randrange(max_shift)])
            return f"{a} >> {k}", neg_a
        if allow_ones_copy and r < 0.95:
            return "ONES", True
        return a, neg_a

    def emit_assign(indent: str):
        expr, neg = rhs()
        if rng.random() < 0.5 or not streams:
            name = fresh()
            lines.append(f"{indent}stream {name} = {expr}")
            streams.append(name)
        else:
            cand = [s for s in streams if s not in inputs]
            if not cand:
                name = fresh()
                lines.append(f"{indent}stream {name} = {expr}")
                streams.append(name)
            else:
                name = rng.choice(cand)
                lines.append(f"{indent}{name} = {expr}")
        if neg:
            maybe_neg.add(name)
        else:
            maybe_neg.discard(name)
        return name

    lines.append("int acc = 0")
    for _ in range(n_stmts):
        r = rng.random()
        if allow_ctrl and r < 0.08:
            # counted loop with array traffic
            lines.append("for i in 0..K {")
            lines.append(f"  stream lv = {operand()} << i")
            lines.append(f"  tmp[i] = lv ^ {operand()}")
            lines.append("}")
        elif allow_ctrl and r < 0.14:
            c = operand(safe=True)
            lines.append(f"if ({c if '[' not in c and c not in ('ZERO', 'ONES') else streams[0]}) {{")
            emit_assign("  ")
            lines.append("}")
        elif allow_ctrl and r < 0.18:
            base = rng.choice([s for s in streams if s not in maybe_neg] or inputs)
            w = fresh()
            lines.append(f"stream {w} = {base} & {rng.choice(inputs)}")
            streams.append(w)
            step = rng.choice([7, 19, 64, 200])
            lines.append(f"while ({w}) {{")
            lines.append(f"  {w} = {w} >> {step}")
            lines.append("  acc = acc + 1")
            lines.append("}")
        elif r < 0.26:
            s = rng.choice([x for x in streams if x not in maybe_neg] or inputs)
            lines.append(f"acc = acc + popcount({s}) * {rng.randrange(1, 4)} - {rng.randrange(3)}")
        else:
            emit_assign("")
    safe = [s for s in streams if s not in maybe_neg] or inputs
    lines.append(f"out0 = {rng.choice(streams)}")
    lines.append(f"out1 = {rng.choice(streams)} ^ {rng.choice(streams)}")
    for j in range(3):
        lines.append(f"outa[{j}] = {rng.choice(streams)}")
    lines.append(f"cnt = acc + popcount({rng.choice(safe)})")
    meta = {"inputs": inputs, "arrays": {"arr_in": 4}, "params": {"K": rng.randrange(0, 4)}}
    return "\n".join(lines) + "\n", meta


def random_case(rng: random.Random, nbits: int, **kw) -> dict:
    src, meta = random_program(rng, **kw)
    inputs = {n: rand_stream(rng, nbits) for n in meta["inputs"]}
    arrays = {"arr_in": {i: rand_stream(rng, nbits) for i in range(4)}}
    return {"src": src, "bitlength": nbits, "inputs": inputs,
            "input_arrays": arrays, "params": meta["params"]}
