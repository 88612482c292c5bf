"""CPU oracle: a restatement of the BitstreamZoo Python reference interpreter.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA executor
is compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it; the
product path (``bitstreamzoo_b200`` and its C ABI) never does.

Semantics follow the normative Python interpreter of the reference:

* tokenizer            -- simulator/pythonsim/lexer.py:74-143
* parser + 3-address   -- simulator/pythonsim/parser.py:156-596
* interpreter          -- simulator/pythonsim/interpreter.py:30-253

Streams are Python integers (bit i = position i, LSB first).  With a bitlength
N > 0, ``~``, ``+`` and ``<<`` are masked to N bits, ``& | ^ >>`` are not, the
constant ``ONES`` is the N-bit mask when used as an operand but ``-1``
("infinitely many ones") when copied into a variable, and ``popcount`` of a
negative value raises (interpreter.py:58-59, 70-79, 150-218).

Pinning: ``tests/test_oracle.py`` checks this module against golden vectors
that ``tests/golden/make_golden.py`` produced by running the reference
interpreter itself, and (where the reference tree is present) against the
reference interpreter on seeded random programs.
"""

from __future__ import annotations

import re

MAX_WHILE_ITERS = 10_000            # interpreter.py:20
COUNTED_OPS = ("~", "&", "|", "^", "<<", ">>", "+")   # interpreter.py:22-23


class OracleParseError(Exception):
    """Syntax error (parser.py:150 ParseError)."""


class OracleThreeAddrError(Exception):
    """3-address-form violation (parser.py:491 ThreeAddrError)."""


class OracleRuntimeError(Exception):
    """Run-time error (interpreter.py:26 RuntimeError_)."""


# ── Tokenizer (lexer.py:74-143) ───────────────────────────────────────────

_KEYWORDS = {"input", "output", "param", "stream", "int", "if", "while",
             "for", "in", "ZERO", "ONES", "popcount"}

# Priority order matters: ``..`` before ``<<``/``>>``, numbers before names.
_TOKEN_RE = re.compile(r"""
    (?P<skip>//[^\n]*|[ \t\r\n]+)
  | (?P<op>\.\.|<<|>>|[{}()\[\]=~&|^+\-*])
  | (?P<num>[0-9]+)
  | (?P<name>[a-zA-Z_][a-zA-Z0-9_]*)
""", re.VERBOSE)


def tokenize(src: str):
    """Return a list of (kind, text, line) with kind in {kw, name, num, op, eof}.

    Like the reference tokenizer (``re.finditer`` over the alternatives),
    characters that match no token are skipped silently.
    """
    toks = []
    line = 1
    for m in _TOKEN_RE.finditer(src):
        text = m.group()
        line += text.count("\n")
        if m.lastgroup == "skip":
            continue
        if m.lastgroup == "name":
            kind = "kw" if text in _KEYWORDS else "name"
        else:
            kind = m.lastgroup
        toks.append((kind, text, line))
    toks.append(("eof", "", line))
    return toks


# ── Parser (parser.py:156-438) ────────────────────────────────────────────
#
# AST as tuples:
#   stream expr: ("var", n) ("elem", n, iexpr) ("const", "ZERO"|"ONES")
#                ("not", e) ("bin", op, l, r) ("shift", op, e, iexpr)
#   int expr:    ("lit", v) ("ivar", n) ("ibin", op, l, r) ("pop", e)
#   statements:  ("local", n, e|None) ("adecl", n, iexpr) ("idecl", n, iexpr)
#                ("assign", n, e) ("aassign", n, iexpr, e) ("iassign", n, iexpr)
#                ("if", cond_e, body) ("while", cond_e, body)
#                ("for", var, lo, hi, body)

class _Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0
        self.int_names: set[str] = set()
        self.output_ints: list[str] = []

    # token helpers
    def peek(self):
        return self.t[self.i]

    def is_(self, *texts) -> bool:
        k, v, _ = self.t[self.i]
        return k in ("kw", "op") and v in texts

    def take(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def want(self, text: str):
        tok = self.take()
        if tok[0] not in ("kw", "op") or tok[1] != text:
            raise OracleParseError(f"line {tok[2]}: expected {text!r}, got {tok[1]!r}")
        return tok

    def want_name(self) -> str:
        tok = self.take()
        if tok[0] != "name":
            raise OracleParseError(f"line {tok[2]}: expected identifier, got {tok[1]!r}")
        return tok[1]

    # program (parser.py:180-226)
    def program(self):
        prog = {"stmts": [], "inputs": [], "outputs": [], "params": [],
                "output_ints": self.output_ints}
        stmts = prog["stmts"]
        while self.peek()[0] != "eof":
            if self.is_("input"):
                self.take(); self.want("stream")
                name = self.want_name()
                if self.is_("["):
                    self.take(); self.int_expr(); self.want("]")
                prog["inputs"].append(name)
            elif self.is_("output"):
                self.take()
                if self.is_("int"):
                    self.take()
                    name = self.want_name()
                    self.int_names.add(name)
                    self.output_ints.append(name)
                    stmts.append(("idecl", name, ("lit", 0)))
                else:
                    self.want("stream")
                    name = self.want_name()
                    if self.is_("["):
                        self.take(); self.int_expr(); self.want("]")
                    prog["outputs"].append(name)
            elif self.is_("param"):
                self.take(); self.want("int")
                name = self.want_name()
                self.int_names.add(name)
                prog["params"].append(name)
            else:
                stmts.append(self.statement(top=True))
        return prog

    def statement(self, top=False):
        if self.is_("stream"):
            self.take()
            name = self.want_name()
            if self.is_("["):
                self.take(); size = self.int_expr(); self.want("]")
                return ("adecl", name, size)
            init = None
            if self.is_("="):
                self.take(); init = self.stream_expr()
            return ("local", name, init)
        if self.is_("int"):
            self.take()
            name = self.want_name()
            self.int_names.add(name)
            self.want("=")
            return ("idecl", name, self.int_expr())
        if self.is_("if", "while"):
            kw = self.take()[1]
            self.want("(")
            cond = self.stream_expr()
            self.want(")")
            return (kw, cond, self.block())
        if self.is_("for"):
            self.take()
            var = self.want_name()
            self.int_names.add(var)
            self.want("in")
            lo = self.int_expr()
            self.want("..")
            hi = self.int_expr()
            return ("for", var, lo, hi, self.block())
        if self.peek()[0] == "name":
            name = self.take()[1]
            if self.is_("["):
                self.take(); idx = self.int_expr(); self.want("]")
                self.want("=")
                return ("aassign", name, idx, self.stream_expr())
            self.want("=")
            if name in self.int_names:
                return ("iassign", name, self.int_expr())
            return ("assign", name, self.stream_expr())
        k, v, line = self.peek()
        where = "unexpected token" if top else "unexpected token in block:"
        raise OracleParseError(f"line {line}: {where} {v!r}")

    def block(self):
        self.want("{")
        body = []
        while not self.is_("}"):
            if self.peek()[0] == "eof":
                raise OracleParseError(f"line {self.peek()[2]}: unexpected end of input in block")
            body.append(self.statement())
        self.want("}")
        return body

    # stream expressions, precedence (high→low): ~, << >>, &, +, ^, |
    # (parser.py:337-409)
    _LEVELS = (("|",), ("^",), ("+",), ("&",))

    def stream_expr(self, level=0):
        if level == len(self._LEVELS):
            return self.shift_expr()
        left = self.stream_expr(level + 1)
        while self.is_(*self._LEVELS[level]):
            op = self.take()[1]
            left = ("bin", op, left, self.stream_expr(level + 1))
        return left

    def shift_expr(self):
        left = self.unary_expr()
        while self.is_("<<", ">>"):
            op = self.take()[1]
            left = ("shift", op, left, self.int_expr())
        return left

    def unary_expr(self):
        if self.is_("~"):
            self.take()
            return ("not", self.unary_expr())
        return self.primary()

    def primary(self):
        if self.is_("ZERO", "ONES"):
            return ("const", self.take()[1])
        if self.is_("("):
            self.take()
            e = self.stream_expr()
            self.want(")")
            return e
        if self.peek()[0] == "name":
            name = self.take()[1]
            if self.is_("["):
                self.take(); idx = self.int_expr(); self.want("]")
                return ("elem", name, idx)
            return ("var", name)
        k, v, line = self.peek()
        raise OracleParseError(f"line {line}: expected stream expression, got {v!r}")

    # int expressions: * binds tighter than + - (parser.py:415-438)
    def int_expr(self):
        left = self.int_term()
        while self.is_("+", "-"):
            op = self.take()[1]
            left = ("ibin", op, left, self.int_term())
        return left

    def int_term(self):
        left = self.int_atom()
        while self.is_("*"):
            self.take()
            left = ("ibin", "*", left, self.int_atom())
        return left

    def int_atom(self):
        k, v, line = self.peek()
        if k == "num":
            self.take()
            return ("lit", int(v))
        if self.is_("("):
            self.take()
            e = self.int_expr()
            self.want(")")
            return e
        if self.is_("popcount"):
            self.take(); self.want("(")
            arg = self.stream_expr()
            self.want(")")
            return ("pop", arg)
        if k == "name":
            self.take()
            return ("ivar", v)
        raise OracleParseError(f"line {line}: expected integer expression, got {v!r}")


_PRIMARY = ("var", "elem", "const")


def _check_rhs(e, ctx):
    """3-address RHS rule (parser.py:501-531)."""
    kind = e[0]
    if kind in _PRIMARY:
        return
    if kind == "not":
        operands = (e[1],)
    elif kind == "bin":
        operands = (e[2], e[3])
    else:
        operands = (e[2],)
    for o in operands:
        if o[0] not in _PRIMARY:
            raise OracleThreeAddrError(f"{ctx}: operand must be a primary")


def _check_stmts(stmts, ctx):
    """3-address statement rules (parser.py:534-564)."""
    for s in stmts:
        k = s[0]
        if k == "local" and s[2] is not None:
            _check_rhs(s[2], ctx)
        elif k == "assign":
            _check_rhs(s[2], ctx)
        elif k == "aassign":
            _check_rhs(s[3], ctx)
        elif k in ("idecl", "iassign"):
            if s[2][0] == "pop" and s[2][1][0] != "var":
                raise OracleThreeAddrError(f"{ctx}: popcount arg must be a variable")
        elif k in ("if", "while"):
            if s[1][0] != "var":
                raise OracleThreeAddrError(f"{ctx}: {k} condition must be a variable")
            _check_stmts(s[2], ctx)
        elif k == "for":
            _check_stmts(s[4], ctx)


def parse(src: str):
    """Parse + validate (parser.py:588-596)."""
    prog = _Parser(tokenize(src)).program()
    _check_stmts(prog["stmts"], prog["inputs"][0] if prog["inputs"] else "<program>")
    return prog


# ── Interpreter (interpreter.py:30-253) ───────────────────────────────────

class Oracle:
    """Executes a parsed program on Python integers."""

    def __init__(self, bitlength: int = 0):
        self.N = bitlength
        self.mask = (1 << bitlength) - 1 if bitlength > 0 else 0
        self.env: dict = {}
        self.arrays: dict = {}
        self.ints: dict = {}
        self.op_count = 0
        self.op_mix: dict = {}

    def _tally(self, op):
        self.op_count += 1
        self.op_mix[op] = self.op_mix.get(op, 0) + 1

    def _masked(self, v):
        return v & self.mask if self.mask else v

    # int expressions (interpreter.py:45-68)
    def ival(self, e):
        k = e[0]
        if k == "lit":
            return e[1]
        if k == "ivar":
            if e[1] not in self.ints:
                raise OracleRuntimeError(f"undefined int variable: {e[1]}")
            return self.ints[e[1]]
        if k == "ibin":
            a, b = self.ival(e[2]), self.ival(e[3])
            return a + b if e[1] == "+" else a - b if e[1] == "-" else a * b
        # popcount: argument is a variable (3-address rule)
        v = self.env[e[1][1]]
        if v < 0:
            raise OracleRuntimeError("popcount on negative value (infinite bits set)")
        self._tally("popcount")
        return v.bit_count()

    # operand read (interpreter.py:70-84): ONES is the N-bit mask here
    def operand(self, e):
        k = e[0]
        if k == "var":
            return self.env[e[1]]
        if k == "const":
            if e[1] == "ZERO":
                return 0
            return self.mask if self.mask else -1
        idx = self.ival(e[2])
        if e[1] not in self.arrays:
            raise OracleRuntimeError(f"undefined array: {e[1]}")
        return self.arrays[e[1]].get(idx, 0)

    # right-hand side (interpreter.py:150-218)
    def rhs(self, e):
        k = e[0]
        if k == "var":
            return self.env[e[1]]
        if k == "const":                 # copy of ONES keeps infinite ones
            return 0 if e[1] == "ZERO" else -1
        if k == "elem":
            return self.operand(e)
        if k == "not":
            r = self._masked(~self.operand(e[1]))
            self._tally("~")
            return r
        if k == "bin":
            a, b = self.operand(e[2]), self.operand(e[3])
            op = e[1]
            if op == "&":
                r = a & b
            elif op == "|":
                r = a | b
            elif op == "^":
                r = a ^ b
            else:
                r = self._masked(a + b)
            self._tally(op)
            return r
        # shift
        v = self.operand(e[2])
        amt = self.ival(e[3])
        r = self._masked(v << amt) if e[1] == "<<" else v >> amt
        self._tally(e[1])
        return r

    def exec_block(self, stmts):
        for s in stmts:
            self.exec_stmt(s)

    def exec_stmt(self, s):
        k = s[0]
        if k == "local":
            self.env[s[1]] = 0 if s[2] is None else self.rhs(s[2])
        elif k == "adecl":
            self.arrays[s[1]] = {i: 0 for i in range(self.ival(s[2]))}
        elif k == "assign":
            self.env[s[1]] = self.rhs(s[2])
        elif k == "aassign":
            idx = self.ival(s[2])
            self.arrays.setdefault(s[1], {})
            self.arrays[s[1]][idx] = self.rhs(s[3])
        elif k == "if":
            if self.env[s[1][1]] != 0:
                self.exec_block(s[2])
        elif k == "while":
            for _ in range(MAX_WHILE_ITERS):
                if self.env[s[1][1]] == 0:
                    break
                self.exec_block(s[2])
            else:
                raise OracleRuntimeError(
                    f"while loop exceeded {MAX_WHILE_ITERS} iterations")
        elif k == "for":
            lo, hi = self.ival(s[2]), self.ival(s[3])
            for i in range(lo, hi):
                self.ints[s[1]] = i
                self.exec_block(s[4])
        elif k in ("idecl", "iassign"):
            self.ints[s[1]] = self.ival(s[2])
        else:  # pragma: no cover - parser never produces other kinds
            raise OracleRuntimeError(f"unknown statement {k}")

    def run(self, prog, inputs, params=None, input_arrays=None):
        """Load inputs, execute, collect outputs (interpreter.py:220-253)."""
        if params:
            self.ints.update(params)
        input_arrays = input_arrays or {}
        for name in prog["inputs"]:
            if name in inputs:
                self.env[name] = inputs[name]
            elif name in input_arrays:
                self.arrays[name] = dict(input_arrays[name])
            else:
                self.env[name] = 0
        self.exec_block(prog["stmts"])
        out = {}
        for name in prog["outputs"]:
            if name in self.env:
                out[name] = self.env[name]
            elif name in self.arrays:
                out[name] = dict(self.arrays[name])
        for name in prog["output_ints"]:
            if name in self.ints:
                out[name] = self.ints[name]
        return out


def run_source(src, bitlength, inputs, params=None, input_arrays=None):
    """Parse and run ``src``; returns (outputs, op_count, op_mix)."""
    prog = parse(src)
    o = Oracle(bitlength)
    out = o.run(prog, inputs, params, input_arrays)
    return out, o.op_count, o.op_mix


def count_static_ops(prog, params=None):
    """Static op count: for-loops multiply, if/while bodies count once.

    Restates ``OpCounter`` (simulator/csim/src/ast_liveness.cpp:629-727),
    which fills the ``static_ops`` field of the bsim_cuda JSON.
    """
    env = dict(params or {})

    def ival(e):
        k = e[0]
        if k == "lit":
            return e[1]
        if k == "ivar":
            return env.get(e[1], 0)
        if k == "ibin":
            a, b = ival(e[2]), ival(e[3])
            return a + b if e[1] == "+" else a - b if e[1] == "-" else a * b
        return 0

    def compute(e):
        return e is not None and e[0] not in _PRIMARY

    def count(stmts):
        total = 0
        for s in stmts:
            k = s[0]
            if k == "local":
                total += 1 if compute(s[2]) else 0
            elif k == "assign":
                total += 1 if compute(s[2]) else 0
            elif k == "aassign":
                total += 1 if compute(s[3]) else 0
            elif k in ("idecl", "iassign"):
                total += 1 if s[2][0] == "pop" else 0
            elif k == "for":
                lo, hi = ival(s[2]), ival(s[3])
                if hi > lo:
                    saved = dict(env)
                    env[s[1]] = lo
                    total += count(s[4]) * (hi - lo)
                    env.clear(); env.update(saved)
            elif k in ("if", "while"):
                total += count(s[2])
        return total

    return count(prog["stmts"])
