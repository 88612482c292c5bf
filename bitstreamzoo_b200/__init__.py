"""B200-native executor for the BitstreamZoo bitstream DSL.

The hot path is native: a C++ host (parser, op-DAG lowering, device runtime)
and hand-written sm_100a CUDA kernels in ``libbsz.so``; this package is a
thin Python layer over its C ABI (include/bsz.h):

* ``Context``      -- one CUDA device + stream; compile / run programs.
* ``B200Backend``  -- the reference harness's backend interface
  (``run`` / ``run_batch`` of benchmark/base.py:CudaBackend, lines 181-254),
  executed in-process instead of through a subprocess.
* ``bsim_cuda_path()`` -- the drop-in executable for
  ``benchmark/run_all.py --backend cuda``.

Values are Python ints (bit i = stream position i, negative = infinitely
many ones, as in the reference interpreter) or numpy uint64 word arrays.
"""

from __future__ import annotations

import ctypes
import json

import numpy as np

from . import _lib
from ._lib import BszError, Stats

MODE_PLAIN = 0
MODE_FUSED = 1
MODE_AUTO = 2
MODE_VM = 3
MODES = {"plain": MODE_PLAIN, "fused": MODE_FUSED, "auto": MODE_AUTO, "vm": MODE_VM}

DEFAULT_SCHEDULE = {"warps": 4, "range_steps": 64, "ctas_per_sm": 0, "min_blocks": 4,
                    "prefetch": 1, "cut_adds": 0, "layout": 0, "chunk_words": 4,
                    "stages": 2, "unroll": 0, "shift_mul": 0}

__all__ = ["Context", "Program", "Run", "B200Backend", "BszError", "MODE_PLAIN", "MODE_FUSED",
           "MODE_AUTO", "MODE_VM",
           "int_to_words", "words_to_int", "bsim_cuda_path"]


def bsim_cuda_path() -> str:
    return _lib.EXE_PATH


def n_words(bitlength: int) -> int:
    return max(1, (bitlength + 63) // 64)


def int_to_words(v: int, nw: int) -> tuple[np.ndarray, int]:
    """Python int -> (nw little-endian uint64 words, tail bit)."""
    tail = 1 if v < 0 else 0
    v &= (1 << (64 * nw)) - 1
    return np.frombuffer(v.to_bytes(8 * nw, "little"), dtype=np.uint64).copy(), tail


def words_to_int(w: np.ndarray, tail: int = 0) -> int:
    v = int.from_bytes(np.ascontiguousarray(w, dtype=np.uint64).tobytes(), "little")
    if tail:
        v -= 1 << (64 * len(w))
    return v


class Context:
    """A CUDA device context (one stream, cached device buffers)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        self.h = self.lib.bsz_create(device)
        if not self.h:
            raise BszError(_lib.last_error())

    def close(self):
        if self.h:
            self.lib.bsz_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return self.lib.bsz_stream(self.h) or 0

    def sync(self):
        _lib.check(self.lib.bsz_sync(self.h))

    def profile(self, enable: bool = True):
        """Start (and reset) or stop per-kernel CUDA-event timing."""
        _lib.check(self.lib.bsz_profile(self.h, 1 if enable else 0))

    def profile_report(self) -> dict:
        js = self.lib.bsz_profile_report(self.h)
        if js is None:
            raise BszError(_lib.last_error())
        return json.loads(js.decode())

    def compile(self, source: str) -> "Program":
        return Program(self, source)

    def run(self, source, bitlength: int, inputs=None, params=None, input_arrays=None,
            broadcast=None, mode: int = MODE_PLAIN, schedule: dict | None = None):
        """Compile + run; returns a finished ``Run``.  ``schedule``: fused
        kernel knobs over DEFAULT_SCHEDULE (see ``Run.set_schedule``)."""
        prog = source if isinstance(source, Program) else self.compile(source)
        r = prog.run(bitlength, mode)
        if schedule:
            r.set_schedule(schedule)
        for k, v in (params or {}).items():
            r.set_param(k, v)
        for k, v in (inputs or {}).items():
            r.bind(k, v)
        for k, arr in (input_arrays or {}).items():
            for i, v in arr.items():
                r.bind(k, v, index=i)
        for k, bits in (broadcast or {}).items():
            r.bind_broadcast(k, bits)
        r.execute()
        return r

    def run_case_json(self, source: str, bsdata_path: str | None = None,
                      json_input: dict | None = None, warmup: bool = False,
                      mode="auto"):
        """bsim_cuda JSON for every case; ``mode`` is a name of ``MODES`` or
        a ``MODE_*`` value."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        flags = (1 if warmup else 0) | (m << 1)
        js = self.lib.bsz_run_case_json(
            self.h, source.encode(), bsdata_path.encode() if bsdata_path else None,
            json.dumps(json_input).encode() if json_input is not None else None, flags)
        if js is None:
            raise BszError(_lib.last_error())
        return json.loads(js.decode())

    # -- per-op data plane on device pointers (ints) --------------------------
    def op(self, name: str, *args):
        fn = getattr(self.lib, f"bsz_op_{name}")
        _lib.check(fn(self.h, *args))

    def popcount(self, a_ptr: int, nw: int) -> int:
        out = ctypes.c_uint64()
        _lib.check(self.lib.bsz_op_popcount(self.h, a_ptr, nw, ctypes.byref(out)))
        return out.value

    def s2p(self, bytes_ptr: int, n_bytes: int, basis_ptrs) -> None:
        """Device byte -> basis-bit transposition into eight device streams of
        ``ceil(n_bytes / 64)`` words (asynchronous on the context's stream)."""
        arr = (ctypes.c_void_p * 8)(*[int(p) for p in basis_ptrs])
        _lib.check(self.lib.bsz_s2p(self.h, bytes_ptr, int(n_bytes), arr))

    def is_nonzero(self, a_ptr: int, nw: int) -> bool:
        out = ctypes.c_int()
        _lib.check(self.lib.bsz_op_is_nonzero(self.h, a_ptr, nw, ctypes.byref(out)))
        return bool(out.value)


class Program:
    def __init__(self, ctx: Context, source: str):
        self.ctx = ctx
        self.source = source
        b = source.encode()
        self.h = ctx.lib.bsz_compile(ctx.h, b, len(b))
        if not self.h:
            raise BszError(_lib.last_error())

    def __del__(self):
        try:
            if self.h:
                self.ctx.lib.bsz_program_free(self.h)
                self.h = None
        except Exception:
            pass

    def static_ops(self, params: dict | None = None) -> int:
        params = params or {}
        names = (ctypes.c_char_p * max(1, len(params)))(*[k.encode() for k in params])
        vals = (ctypes.c_int64 * max(1, len(params)))(*params.values())
        return self.ctx.lib.bsz_static_ops(self.h, names, vals, len(params))

    def run(self, bitlength: int, mode: int = MODE_PLAIN) -> "Run":
        return Run(self, bitlength, mode)


class Run:
    def __init__(self, prog: Program, bitlength: int, mode: int):
        self.prog = prog
        self.lib = prog.ctx.lib
        self.bitlength = bitlength
        self.nw = n_words(bitlength)
        self.h = self.lib.bsz_run_create(prog.h, bitlength, mode)
        if not self.h:
            raise BszError(_lib.last_error())
        self.stats = None

    def __del__(self):
        try:
            if self.h:
                self.lib.bsz_run_free(self.h)
                self.h = None
        except Exception:
            pass

    def set_param(self, name: str, value: int):
        _lib.check(self.lib.bsz_set_param(self.h, name.encode(), int(value)))

    def set_schedule(self, schedule: dict):
        """Fused-kernel schedule: keys of ``DEFAULT_SCHEDULE`` (missing keys keep defaults)."""
        s = dict(DEFAULT_SCHEDULE)
        s.update(schedule or {})
        st = _lib.Schedule(**{k: int(s[k]) for k, _ in _lib.Schedule._fields_})
        _lib.check(self.lib.bsz_run_set_schedule(self.h, ctypes.byref(st)))

    def bind(self, name: str, value, index: int = -1, tail: int = 0):
        """Bind a Python int, a numpy uint64 array, or a device pointer:
        ``("device", ptr, n_words)`` copies it, ``("borrow", ptr, n_words)``
        uses it in place (it must outlive this run)."""
        if isinstance(value, tuple) and value and value[0] in ("device", "borrow"):
            kind, ptr, nw = value[:3]
            t = value[3] if len(value) > 3 else tail
            flag = 1 if kind == "device" else 2
            _lib.check(self.lib.bsz_bind_input(self.h, name.encode(), index, ptr, nw, t, flag))
            return
        if isinstance(value, np.ndarray):
            w = np.ascontiguousarray(value, dtype=np.uint64)
            t = tail
        else:
            w, t = int_to_words(int(value), self.nw)
        _lib.check(self.lib.bsz_bind_input(self.h, name.encode(), index, w.ctypes.data, w.size, t, 0))

    def bind_broadcast(self, name: str, ones):
        arr = (ctypes.c_uint8 * max(1, len(ones)))(*[1 if x else 0 for x in ones])
        _lib.check(self.lib.bsz_bind_broadcast(self.h, name.encode(), arr, len(ones)))

    def execute(self) -> dict:
        st = Stats()
        _lib.check(self.lib.bsz_execute(self.h, ctypes.byref(st)))
        self.stats = st.as_dict()
        return self.stats

    def launch(self):
        """Enqueue the run's device work and return without waiting
        (``bsz_execute_async``); :meth:`wait` (or reading any result)
        finishes it."""
        _lib.check(self.lib.bsz_execute_async(self.h))

    def wait(self) -> dict:
        st = Stats()
        _lib.check(self.lib.bsz_run_wait(self.h, ctypes.byref(st)))
        self.stats = st.as_dict()
        return self.stats

    def stream(self, name: str, index: int = -1) -> np.ndarray:
        out = np.empty(self.nw, dtype=np.uint64)
        _lib.check(self.lib.bsz_get_stream(self.h, name.encode(), index, out.ctypes.data, self.nw))
        return out

    def stream_int(self, name: str, index: int = -1) -> int:
        return words_to_int(self.stream(name, index))

    def stream_device_ptr(self, name: str, index: int = -1) -> int:
        p = ctypes.c_void_p()
        _lib.check(self.lib.bsz_get_stream_device(self.h, name.encode(), index, ctypes.byref(p)))
        return p.value

    def int(self, name: str) -> int:
        v = ctypes.c_int64()
        _lib.check(self.lib.bsz_get_int(self.h, name.encode(), ctypes.byref(v)))
        return v.value

    def array_indices(self, name: str) -> list[int] | None:
        n = self.lib.bsz_array_indices(self.h, name.encode(), None, 0)
        if n < 0:
            return None
        buf = (ctypes.c_int64 * max(1, n))()
        self.lib.bsz_array_indices(self.h, name.encode(), buf, n)
        return list(buf[:n])

    def has_stream(self, name: str) -> bool:
        out = np.empty(1, dtype=np.uint64)
        return self.lib.bsz_get_stream(self.h, name.encode(), -1, out.ctypes.data, 0) == 0


class Batch:
    """Many instances of several straight-line programs in one graph-captured launch.

    ``instances`` is a list of ``(program_index, bitlength, input_ptrs, output_ptrs)``
    with device pointers (ints) in the order of each program's declared scalar
    inputs / output streams (0 = do not store that output).
    """

    def __init__(self, ctx: Context, programs: list, instances: list, schedule: dict | None = None):
        self.ctx = ctx
        self.lib = ctx.lib
        self.programs = programs
        n = len(instances)
        self._keep = []
        arr = (_lib.Instance * max(1, n))()
        for i, (p, bits, ins, outs) in enumerate(instances):
            ia = (ctypes.c_void_p * max(1, len(ins)))(*ins)
            oa = (ctypes.c_void_p * max(1, len(outs)))(*[o or None for o in outs])
            self._keep += [ia, oa]
            arr[i].program = p
            arr[i].bitlength = bits
            arr[i].inputs = ctypes.cast(ia, ctypes.POINTER(ctypes.c_void_p))
            arr[i].outputs = ctypes.cast(oa, ctypes.POINTER(ctypes.c_void_p))
        s = dict(DEFAULT_SCHEDULE)
        s.update(schedule or {})
        st = _lib.Schedule(**{k: int(s[k]) for k, _ in _lib.Schedule._fields_})
        progs = (ctypes.c_void_p * len(programs))(*[p.h for p in programs])
        self.n = n
        self.h = self.lib.bsz_batch_create(ctx.h, progs, len(programs), arr, n, ctypes.byref(st))
        if not self.h:
            raise BszError(_lib.last_error())
        self.items = self.lib.bsz_batch_items(self.h)

    def launch(self):
        _lib.check(self.lib.bsz_batch_launch(self.h))

    def finish(self) -> dict:
        st = Stats()
        _lib.check(self.lib.bsz_batch_finish(self.h, ctypes.byref(st)))
        return st.as_dict()

    def ints(self, instance: int) -> list[int]:
        buf = (ctypes.c_int64 * 64)()
        n = self.lib.bsz_batch_ints(self.h, instance, buf, 64)
        if n < 0:
            raise BszError(_lib.last_error())
        return list(buf[:n])

    def __del__(self):
        try:
            if self.h:
                self.lib.bsz_batch_free(self.h)
                self.h = None
        except Exception:
            pass


def _source_of(prog) -> str:
    if isinstance(prog, str):
        return prog
    path = getattr(prog, "source_path", None)
    if path:
        with open(path) as f:
            return f.read()
    return prog.source


class B200Backend:
    """Mirror of the reference harness backend (benchmark/base.py:181-254).

    ``run`` returns (outputs, op_count, exec_ms) with stream outputs as Python
    ints and array outputs as {index: int}; ``run_batch`` returns the
    bsim_cuda JSON dicts, one per case.  ``prog`` is a reference
    ``ProgramInfo`` (anything with ``source_path``) or DSL source text.
    """

    def __init__(self, device: int = 0, mode="auto", ctx: Context | None = None):
        self.ctx = ctx or Context(device)
        self.mode = mode

    def run(self, prog, inputs, params=None, input_arrays=None, bitlength=0,
            iterations=1, feedback=None, bsdata_path=None):
        src = _source_of(prog)
        if bsdata_path:
            out = self.ctx.run_case_json(src, bsdata_path=bsdata_path, mode=self.mode)
        else:
            payload = {"inputs": {k: hex(v) for k, v in inputs.items()},
                       "params": params or {}, "n_vectors": bitlength}
            if input_arrays:
                payload["input_arrays"] = {
                    k: [hex(a.get(i, 0)) for i in range(max(a) + 1)] if a else []
                    for k, a in input_arrays.items()}
            if iterations > 1:
                payload["iterations"] = iterations
            if feedback:
                payload["feedback"] = feedback
            out = self.ctx.run_case_json(src, json_input=payload, mode=self.mode)
        return _parse_outputs(out["outputs"]), out["op_count"], out.get("exec_ms", 0.0)

    def run_batch(self, prog, bsdata_paths):
        src = _source_of(prog)
        results = []
        for p in bsdata_paths:
            out = self.ctx.run_case_json(src, bsdata_path=p, mode=self.mode)
            results.extend(out if isinstance(out, list) else [out])
        return results


def _parse_outputs(outputs: dict) -> dict:
    res = {}
    for k, v in outputs.items():
        if isinstance(v, str) and v.startswith("0x"):
            res[k] = int(v, 16)
        elif isinstance(v, dict):
            res[k] = {int(i): int(x, 16) if isinstance(x, str) else x for i, x in v.items()}
        else:
            res[k] = v
    return res
