"""Schedule autotuner and learned cost model for the fused backend.

The fused backend's generated kernels take a schedule (``bsz_schedule`` in
include/bsz.h): CTA size in warps, the launch-bounds minimum of resident
CTAs per SM (which caps registers per thread), an occupancy cap, the minimum
run of 32-word steps a warp owns, software prefetch of the next step's
loads, the kernel form (warp ranges, thread ranges in registers, thread
ranges through TMA boxes) with its chunk size and shift instructions, and
the carry scheme (speculative carry state inside the generated kernels, or
every addition by the plain look-back carry scan).  The best setting depends on
the DAG (op mix, shift distances, carry chains, live temporaries) and on the
stream length, so it is searched, not fixed:

* :data:`CANDIDATES` -- the search space.
* :func:`measure` -- device time of one (program, length, schedule): the sum
  of the executor's per-kernel CUDA events over one execution (fused
  kernels plus any exact re-runs), median over repetitions.
* :class:`Autotuner` -- exhaustive search, cached in a JSON file keyed by
  the program text and the length.
* :class:`CostModel` -- an MLP over DAG features (``bsz_program_features``),
  log2 length and the schedule encoding, predicting log(ms).  Its training
  and inference run on the GPU through libbsz's hand-written kernels
  (``bsz_mlp_*``: tiled FP32 GEMMs with fused bias/ReLU, MSE, column sums,
  Adam).  :meth:`CostModel.choose` picks a schedule with no measurement,
  or measures only the ``top_k`` best predictions.

The model is fitted on a random sample of the (program, length, schedule)
timings of training programs and evaluated on held-out programs by pick regret:
time of the picked schedule / time of the exhaustive best - 1.
"""

from __future__ import annotations

import ctypes
import hashlib
import itertools
import json
import math
import os

import numpy as np

from . import _lib
from . import DEFAULT_SCHEDULE, MODE_FUSED, BszError

# ------------------------------------------------------------ search space --

# Knobs that change the generated code (one NVRTC compile each) and knobs
# that only change the launch.
# A wider space (min_blocks 8, cut_adds 1: 48 candidates) was timed on 8
# held-out DAGs x 3 lengths and never held the fastest schedule, while those
# choices are the ones that are catastrophically slow elsewhere (up to 25x),
# so the searched space leaves them out.
CODEGEN_AXES = {"warps": (4, 8), "min_blocks": (2, 4), "prefetch": (0, 1), "cut_adds": (0,)}
LAUNCH_AXES = {"ctas_per_sm": (0, 2)}
# The thread-sequential form (layout 1): its register-resident chunk needs
# the full register file (min_blocks 1; at min_blocks 2 the 2,000-op regex
# DAG spills and runs 2x slower), and prefetch / range_steps do not apply.
# Its axes: CTA size (2 to 16 warps: 16 warps cap registers at 128 per
# thread) and 4- or 8-word register chunks.  Shifts as integer multiply-adds
# (shift_mul) measured slower on the regex DAG (0.228 vs 0.211 ms) and on
# batches, so the space keeps the funnel shifts.
SEQ_AXES = {"layout": (1,), "warps": (2, 4, 8, 16), "min_blocks": (1,), "prefetch": (0,), "cut_adds": (0,),
            "ctas_per_sm": (0,), "chunk_words": (4, 8)}
# The TMA form (layout 2): 4-word rows for 8 warps per CTA (2 or 3 stages)
# and for 4 warps (two CTAs per SM; 2 or 3 stages); 8-word rows leave room
# for only 4 warps per SM and measured 1.7x slower on the regex DAG, so they
# are out.
TMA_CANDIDATES = [{"layout": 2, "chunk_words": 4, "warps": 8, "min_blocks": 1, "prefetch": 0, "stages": 2},
                  {"layout": 2, "chunk_words": 4, "warps": 8, "min_blocks": 1, "prefetch": 0, "stages": 3},
                  {"layout": 2, "chunk_words": 4, "warps": 4, "min_blocks": 1, "prefetch": 0, "stages": 2},
                  {"layout": 2, "chunk_words": 4, "warps": 4, "min_blocks": 1, "prefetch": 0, "stages": 3}]
# The carry-scheme axis: every addition run by the plain single-pass
# carry scan (decoupled look-back) on materialized operands, the rest of
# the DAG in generated kernels of each form (cut_adds 2), against the
# speculative carry state of every other candidate.
CARRY_CANDIDATES = [{"layout": 0, "warps": 4, "min_blocks": 4, "prefetch": 1, "cut_adds": 2},
                    {"layout": 1, "warps": 8, "min_blocks": 1, "prefetch": 0, "cut_adds": 2},
                    {"layout": 1, "warps": 4, "min_blocks": 1, "prefetch": 0, "chunk_words": 8, "cut_adds": 2},
                    {"layout": 2, "chunk_words": 4, "warps": 8, "min_blocks": 1, "prefetch": 0, "stages": 2,
                     "cut_adds": 2}]


def candidate_space(codegen=None, launch=None, seq=None) -> list[dict]:
    """Cartesian product of the axes, each a full schedule dict: the warp
    form's codegen x launch axes, then the thread-sequential form's axes,
    the TMA form's candidates and the look-back carry scheme's (``seq``;
    pass an empty dict to leave all but the warp form out)."""
    codegen = codegen or CODEGEN_AXES
    launch = launch or LAUNCH_AXES
    seq = SEQ_AXES if seq is None else seq
    keys = list(codegen) + list(launch)
    out = []
    for vals in itertools.product(*[codegen[k] for k in codegen], *[launch[k] for k in launch]):
        s = dict(DEFAULT_SCHEDULE)
        s.update(dict(zip(keys, vals)))
        out.append(s)
    if seq:
        for vals in itertools.product(*[seq[k] for k in seq]):
            s = dict(DEFAULT_SCHEDULE)
            s.update(dict(zip(list(seq), vals)))
            out.append(s)
        for t in TMA_CANDIDATES + CARRY_CANDIDATES:
            s = dict(DEFAULT_SCHEDULE)
            s.update(t)
            out.append(s)
    return out


CANDIDATES = candidate_space()


def schedule_key(s: dict) -> tuple:
    return tuple(int(s[k]) for k, _ in _lib.Schedule._fields_)


def encode_schedule(s: dict) -> list[float]:
    """Schedule features (13): log2 warps, log2 min_blocks, occupancy cap
    (0 = none), log2 range_steps, prefetch, additions materialized (carry
    scheme 1), log2 threads x min_blocks (the register cap's denominator),
    thread-sequential form, TMA form, log2 chunk words (thread forms), stages
    (TMA form), multiply-form shifts (thread forms) and look-back additions
    (carry scheme 2); 0 where a knob does not apply."""
    layout = int(s.get("layout", 0))
    cut = int(s.get("cut_adds", 0))
    return [math.log2(s["warps"]), math.log2(max(1, s["min_blocks"])),
            math.log2(1 + max(0, s["ctas_per_sm"])), math.log2(max(1, s["range_steps"])),
            float(s["prefetch"]), float(cut == 1),
            math.log2(32 * s["warps"] * max(1, s["min_blocks"])),
            float(layout >= 1), float(layout == 2),
            math.log2(s.get("chunk_words", 4)) if layout >= 1 else 0.0,
            float(s.get("stages", 2)) if layout == 2 else 0.0,
            float(s.get("shift_mul", 0)) if layout >= 1 else 0.0,
            float(cut == 2)]


N_SCHEDULE_FEATURES = 13
N_PROGRAM_FEATURES = 15
N_FEATURES = N_PROGRAM_FEATURES + 1 + N_SCHEDULE_FEATURES + 1

# The fitted model shipped with the package (written by
# ``python -m bitstreamzoo_b200.tuner --out``).
DEFAULT_MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "cost_model.npz")


def program_features(prog) -> list[float]:
    """DAG features of a compiled :class:`Program` (``bsz_program_features``)."""
    lib = prog.ctx.lib
    buf = (ctypes.c_float * 64)()
    n = lib.bsz_program_features(prog.ctx.h, prog.h, buf, 64)
    if n < 0:
        raise BszError(_lib.last_error())
    return list(buf[:n])


def register_pressure(pfeat: list[float], sched: dict) -> float:
    """log2 of (registers the DAG's peak live values need, 2 per 64-bit value
    plus ~16 of bookkeeping) over the register cap the schedule's launch
    bounds allow: above 0 the generated kernel spills."""
    peak = 2 ** pfeat[14] - 1
    blocks = 1 if int(sched.get("layout", 0)) == 2 else max(1, sched["min_blocks"])
    cap = min(255.0, 65536.0 / (32 * sched["warps"] * blocks))
    return math.log2(2 * peak + 16) - math.log2(cap)


def feature_row(pfeat: list[float], nbits: int, sched: dict) -> list[float]:
    return (list(pfeat) + [math.log2(max(2, nbits))] + encode_schedule(sched)
            + [register_pressure(pfeat, sched)])


# ------------------------------------------------------------- measurement --


def measure(ctx, prog, nbits: int, inputs: dict, sched: dict, reps: int = 3, warm: int = 1) -> float:
    """Median device ms of one fused execution under ``sched``.

    ``inputs`` maps input names to device buffers as ``(ptr, n_words)`` (they
    are bound in place).  The first ``warm`` executions compile the kernels
    and are not timed."""
    times = []
    for i in range(warm + reps):
        r = prog.run(nbits, MODE_FUSED)
        r.set_schedule(sched)
        for k, (ptr, nw) in inputs.items():
            r.bind(k, ("borrow", ptr, nw))
        ctx.profile(True)
        r.execute()
        rep = ctx.profile_report()
        ctx.profile(False)
        del r
        if i >= warm:
            times.append(sum(v["ms"] for v in rep.values()))
    return float(np.median(times))


def regret(times: dict, pick) -> float:
    """Time of the picked schedule over the best in ``times`` (schedule key ->
    ms), minus one."""
    best = min(times.values())
    return times[schedule_key(pick) if isinstance(pick, dict) else pick] / best - 1.0


class Autotuner:
    """Exhaustive search over ``candidates``, cached per (program, length).

    The cache is a JSON file mapping sha1(program text) + ':' + length to the
    best schedule and every timing."""

    def __init__(self, ctx, candidates=None, cache_path: str | None = None, reps: int = 3):
        self.ctx = ctx
        self.candidates = candidates or CANDIDATES
        self.cache_path = cache_path
        self.reps = reps
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    @staticmethod
    def key(source: str, nbits: int) -> str:
        return hashlib.sha1(source.encode()).hexdigest() + ":" + str(int(nbits))

    def sweep(self, prog, source: str, nbits: int, inputs: dict) -> dict:
        """Times every candidate; returns {schedule key: ms}."""
        k = self.key(source, nbits)
        if k in self.cache:
            return {tuple(json.loads(t)): ms for t, ms in self.cache[k]["times"].items()}
        times = {}
        for s in self.candidates:
            times[schedule_key(s)] = measure(self.ctx, prog, nbits, inputs, s, reps=self.reps)
        best = min(times, key=times.get)
        self.cache[k] = {"best": list(best), "times": {json.dumps(list(t)): ms for t, ms in times.items()}}
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump(self.cache, f)
        return times

    def best(self, prog, source: str, nbits: int, inputs: dict) -> dict:
        times = self.sweep(prog, source, nbits, inputs)
        bk = min(times, key=times.get)
        return dict(zip([k for k, _ in _lib.Schedule._fields_], bk))


# -------------------------------------------------------------- cost model --


class CostModel:
    """MLP cost model (in -> hidden x layers -> 1, ReLU, FP32) on libbsz's
    CUDA kernels.  Inputs are standardised with the training set's mean and
    standard deviation; the target is standardised log(ms)."""

    def __init__(self, ctx, in_dim: int, hidden: int = 256, layers: int = 3, seed: int = 1,
                 weight_decay: float = 0.0):
        self.ctx = ctx
        self.lib = ctx.lib
        self.in_dim = in_dim
        self.h = self.lib.bsz_mlp_create(ctx.h, in_dim, hidden, layers, seed)
        if not self.h:
            raise BszError(_lib.last_error())
        self.set_weight_decay(weight_decay)
        self.mu = np.zeros(in_dim, np.float32)
        self.sd = np.ones(in_dim, np.float32)
        self.y_mu = 0.0
        self.y_sd = 1.0
        # the training rows' feature range: inputs are clipped to it, so a
        # program or length outside the training suite (longer streams, more
        # outputs) is predicted as the nearest trained one, not extrapolated
        self.lo = None
        self.hi = None

    def __del__(self):
        try:
            if self.h:
                self.lib.bsz_mlp_free(self.h)
                self.h = None
        except Exception:
            pass

    def set_weight_decay(self, wd: float):
        _lib.check(self.lib.bsz_mlp_set_weight_decay(self.h, ctypes.c_float(wd)))

    # raw access (standardised units), used by the gradient checks
    @property
    def n_params(self) -> int:
        return int(self.lib.bsz_mlp_num_params(self.h))

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        _lib.check(self.lib.bsz_mlp_params(self.h, p.ctypes.data, 1))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        _lib.check(self.lib.bsz_mlp_params(self.h, p.ctypes.data, 0))

    def raw_predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty(x.shape[0], np.float32)
        _lib.check(self.lib.bsz_mlp_predict(self.h, x.ctypes.data, x.shape[0], out.ctypes.data))
        return out

    def raw_gradients(self, x: np.ndarray, y: np.ndarray) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.empty(self.n_params, np.float32)
        loss = ctypes.c_float()
        _lib.check(self.lib.bsz_mlp_gradients(self.h, x.ctypes.data, y.ctypes.data, x.shape[0],
                                               g.ctypes.data, ctypes.byref(loss)))
        return float(loss.value), g

    def raw_train_step(self, x: np.ndarray, y: np.ndarray, lr: float) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = ctypes.c_float()
        _lib.check(self.lib.bsz_mlp_train_step(self.h, x.ctypes.data, y.ctypes.data, x.shape[0],
                                                ctypes.c_float(lr), ctypes.byref(loss)))
        return float(loss.value)

    # standardised training and prediction
    def fit(self, X, ms, steps: int = 1500, batch: int = 256, lr: float = 1e-3, seed: int = 0,
            groups=None) -> list:
        """Fits log(ms); returns the loss of every step.  With ``groups`` (one
        label per row, e.g. the (program, length) case), the target is log(ms)
        minus its group's mean: the model then learns how schedules rank
        within a case, which is all a pick needs, instead of spending its
        capacity on the cases' absolute times."""
        X = np.asarray(X, np.float32)
        y = np.log(np.asarray(ms, np.float64))
        if groups is not None:
            groups = np.asarray(groups)
            for g in np.unique(groups):
                sel = groups == g
                y[sel] -= y[sel].mean()
        self.mu = X.mean(0)
        self.sd = np.maximum(X.std(0), 1e-3).astype(np.float32)
        self.lo, self.hi = X.min(0), X.max(0)
        self.y_mu = float(y.mean())
        self.y_sd = float(max(y.std(), 1e-3))
        Xs = (X - self.mu) / self.sd
        ys = ((y - self.y_mu) / self.y_sd).astype(np.float32)
        rng = np.random.default_rng(seed)
        losses = []
        n = Xs.shape[0]
        for t in range(steps):
            idx = rng.integers(0, n, size=min(batch, n))
            # cosine decay to 5% of the initial rate
            rate = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * t / max(1, steps))))
            losses.append(self.raw_train_step(Xs[idx], ys[idx], rate))
        return losses

    def predict_ms(self, X) -> np.ndarray:
        X = np.asarray(X, np.float32)
        if self.lo is not None:
            X = np.clip(X, self.lo, self.hi)
        X = (X - self.mu) / self.sd
        return np.exp(self.raw_predict(X).astype(np.float64) * self.y_sd + self.y_mu)

    def rank(self, pfeat: list[float], nbits: int, candidates=None) -> list[dict]:
        """Candidates sorted by predicted time (fastest first)."""
        candidates = candidates or CANDIDATES
        pred = self.predict_ms([feature_row(pfeat, nbits, s) for s in candidates])
        return [candidates[i] for i in np.argsort(pred, kind="stable")]

    def choose(self, prog, nbits: int, candidates=None, top_k: int = 1, inputs: dict | None = None,
               reps: int = 3) -> dict:
        """The predicted-fastest schedule; with ``top_k`` > 1 (and device
        ``inputs``) the fastest measured of the ``top_k`` best predictions."""
        ranked = self.rank(program_features(prog), nbits, candidates)
        if top_k <= 1 or inputs is None:
            return ranked[0]
        timed = [(measure(self.ctx, prog, nbits, inputs, s, reps=reps), i) for i, s in enumerate(ranked[:top_k])]
        return ranked[min(timed)[1]]

    def save(self, path: str):
        extra = {} if self.lo is None else {"lo": self.lo, "hi": self.hi}
        np.savez(path, params=self.params(), mu=self.mu, sd=self.sd, y=np.array([self.y_mu, self.y_sd]),
                 in_dim=np.array([self.in_dim]), **extra)

    @classmethod
    def load_default(cls, ctx, path: str | None = None):
        """The shipped model, or None when it has not been trained for the
        current feature encoding."""
        path = path or DEFAULT_MODEL_PATH
        if not os.path.exists(path):
            return None
        with np.load(path) as z:
            if int(z["in_dim"][0]) != N_FEATURES:
                return None
        m = cls(ctx, N_FEATURES)
        m.load(path)
        return m

    def load(self, path: str):
        z = np.load(path)
        if int(z["in_dim"][0]) != self.in_dim:
            raise ValueError(f"{path}: a model over {int(z['in_dim'][0])} features, not {self.in_dim}")
        self.set_params(z["params"])
        self.mu, self.sd = z["mu"], z["sd"]
        self.y_mu, self.y_sd = float(z["y"][0]), float(z["y"][1])
        if "lo" in z:
            self.lo, self.hi = z["lo"], z["hi"]


# ------------------------------------------------------------------- study --


def tuning_suite(n_train: int = 24, n_test: int = 8, seed: int = 20261210, max_ops: int = 1500):
    """Seeded training and held-out program sources.

    Each DAG draws its op mix from Dirichlet(1) over five classes (AND/OR/
    XOR, shift left, ADD, shift right, NOT), its size log-uniformly from 50
    to ``max_ops`` generator ops, an operand window from {all, 6, 24, 96}
    and a maximum shift distance from {1, 7, 70}.  The held-out set starts
    with the 300- and 2,000-op regex-shaped DAGs (so a time-budgeted study
    always evaluates them)."""
    from .workloads import regex_dag_src, shaped_dag_src

    rng = np.random.default_rng(seed)

    def draw(k):
        p = rng.dirichlet(np.ones(5))
        n_ops = int(round(math.exp(rng.uniform(math.log(50), math.log(max_ops)))))
        return shaped_dag_src(n_ops=n_ops, seed=seed + k, window=int(rng.choice([0, 6, 24, 96])),
                              p_bit=float(p[0]), p_shl=float(p[1]), p_add=float(p[2]), p_shr=float(p[3]),
                              max_shift=int(rng.choice([1, 7, 70])))

    train = [draw(k) for k in range(n_train)]
    test = [regex_dag_src(n_ops=300, seed=seed + 7), regex_dag_src(n_ops=2000)][: max(0, n_test)]
    test += [draw(1000 + k) for k in range(max(0, n_test - 2))]
    return train, test


def _device_inputs(nbits: int, n_inputs: int, seed: int):
    import torch

    nw = (nbits + 63) // 64
    g = torch.Generator(device="cuda").manual_seed(seed)
    bufs = [torch.randint(-2**63, 2**63 - 1, (nw,), dtype=torch.int64, device="cuda", generator=g)
            for _ in range(n_inputs)]
    if nbits % 64:
        mask = (1 << (nbits % 64)) - 1
        for b in bufs:
            b[-1:].bitwise_and_(mask if mask < 2**63 else mask - 2**64)
    torch.cuda.synchronize()
    return bufs, {f"b{i}": (b.data_ptr(), nw) for i, b in enumerate(bufs)}


CODEGEN_KEYS = ("warps", "min_blocks", "prefetch", "cut_adds", "layout", "chunk_words", "stages", "unroll",
                "shift_mul")


def codegen_key(s: dict) -> tuple:
    """The knobs that change the generated source (one NVRTC compile each)."""
    return tuple(int(s.get(k, DEFAULT_SCHEDULE[k])) for k in CODEGEN_KEYS)


def precompile(srcs, candidates=None, nbits: int = 1 << 22, threads: int | None = None, log=None,
               only=None) -> float:
    """Compiles the fused kernels of every (program, code variant) pair
    ahead of timing, in parallel host threads, each with its own context
    (NVRTC runs on the host; the process-wide kernel cache then serves the
    timing runs).  Kernels do not depend on the stream length beyond its
    word alignment, so one short run per pair (``nbits``, a multiple of 64
    long enough for every form) compiles what every length uses.  ``only``
    (one set of :func:`codegen_key` values per source, or None for all)
    limits a source to the variants that will be timed.  Returns the wall
    seconds."""
    import concurrent.futures as cf
    import threading
    import time as _time

    from . import Context

    candidates = candidates or CANDIDATES
    reps = {}
    for s in candidates:
        reps.setdefault(codegen_key(s), s)
    jobs = [(src, s) for i, src in enumerate(srcs) for k, s in reps.items()
            if only is None or only[i] is None or k in only[i]]
    local = threading.local()
    ctxs = []
    lock = threading.Lock()
    nw = (nbits + 63) // 64
    rng = np.random.default_rng(7)
    host_in = [rng.integers(0, 2**64, size=nw, dtype=np.uint64) for _ in range(8)]

    def work(job):
        if not hasattr(local, "ctx"):
            local.ctx = Context(0)
            local.progs = {}
            with lock:
                ctxs.append(local.ctx)
        src, sched = job
        prog = local.progs.get(src)
        if prog is None:
            prog = local.progs[src] = local.ctx.compile(src)
        r = prog.run(nbits, MODE_FUSED)
        r.set_schedule(sched)
        for i in range(8):
            try:
                r.bind(f"b{i}", host_in[i])
            except BszError:
                pass   # the program has fewer inputs
        r.execute()

    t0 = _time.time()
    with cf.ThreadPoolExecutor(max_workers=threads or min(16, os.cpu_count() or 4)) as ex:
        for k, _ in enumerate(ex.map(work, jobs)):
            if log and (k + 1) % 200 == 0:
                log(f"precompiled {k + 1}/{len(jobs)} t={_time.time() - t0:.0f}s")
    for c in ctxs:
        c.close()
    return _time.time() - t0


def study(ctx, train_srcs, test_srcs, sizes=(1 << 22, 1 << 25, 1 << 28), candidates=None,
          sample_frac: float = 0.5, reps: int = 3, steps: int = 1500, seed: int = 0, log=None,
          weight_decay: float = 0.05, precompile_threads: int = 0, train_budget_s: float | None = None,
          test_budget_s: float | None = None, batch: int = 24, collect_only: bool = False) -> dict:
    """Collects timings, fits a :class:`CostModel` and reports pick regret on
    the held-out programs for the model's top-1 and top-4 picks and for the
    default schedule.

    Sampling budget: compiling a generated kernel costs far more than timing
    it, so each training program draws a ``sample_frac`` share of the
    code-generation variants (warps, register cap, prefetch, add cuts) and
    times every launch variant of those at every length.  Held-out programs
    are timed exhaustively (that is the regret's reference).  Programs are
    compiled in batches of ``batch``; with ``train_budget_s`` /
    ``test_budget_s`` no new program starts once that many seconds of the
    phase have passed (the report gives how many programs each phase used).
    ``collect_only`` returns the training rows without fitting."""
    import time as _time

    candidates = candidates or CANDIDATES
    rng = np.random.default_rng(seed)
    t0 = _time.time()
    X, y = [], []
    n_timed = 0
    bufs_by_size = {n: _device_inputs(n, 8, seed + n % 997) for n in sizes}
    progs = {}

    def prog_of(src):
        if src not in progs:
            progs[src] = (ctx.compile(src), None)
            progs[src] = (progs[src][0], program_features(progs[src][0]))
        return progs[src]

    groups = []
    variants = sorted({codegen_key(s) for s in candidates})
    chosen_by = []
    for i in range(len(train_srcs)):
        k = max(1, int(round(sample_frac * len(variants))))
        chosen_by.append({variants[j] for j in rng.choice(len(variants), size=k, replace=False)})
    t_pc = 0.0

    def compile_batch(srcs, only):
        nonlocal t_pc
        if precompile_threads:
            t_pc += precompile(srcs, candidates, threads=precompile_threads, only=only)

    t0 = _time.time()
    n_train_used = len(train_srcs)
    for i, src in enumerate(train_srcs):
        if train_budget_s is not None and _time.time() - t0 > train_budget_s:
            n_train_used = i
            break
        if i % batch == 0:
            compile_batch(train_srcs[i:i + batch], chosen_by[i:i + batch])
        prog, pf = prog_of(src)
        chosen = chosen_by[i]
        for n in sizes:
            for s in candidates:
                if codegen_key(s) not in chosen:
                    continue
                ms = measure(ctx, prog, n, bufs_by_size[n][1], s, reps=reps)
                X.append(feature_row(pf, n, s))
                y.append(ms)
                groups.append(i * 1000 + sizes.index(n))
                n_timed += 1
        if log:
            log(f"train {i + 1}/{len(train_srcs)} timed={n_timed} t={_time.time() - t0:.0f}s")
    t_collect = _time.time() - t0
    if collect_only:
        return {"X": X, "y": y, "groups": groups, "n_train_programs": n_train_used, "n_train_timings": n_timed,
                "precompile_s": t_pc, "collect_s": t_collect}
    model = CostModel(ctx, len(X[0]), seed=seed + 1, weight_decay=weight_decay)
    t1 = _time.time()
    losses = model.fit(X, y, steps=steps, seed=seed, groups=groups)
    t_fit = _time.time() - t1

    default_key = schedule_key(DEFAULT_SCHEDULE)
    rows = []
    raw_test = []
    t2 = _time.time()
    n_test_used = len(test_srcs)
    for i, src in enumerate(test_srcs):
        if test_budget_s is not None and _time.time() - t2 > test_budget_s:
            n_test_used = i
            break
        if i % batch == 0:
            compile_batch(test_srcs[i:i + batch], None)
        prog, pf = prog_of(src)
        for n in sizes:
            times = {schedule_key(s): measure(ctx, prog, n, bufs_by_size[n][1], s, reps=reps)
                     for s in candidates}
            if default_key not in times:
                times[default_key] = measure(ctx, prog, n, bufs_by_size[n][1], DEFAULT_SCHEDULE, reps=reps)
            raw_test.append({"program": i, "bits": n,
                             "X": [feature_row(pf, n, s) for s in candidates],
                             "ms": [times[schedule_key(s)] for s in candidates],
                             "default_ms": times[default_key]})
            ranked = model.rank(pf, n, candidates)
            top4 = min(times[schedule_key(s)] for s in ranked[:4])
            best = min(times.values())
            cand_ms = [times[schedule_key(s)] for s in candidates]
            rows.append({"program": i, "ops": int(round(2 ** pf[0] - 1)), "bits": n, "best_ms": best,
                         "best": list(min(times, key=times.get)),
                         "regret_top1": times[schedule_key(ranked[0])] / best - 1,
                         "regret_top4": top4 / best - 1,
                         "regret_default": times[default_key] / best - 1,
                         # a uniformly random pick from the space, in expectation
                         "regret_random": float(np.mean(cand_ms)) / best - 1,
                         "tuning_ms_exhaustive": float(sum(cand_ms)) * (reps + 1),
                         "tuning_ms_top4": float(sum(times[schedule_key(s)] for s in ranked[:4])) * (reps + 1)})
        if log:
            log(f"test {i + 1}/{len(test_srcs)} t={_time.time() - t0:.0f}s")

    def stats(key):
        v = np.array([r[key] for r in rows])
        return {"mean": float(v.mean()), "median": float(np.median(v)), "max": float(v.max())}

    return {"model": model, "rows": rows, "n_candidates": len(candidates), "n_train_programs": n_train_used,
            "n_test_programs": n_test_used, "sizes": list(sizes), "sample_frac": sample_frac,
            "precompile_s": t_pc, "test_s": _time.time() - t2,
            "n_train_timings": n_timed, "loss_first": float(np.mean(losses[:20])),
            "loss_last": float(np.mean(losses[-20:])), "collect_s": t_collect, "fit_s": t_fit,
            "regret_top1": stats("regret_top1"), "regret_top4": stats("regret_top4"),
            "regret_default": stats("regret_default"), "regret_random": stats("regret_random"),
            "top1_beats_default_frac": float(np.mean([r["regret_top1"] <= r["regret_default"] for r in rows])),
            "device_time_saved_top4": 1.0 - float(np.sum([r["tuning_ms_top4"] for r in rows]) /
                                                  np.sum([r["tuning_ms_exhaustive"] for r in rows])),
            "exhaustive_timings_per_case": len(candidates),
            # every timing, for offline study of the model
            "raw": {"train_X": X, "train_ms": y, "train_groups": groups, "test": raw_test}}


def extend(ctx, prev: dict, train_srcs, sizes, steps: int = 1500, seed: int = 0, weight_decay: float = 0.05,
           **collect) -> tuple:
    """Adds training rows at new lengths to a previous study's report
    (``prev``, with its ``raw`` timings), refits on all rows and re-scores
    the previous held-out cases from their recorded timings (no re-timing).
    Returns (model, summary)."""
    new = study(ctx, train_srcs, [], sizes=sizes, seed=seed, collect_only=True, **collect)
    raw = prev["raw"]
    X = list(raw["train_X"]) + new["X"]
    y = list(raw["train_ms"]) + new["y"]
    # new groups: offset past every (program, length) id of the previous rows
    groups = list(raw["train_groups"]) + [10 ** 6 + g for g in new["groups"]]
    model = CostModel(ctx, len(X[0]), seed=seed + 1, weight_decay=weight_decay)
    losses = model.fit(X, y, steps=steps, seed=seed, groups=groups)
    rows = []
    for c in raw["test"]:
        ms = np.asarray(c["ms"], np.float64)
        order = np.argsort(model.predict_ms(c["X"]), kind="stable")
        best = float(ms.min())
        rows.append({"regret_top1": ms[order[0]] / best - 1, "regret_top4": ms[order[:4]].min() / best - 1,
                     "regret_default": c["default_ms"] / best - 1, "regret_random": float(ms.mean()) / best - 1})

    def stats(key):
        v = np.array([r[key] for r in rows])
        return {"mean": float(v.mean()), "median": float(np.median(v)), "max": float(v.max())}

    summary = {"n_rows": len(X), "n_new_rows": len(new["X"]), "n_new_programs": new["n_train_programs"],
               "new_sizes": list(sizes), "collect_s": new["collect_s"], "precompile_s": new["precompile_s"],
               "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:])),
               "held_out_cases": len(rows)}
    for k in ("regret_top1", "regret_top4", "regret_default", "regret_random"):
        summary[k] = stats(k)
    return model, summary


def main(argv=None):
    """python -m bitstreamzoo_b200.tuner [--out model.npz] [--json report.json]
    runs :func:`study` on the default suite and saves the fitted model."""
    import argparse

    from . import Context

    # tens of thousands of kernels: keep them in this process, not on disk
    os.environ.setdefault("BSZ_KERNEL_CACHE", "off")
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--json", default=None)
    ap.add_argument("--train", type=int, default=48)
    ap.add_argument("--test", type=int, default=8)
    ap.add_argument("--sample-frac", type=float, default=0.5)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--max-ops", type=int, default=3000)
    ap.add_argument("--threads", type=int, default=16, help="parallel precompile threads (0: none)")
    ap.add_argument("--sizes", default="22,25,28", help="log2 stream lengths (bits), comma-separated")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--train-budget", type=float, default=None, help="seconds: no new training batch after")
    ap.add_argument("--test-budget", type=float, default=None, help="seconds: no new held-out batch after")
    ap.add_argument("--extend", default=None,
                    help="a previous study's JSON report: time its first --train training programs at --sizes, "
                         "refit on all rows, re-score its held-out cases")
    a = ap.parse_args(argv)
    ctx = Context(0)
    train, test = tuning_suite(a.train, a.test, max_ops=a.max_ops)
    sizes = tuple(1 << int(x) for x in a.sizes.split(","))
    if a.extend:
        with open(a.extend) as f:
            prev = json.load(f)
        model, summary = extend(ctx, prev, train, sizes, steps=a.steps, sample_frac=a.sample_frac, reps=a.reps,
                                log=lambda m: print(m, flush=True), precompile_threads=a.threads,
                                train_budget_s=a.train_budget)
        if a.out:
            model.save(a.out)
        print(json.dumps(summary))
        if a.json:
            with open(a.json, "w") as f:
                json.dump(summary, f, indent=1)
        return 0
    rep = study(ctx, train, test, sizes=sizes, sample_frac=a.sample_frac, steps=a.steps, reps=a.reps,
                log=lambda m: print(m, flush=True), precompile_threads=a.threads,
                train_budget_s=a.train_budget, test_budget_s=a.test_budget)
    model = rep.pop("model")
    if a.out:
        model.save(a.out)
    summary = {k: v for k, v in rep.items() if k not in ("rows", "raw")}
    print(json.dumps(summary))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
