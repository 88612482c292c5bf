"""ctypes binding of include/bsz.h (libbsz.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libbsz.so")
EXE_PATH = os.path.join(PKG, "lib", "bsim_cuda")

u64p = ctypes.POINTER(ctypes.c_uint64)
i64p = ctypes.POINTER(ctypes.c_int64)
c_void_p = ctypes.c_void_p


class Stats(ctypes.Structure):
    _fields_ = [("op_count", ctypes.c_int64), ("n_kernel_launches", ctypes.c_int64),
                ("n_mallocs", ctypes.c_int64), ("n_segments", ctypes.c_int64),
                ("n_syncs", ctypes.c_int64), ("peak_bytes", ctypes.c_int64),
                ("max_live", ctypes.c_int64), ("kernel_ms", ctypes.c_double),
                ("compile_ms", ctypes.c_double), ("n_fused_launches", ctypes.c_int64),
                ("n_fused_fallbacks", ctypes.c_int64), ("n_vm_launches", ctypes.c_int64),
                ("walk_replayed", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Schedule(ctypes.Structure):
    _fields_ = [("warps", ctypes.c_int32), ("range_steps", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("min_blocks", ctypes.c_int32),
                ("prefetch", ctypes.c_int32), ("cut_adds", ctypes.c_int32), ("layout", ctypes.c_int32),
                ("chunk_words", ctypes.c_int32), ("stages", ctypes.c_int32),
                ("unroll", ctypes.c_int32), ("shift_mul", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Instance(ctypes.Structure):
    _fields_ = [("program", ctypes.c_int32), ("bitlength", ctypes.c_int64),
                ("inputs", ctypes.POINTER(ctypes.c_void_p)), ("outputs", ctypes.POINTER(ctypes.c_void_p))]


# name -> (restype, argtypes); every symbol declared in include/bsz.h
SIGNATURES = {
    "bsz_version": (ctypes.c_char_p, []),
    "bsz_last_error": (ctypes.c_char_p, []),
    "bsz_create": (c_void_p, [ctypes.c_int]),
    "bsz_destroy": (None, [c_void_p]),
    "bsz_stream": (c_void_p, [c_void_p]),
    "bsz_sync": (ctypes.c_int, [c_void_p]),
    "bsz_profile": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "bsz_profile_report": (ctypes.c_char_p, [c_void_p]),
    "bsz_compile": (c_void_p, [c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "bsz_program_free": (None, [c_void_p]),
    "bsz_static_ops": (ctypes.c_int64, [c_void_p, ctypes.POINTER(ctypes.c_char_p), i64p, ctypes.c_int]),
    "bsz_run_create": (c_void_p, [c_void_p, ctypes.c_int64, ctypes.c_int]),
    "bsz_run_free": (None, [c_void_p]),
    "bsz_set_param": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int64]),
    "bsz_run_set_schedule": (ctypes.c_int, [c_void_p, ctypes.POINTER(Schedule)]),
    "bsz_bind_input": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int64, c_void_p,
                                      ctypes.c_uint64, ctypes.c_int, ctypes.c_int]),
    "bsz_bind_broadcast": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint8),
                                          ctypes.c_int64]),
    "bsz_execute": (ctypes.c_int, [c_void_p, ctypes.POINTER(Stats)]),
    "bsz_execute_async": (ctypes.c_int, [c_void_p]),
    "bsz_run_wait": (ctypes.c_int, [c_void_p, ctypes.POINTER(Stats)]),
    "bsz_get_stream": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int64, c_void_p,
                                      ctypes.c_uint64]),
    "bsz_get_stream_device": (ctypes.c_int, [c_void_p, ctypes.c_char_p, ctypes.c_int64,
                                             ctypes.POINTER(c_void_p)]),
    "bsz_get_int": (ctypes.c_int, [c_void_p, ctypes.c_char_p, i64p]),
    "bsz_array_indices": (ctypes.c_int64, [c_void_p, ctypes.c_char_p, i64p, ctypes.c_int64]),
    "bsz_batch_create": (c_void_p, [c_void_p, ctypes.POINTER(c_void_p), ctypes.c_int,
                                    ctypes.POINTER(Instance), ctypes.c_int64, ctypes.POINTER(Schedule)]),
    "bsz_batch_launch": (ctypes.c_int, [c_void_p]),
    "bsz_batch_finish": (ctypes.c_int, [c_void_p, ctypes.POINTER(Stats)]),
    "bsz_batch_ints": (ctypes.c_int, [c_void_p, ctypes.c_int64, i64p, ctypes.c_int]),
    "bsz_batch_items": (ctypes.c_int64, [c_void_p]),
    "bsz_batch_free": (None, [c_void_p]),
    "bsz_program_features": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "bsz_mlp_create": (c_void_p, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64]),
    "bsz_mlp_num_params": (ctypes.c_int64, [c_void_p]),
    "bsz_mlp_train_step": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int, ctypes.c_float,
                                          ctypes.POINTER(ctypes.c_float)]),
    "bsz_mlp_predict": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_void_p]),
    "bsz_mlp_gradients": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int, c_void_p,
                                         ctypes.POINTER(ctypes.c_float)]),
    "bsz_mlp_params": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int]),
    "bsz_mlp_set_weight_decay": (ctypes.c_int, [c_void_p, ctypes.c_float]),
    "bsz_mlp_free": (None, [c_void_p]),
    "bsz_run_case_json": (ctypes.c_char_p, [c_void_p, ctypes.c_char_p, ctypes.c_char_p,
                                            ctypes.c_char_p, ctypes.c_int]),
    "bsz_op_not": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_uint64, ctypes.c_int64]),
    "bsz_op_and": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_uint64]),
    "bsz_op_or": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_uint64]),
    "bsz_op_xor": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_uint64]),
    "bsz_op_andnot": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_uint64]),
    "bsz_op_add": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_uint64,
                                  ctypes.c_int64]),
    "bsz_op_shl": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                  ctypes.c_int64]),
    "bsz_op_shr": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                  ctypes.c_int]),
    "bsz_op_popcount": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_uint64, u64p]),
    "bsz_add_noalloc": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_uint64, ctypes.c_int64,
                                       c_void_p]),
    "bsz_debug_add_lookback_hook": (None, [ctypes.c_int64, ctypes.c_int]),
    "bsz_s2p": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int64, ctypes.POINTER(c_void_p)]),
    "bsz_op_is_nonzero": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_uint64,
                                         ctypes.POINTER(ctypes.c_int)]),
}

_LIB = None


class BszError(RuntimeError):
    """An error reported by libbsz (parse, 3-address, runtime or CUDA)."""


def load():
    """Load libbsz.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m bitstreamzoo_b200.build` "
            "(the executor has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int):
    if rc != 0:
        raise BszError(load().bsz_last_error().decode(errors="replace"))


def last_error() -> str:
    return load().bsz_last_error().decode(errors="replace")
