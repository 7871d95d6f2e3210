"""ctypes binding of libsumcheck_b200.so (the C ABI of include/sumcheck_b200.h).

The library is built in-tree by ``sumcheck-triton_b200/build.py``. There is no fallback:
if it is missing or fails to load, every prover call raises.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p
from pathlib import Path

from .fields import UnsafeModulusError

LIB_PATH = Path(os.environ.get("SUMCHECK_B200_LIB", Path(__file__).resolve().parent / "libsumcheck_b200.so"))

SC_OK = 0
SC_ERR_INVALID = 1
SC_ERR_UNSAFE_MODULUS = 2
SC_ERR_CUDA = 3
SC_ERR_UNSUPPORTED = 4
SC_ERR_DEVICE = 5
SC_ERR_NOMEM = 6
SC_ERR_TIMEOUT = 7
SC_ERR_PENDING = 8
SC_SUSPENDED = 9

SC_SERVE_CONTINUOUS = 0
SC_SERVE_FIFO_PLAIN = 1
SERVE_POLICIES = {"continuous": SC_SERVE_CONTINUOUS, "fifo_plain": SC_SERVE_FIFO_PLAIN}

SC_CHALLENGE_SHA3 = 0
SC_CHALLENGE_FIXED = 1
SC_CHALLENGE_EXPLICIT = 2
CHALLENGE_MODES = {"sha3": SC_CHALLENGE_SHA3, "fixed": SC_CHALLENGE_FIXED, "explicit": SC_CHALLENGE_EXPLICIT}

SC_TABLE_UNIFORM = 0
SC_TABLE_BERNOULLI = 1
SC_TABLE_ARITH = 2

U32P = POINTER(c_uint32)
U64P = POINTER(c_uint64)
F64P = POINTER(c_double)


class ServerStats(ctypes.Structure):
    """sc_server_stats."""

    _fields_ = [
        ("submitted", c_uint64), ("completed", c_uint64), ("failed", c_uint64), ("suspended", c_uint64),
        ("ticks", c_uint64),
        ("items", c_uint64), ("peak_inflight", c_uint64), ("peak_footprint", c_uint64), ("budget", c_uint64),
        ("busy_s", c_double), ("alloc_s", c_double), ("wait_s", c_double), ("build_s", c_double),
    ]


# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "sc_version": (c_int, []),
    "sc_last_error": (c_char_p, []),
    "sc_ctx_create": (c_int, [c_int, c_void_p, POINTER(c_void_p)]),
    "sc_ctx_destroy": (c_int, [c_void_p]),
    "sc_ctx_synchronize": (c_int, [c_void_p]),
    "sc_ctx_set_timing": (c_int, [c_void_p, c_int]),
    "sc_ctx_launch_times": (c_int, [c_void_p, POINTER(c_float), c_int, POINTER(c_int)]),
    "sc_field_init": (c_int, [c_int, U32P, c_uint32, POINTER(c_void_p)]),
    "sc_field_destroy": (c_int, [c_void_p]),
    "sc_expr_compile": (
        c_int,
        [c_int, c_int, POINTER(c_int64), U32P, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32), POINTER(c_void_p)],
    ),
    "sc_expr_destroy": (c_int, [c_void_p]),
    "sc_expr_degree": (c_int, [c_void_p]),
    "sc_expr_num_vars": (c_int, [c_void_p]),
    "sc_tables_generate": (c_int, [c_void_p, c_void_p, c_int, c_int, POINTER(c_int32), c_uint64, c_void_p]),
    "sc_tables_to_mont": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_int]),
    "sc_tables_from_mont": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_int]),
    "sc_field_apply": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_uint64]),
    "sc_prove_noalloc": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, U32P, U32P, U32P, U32P, U32P, U64P],
    ),
    "sc_batch_create": (
        c_int,
        [c_void_p, c_void_p, c_int, POINTER(c_void_p), POINTER(c_int32), POINTER(c_void_p), c_int, c_int, c_int,
         POINTER(c_void_p)],
    ),
    "sc_batch_create_tiled": (
        c_int,
        [c_void_p, c_void_p, c_int, POINTER(c_void_p), POINTER(c_int32), POINTER(c_void_p), c_int, POINTER(c_int32),
         POINTER(c_int32), POINTER(c_void_p)],
    ),
    "sc_batch_run": (c_int, [c_void_p]),
    "sc_batch_launch": (c_int, [c_void_p]),
    "sc_batch_join": (c_int, [c_void_p]),
    "sc_batch_wait": (c_int, [c_void_p]),
    "sc_batch_result": (c_int, [c_void_p, c_int, U32P, U32P, U32P, U32P, U64P]),
    "sc_batch_results": (c_int, [c_void_p, U32P, U32P, U32P, U32P, U64P]),
    "sc_batch_tick_times": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), c_int, POINTER(c_int)]),
    "sc_batch_classes": (c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), c_int, POINTER(c_int)]),
    "sc_batch_class_proofs": (c_int, [c_void_p, c_int, POINTER(c_int32), c_int, POINTER(c_int)]),
    "sc_batch_destroy": (c_int, [c_void_p]),
    "sc_calibrate_imad": (c_int, [c_void_p, POINTER(c_double)]),
    "sc_split_create": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_int, POINTER(c_void_p)]),
    "sc_split_local_rounds": (c_int, [c_void_p]),
    "sc_split_round": (c_int, [c_void_p, c_int, U32P]),
    "sc_split_commit": (c_int, [c_void_p, c_int, U32P]),
    "sc_split_last_entries": (c_int, [c_void_p, U32P]),
    "sc_split_finish": (c_int, [c_void_p, U32P]),
    "sc_split_result": (c_int, [c_void_p, U32P, U32P, U32P, U32P, U64P]),
    "sc_split_destroy": (c_int, [c_void_p]),
    "sc_server_create": (
        c_int, [c_int, c_void_p, c_int, c_uint64, c_int, c_int, c_int, c_int, c_int, POINTER(c_void_p)],
    ),
    "sc_server_footprint": (c_int, [c_void_p, c_void_p, c_int, U64P]),
    "sc_server_reserve": (c_int, [c_void_p, c_uint64]),
    "sc_server_submit": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_int32), c_uint64, c_int, U64P]),
    "sc_server_wait": (c_int, [c_void_p, c_uint64, c_int]),
    "sc_server_drain": (c_int, [c_void_p, c_int]),
    "sc_server_result": (c_int, [c_void_p, c_uint64, U32P, U32P, U32P, U32P, U64P]),
    "sc_server_times": (c_int, [c_void_p, c_uint64, F64P, F64P, F64P]),
    "sc_server_release": (c_int, [c_void_p, c_uint64]),
    "sc_server_stats_get": (c_int, [c_void_p, POINTER(ServerStats)]),
    "sc_server_suspend": (c_int, [c_void_p, c_uint64]),
    "sc_server_transcript": (c_int, [c_void_p, c_uint64, U32P, c_uint64]),
    "sc_server_submit_resume": (c_int, [c_void_p, c_void_p, POINTER(c_int32), c_uint64, U32P, c_uint64, U64P]),
    "sc_transcript_words": (c_int, [c_void_p, c_void_p, c_int, U64P]),
    "sc_transcript_init": (c_int, [c_void_p, c_void_p, c_int, c_int, c_uint64, U32P, c_uint64]),
    "sc_transcript_info": (c_int, [U32P, c_uint64, POINTER(c_int), POINTER(c_int), POINTER(c_int), U64P]),
    "sc_transcript_result": (c_int, [c_void_p, c_void_p, U32P, c_uint64, U32P, U32P, U32P, U32P, U64P]),
    "sc_tables_tag": (c_int, [c_int, POINTER(c_int32), c_uint64, U64P]),
    "sc_prove_resume": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, U32P, c_int, U32P, c_uint64]),
    "sc_server_destroy": (c_int, [c_void_p]),
    "sc_prove_launches": (c_int, [c_void_p, c_void_p, c_void_p, c_int, POINTER(c_int), POINTER(c_int)]),
    "sc_prove": (
        c_int,
        [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, U32P, U32P, U32P, U32P, U32P, U64P],
    ),
}


class SumcheckError(RuntimeError):
    """A failure reported by the native library."""


_lib = None


def load() -> ctypes.CDLL:
    """The loaded library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built; run `python sumcheck-triton_b200/build.py` "
            "(the prover has no CPU fallback)"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().sc_last_error().decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc == SC_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc == SC_ERR_UNSAFE_MODULUS:
        raise UnsafeModulusError(msg)
    if rc in (SC_ERR_INVALID, SC_ERR_UNSUPPORTED):
        raise ValueError(msg)
    if rc == SC_ERR_NOMEM:
        raise MemoryError(msg)
    if rc == SC_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise SumcheckError(msg)


def u32_array(values) -> ctypes.Array:
    vals = [int(v) & 0xFFFFFFFF for v in values]
    return (c_uint32 * max(1, len(vals)))(*vals)


def i32_array(values) -> ctypes.Array:
    vals = [int(v) for v in values]
    return (c_int32 * max(1, len(vals)))(*vals)


def i64_array(values) -> ctypes.Array:
    vals = [int(v) for v in values]
    return (c_int64 * max(1, len(vals)))(*vals)
