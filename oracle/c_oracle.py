"""ctypes wrapper of the C oracle (oracle/_build/liboracle.so) -- test infrastructure only.

Same call as ``oracle.prove`` but over limb-planar numpy tables, multithreaded, for sizes
the Python oracle cannot reach; also the timed CPU baseline of bench.py.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_int, c_int32, c_int64, c_size_t, c_uint8, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        subprocess.check_call(["make", "-s", "-C", str(HERE)])
    lib = ctypes.CDLL(str(LIB))
    lib.oracle_prove.restype = c_int
    lib.oracle_prove.argtypes = [c_int, POINTER(c_uint32), c_int, c_int, POINTER(c_int64), POINTER(c_int32),
                                 POINTER(c_int32), POINTER(c_int32), c_int, c_void_p, c_int, POINTER(c_uint32),
                                 c_int, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_uint64)]
    lib.oracle_prove_seeded.restype = c_int
    lib.oracle_prove_seeded.argtypes = [c_int, POINTER(c_uint32), c_int, c_int, POINTER(c_int64), POINTER(c_int32),
                                        POINTER(c_int32), POINTER(c_int32), c_int, POINTER(c_int32), c_uint64, c_int,
                                        POINTER(c_uint32), c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                        POINTER(c_uint64)]
    lib.oracle_generate.restype = c_int
    lib.oracle_generate.argtypes = [c_int, POINTER(c_uint32), c_int, c_int, POINTER(c_int32), c_uint64, c_void_p]
    lib.oracle_sha3_256.restype = None
    lib.oracle_sha3_256.argtypes = [POINTER(c_uint8), c_size_t, POINTER(c_uint8)]
    _lib = lib
    return lib


def _u32(xs):
    xs = [int(x) & 0xFFFFFFFF for x in xs]
    return (c_uint32 * max(1, len(xs)))(*xs)


def _limbs(x, L):
    return [(int(x) >> (32 * i)) & 0xFFFFFFFF for i in range(L)]


def generate(p: int, L: int, kinds, n: int, seed: int) -> np.ndarray:
    """Canonical limb-planar tables (K, L, 2^n) uint32; kinds as the C ABI's SC_TABLE_*."""
    K = len(kinds)
    out = np.empty((K, L, 1 << n), dtype=np.uint32)
    load().oracle_generate(L, _u32(_limbs(p, L)), K, n, (c_int32 * K)(*kinds), c_uint64(seed & (2**64 - 1)),
                           out.ctypes.data_as(c_void_p))
    return out


def sha3_256(data: bytes) -> bytes:
    buf = (c_uint8 * max(1, len(data))).from_buffer_copy(data or b"\0")
    out = (c_uint8 * 32)()
    load().oracle_sha3_256(buf, len(data), out)
    return bytes(out)


def _encode_terms(terms):
    coeffs = [int(c) for c, _f in terms]
    lens = [len(f) for _c, f in terms]
    offs, flat = [], []
    for _c, f in terms:
        offs.append(len(flat))
        flat.extend(f)
    return ((c_int64 * len(coeffs))(*coeffs), (c_int32 * len(lens))(*lens), (c_int32 * len(offs))(*offs),
            (c_int32 * max(1, len(flat)))(*flat), max(lens))


def _run(call, terms, K: int, p: int, L: int, n: int, mode: str, explicit, threads):
    coeffs, lens, offs, flat, d = _encode_terms(terms)
    polys = np.zeros((n, d + 1, L), dtype=np.uint32)
    chals = np.zeros((n, L), dtype=np.uint32)
    finals = np.zeros((1 + K, L), dtype=np.uint32)
    claim0 = np.zeros((L,), dtype=np.uint32)
    cs = c_uint64(0)
    m = {"sha3": 0, "fixed": 1, "explicit": 2}[mode]
    ex = _u32([w for c in (explicit or [0] * n) for w in _limbs(int(c) % p, L)])
    threads = threads or os.cpu_count() or 1
    rc = call(coeffs, lens, offs, flat, m, ex, int(threads), polys.ctypes.data_as(c_void_p),
              chals.ctypes.data_as(c_void_p), finals.ctypes.data_as(c_void_p), claim0.ctypes.data_as(c_void_p),
              ctypes.byref(cs))
    if rc:
        raise RuntimeError(f"oracle prove failed ({rc})")
    return {"round_polys": polys, "challenges": chals, "finals": finals, "claim0": claim0, "checksum": int(cs.value)}


def prove(terms, num_tables: int, p: int, L: int, tables: np.ndarray, mode: str = "sha3",
          explicit=None, threads: int | None = None) -> dict:
    """Outputs as Montgomery limb arrays: round_polys (n, d+1, L), challenges (n, L),
    finals (1+K, L), claim0 (L,), checksum int."""
    K = num_tables
    n = int(tables.shape[2]).bit_length() - 1
    t = np.ascontiguousarray(tables, dtype=np.uint32)
    return _run(lambda co, le, of, fl, m, ex, th, *out:
                load().oracle_prove(L, _u32(_limbs(p, L)), K, len(terms), co, le, of, fl, n,
                                    t.ctypes.data_as(c_void_p), m, ex, th, *out),
                terms, K, p, L, n, mode, explicit, threads)


def prove_seeded(terms, num_tables: int, p: int, L: int, n: int, kinds, seed: int, mode: str = "sha3",
                 explicit=None, threads: int | None = None) -> dict:
    """``prove`` of the tables ``generate(p, L, kinds, n, seed)`` would return, without
    holding them: round 0 generates its entries on the fly, so a proof of 2^n entries per
    table needs host memory for 2^(n-1) (Montgomery) entries per table only."""
    K = num_tables
    return _run(lambda co, le, of, fl, m, ex, th, *out:
                load().oracle_prove_seeded(L, _u32(_limbs(p, L)), K, len(terms), co, le, of, fl, n,
                                           (c_int32 * K)(*kinds), c_uint64(seed & (2**64 - 1)), m, ex, th, *out),
                terms, K, p, L, n, mode, explicit, threads)
