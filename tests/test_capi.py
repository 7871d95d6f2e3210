"""The C ABI without a GPU: the library loads, exports every declared symbol, and rejects
bad moduli and malformed expressions before touching the device."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from zkduel_b200 import _lib
from zkduel_b200.fields import FIELD_SPECS, montgomery_nprime

HEADER = Path(__file__).resolve().parents[1] / "include" / "sumcheck_b200.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(sc_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES)
    assert lib.sc_version() >= 100


def _field_init(p: int, L: int, nprime: int | None = None):
    lib = _lib.load()
    h = ctypes.c_void_p()
    limbs = _lib.u32_array([(p >> (32 * i)) & 0xFFFFFFFF for i in range(L)])
    rc = lib.sc_field_init(L, limbs, montgomery_nprime(p) if nprime is None else nprime, ctypes.byref(h))
    return rc, h


@pytest.mark.parametrize("p,L", [((1 << 64) - 59, 2), ((1 << 128) - 159, 4), (0xFFFFFFFF00000001 + 2, 2)])
def test_unsafe_moduli_rejected_by_library(p, L):
    rc, h = _field_init(p, L)
    assert rc == _lib.SC_ERR_UNSAFE_MODULUS and not h.value
    assert "valid only when" in _lib.last_error()


def test_wrong_nprime_and_even_modulus_rejected():
    rc, _ = _field_init((1 << 61) - 1, 2, 0x12345)
    assert rc == _lib.SC_ERR_UNSAFE_MODULUS and "nprime" in _lib.last_error()
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.sc_field_init(2, _lib.u32_array([0xFFFFFFFE, 1]), 1, ctypes.byref(h))
    assert rc == _lib.SC_ERR_UNSAFE_MODULUS and "odd modulus" in _lib.last_error()
    rc = lib.sc_field_init(3, _lib.u32_array([1, 2, 3]), 1, ctypes.byref(h))
    assert rc == _lib.SC_ERR_UNSUPPORTED


def _compile(nv, coeffs, lens, offs, flat):
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.sc_expr_compile(nv, len(coeffs), _lib.i64_array(coeffs), None, _lib.i32_array(lens),
                             _lib.i32_array(offs), _lib.i32_array(flat), ctypes.byref(h))
    return rc, h


def test_expression_compile_and_limits():
    lib = _lib.load()
    rc, h = _compile(3, [1, -2], [2, 3], [0, 2], [0, 1, 2, 2, 0])
    assert rc == 0 and lib.sc_expr_degree(h) == 3 and lib.sc_expr_num_vars(h) == 3
    lib.sc_expr_destroy(h)
    assert _compile(2, [1], [2], [0], [0, 2])[0] == _lib.SC_ERR_INVALID        # table out of range
    assert _compile(2, [1], [2], [1], [0, 1])[0] == _lib.SC_ERR_INVALID        # bad offset
    assert _compile(1, [1], [8], [0], [0] * 8)[0] == _lib.SC_ERR_UNSUPPORTED   # degree 8
    assert _compile(33, [1], [1], [0], [0])[0] == _lib.SC_ERR_UNSUPPORTED      # 33 tables


def test_configured_moduli_pass_the_library_guard_checks():
    # Acceptance then needs the device; without one the call fails after the guard, with
    # a CUDA error rather than a modulus error.
    for f in FIELD_SPECS.values():
        rc, h = _field_init(f.modulus, f.limbs)
        assert rc in (0, _lib.SC_ERR_CUDA), _lib.last_error()
        if rc == 0:
            _lib.load().sc_field_destroy(h)
