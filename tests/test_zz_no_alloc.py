"""sc_prove_noalloc: proving for callers that cannot allocate device memory (GPU).

Some callers cannot call cudaMalloc: code that runs inside another framework's memory pool
or under a fixed device-memory budget, or a plug-in that must not grow the process's device
footprint once it has started. For them the library has sc_prove_noalloc, which keeps its
scratch in one array of device memory set aside when the library loads (32 MiB per GPU)
and allocates nothing when it is called.

These tests call it through the C ABI and compare every output with sc_prove's on the same
tables, bit for bit (integer work: the tolerance is zero), on two calls in a row -- the
second call finds the first call's leftovers in the shared array and must not be affected.
They pass alone in a fresh process and after the rest of the suite.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from zkduel_b200 import _lib, api
from zkduel_b200.configs import PLAIN_CONFIGS
from zkduel_b200.expression import encode_expression
from zkduel_b200.fields import get_field

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)


def _noalloc(ctx, fld, expr, n, tables, mode, L, d, K, explicit=None):
    polys = np.zeros((n, d + 1, L), dtype=np.uint32)
    chals = np.zeros((n, L), dtype=np.uint32)
    finals = np.zeros((1 + K, L), dtype=np.uint32)
    claim0 = np.zeros((L,), dtype=np.uint32)
    cs = ctypes.c_uint64(0)
    p = lambda a: a.ctypes.data_as(_lib.U32P)  # noqa: E731
    rc = _lib.load().sc_prove_noalloc(ctx.handle, fld.handle, expr.handle, n, ctypes.c_void_p(tables.data_ptr()),
                                      _lib.CHALLENGE_MODES[mode], explicit, p(polys), p(chals), p(finals),
                                      p(claim0), ctypes.byref(cs))
    return rc, polys, chals, finals, claim0, int(cs.value)


# (bit width, expression, table kinds, num_vars, challenge mode)
DEG7 = [["a", "b", "c", "d", "e", "f", "g"], (5, ["a", "h"]), (-1, ["c", "d", "e"])]
CASES = [
    (64, PLAIN_CONFIGS["plain_goldilocks"].expression, PLAIN_CONFIGS["plain_goldilocks"].table_kinds(), 12, "sha3"),
    (256, PLAIN_CONFIGS["plain_bls"].expression, None, 10, "sha3"),
    (32, PLAIN_CONFIGS["plain_p32"].expression, None, 15, "fixed"),
    (64, PLAIN_CONFIGS["plain_goldilocks"].expression, PLAIN_CONFIGS["plain_goldilocks"].table_kinds(), 1, "sha3"),
    (128, [["a", "b", "c"], (3, ["d"])], None, 14, "sha3"),   # 2^127 - 1: the Mersenne product
    (64, DEG7, None, 9, "sha3"),                              # the degree <= 7 kernel class
    (256, DEG7, None, 7, "sha3"),
    # the largest 1-limb proof of 10 tables that fits: fold buffers of 10 x 3 x 2^18 words
    # (30 MiB) end 2 MiB short of the 32 MiB array, so the carve's last offsets are in use
    (32, [["t0", "t1"], ["t2", "t3", "t4"], ["t5"], ["t6", "t7"], ["t8", "t9"]], None, 20, "sha3"),
]


@pytest.mark.parametrize("bw,expr_src,kinds,n,mode", CASES,
                         ids=[f"{bw}-n{n}-{m}-{i}" for i, (bw, _e, _k, n, m) in enumerate(CASES)])
def test_noalloc_matches_sc_prove_on_two_calls_in_a_row(bw, expr_src, kinds, n, mode):
    spec = get_field(bw)
    enc = encode_expression(expr_src)
    kinds = [_lib.SC_TABLE_BERNOULLI if k == "bernoulli" else _lib.SC_TABLE_UNIFORM
             for k in (kinds or ["uniform"] * enc.num_vars)]
    tables = api.generate_tables(spec, enc.num_vars, n, kinds, seed=77)
    expr = api.CompiledExpression(enc, spec.modulus)
    ref = api.prove_device(tables, expr, spec, n, mode)  # the existing entry point, sc_prove
    ctx = api.get_context(tables.device)
    fld = api.get_device_field(spec, ctx.device)
    for _call in range(2):
        rc, polys, chals, finals, claim0, cs = _noalloc(ctx, fld, expr, n, tables, mode, spec.limbs, enc.degree,
                                                        enc.num_vars)
        assert rc == _lib.SC_OK, _lib.last_error()
        assert np.array_equal(polys, ref.round_polys_mont)
        assert np.array_equal(chals, ref.challenges_mont)
        assert np.array_equal(finals, ref.finals_mont)
        assert np.array_equal(claim0, ref.claim0_mont)
        assert cs == ref.checksum


def test_noalloc_explicit_challenges_match_sc_prove():
    spec = get_field(256)
    expr_src = [["a", "b", "c"], (-3, ["a", "d"])]
    enc = encode_expression(expr_src)
    n = 6
    tables = api.generate_tables(spec, enc.num_vars, n, [0] * enc.num_vars, seed=5)
    expr = api.CompiledExpression(enc, spec.modulus)
    ch = [(i * 0x1234567 + 99) % spec.modulus for i in range(n)]
    ref = api.prove_device(tables, expr, spec, n, "explicit", ch)
    words = _lib.u32_array([w for c in ch for w in spec.montgomery_limbs(c)])
    ctx = api.get_context(tables.device)
    fld = api.get_device_field(spec, ctx.device)
    for _call in range(2):
        rc, polys, chals, finals, claim0, cs = _noalloc(ctx, fld, expr, n, tables, "explicit", spec.limbs, enc.degree,
                                                        enc.num_vars, explicit=words)
        assert rc == _lib.SC_OK, _lib.last_error()
        assert np.array_equal(polys, ref.round_polys_mont) and np.array_equal(finals, ref.finals_mont)
        assert cs == ref.checksum


def test_noalloc_rejects_one_table_more_than_the_largest_fit():
    """The largest-fit case above with an 11th table needs 33 MiB: rejected, nothing runs."""
    spec = get_field(32)
    enc = encode_expression([["t0", "t1"], ["t2", "t3", "t4"], ["t5"], ["t6", "t7"], ["t8", "t9", "t10"]])
    expr = api.CompiledExpression(enc, spec.modulus)
    small = api.generate_tables(spec, enc.num_vars, 4, [0] * enc.num_vars, seed=1)
    ctx = api.get_context(small.device)
    fld = api.get_device_field(spec, ctx.device)
    rc, *_ = _noalloc(ctx, fld, expr, 20, small, "sha3", spec.limbs, enc.degree, enc.num_vars)
    assert rc == _lib.SC_ERR_UNSUPPORTED and "scratch" in _lib.last_error()


def test_noalloc_rejects_proofs_beyond_its_scratch():
    # 9 Goldilocks tables of 2^24 entries need ~1.2 GB of fold buffers: rejected before any
    # launch, so the small table tensor passed here is never read.
    cfg = PLAIN_CONFIGS["plain_goldilocks"]
    spec = get_field(cfg.bit_width)
    enc = encode_expression(cfg.expression)
    expr = api.CompiledExpression(enc, spec.modulus)
    small = api.generate_tables(spec, enc.num_vars, 4, [0] * enc.num_vars, seed=1)
    ctx = api.get_context(small.device)
    fld = api.get_device_field(spec, ctx.device)
    rc, *_ = _noalloc(ctx, fld, expr, 24, small, "sha3", spec.limbs, enc.degree, enc.num_vars)
    assert rc == _lib.SC_ERR_UNSUPPORTED
    assert "scratch" in _lib.last_error() and "sc_prove" in _lib.last_error()
