"""Suspending and resuming proofs (GPU): a proof stopped at any round boundary and continued
-- on the plain path, after a round trip through bytes, or by a server -- equals the
uninterrupted proof bit for bit; transcripts bind to their field, expression and tables.
"""

from __future__ import annotations

import random
import time

import numpy as np
import pytest

from zkduel_b200 import _lib, api
from zkduel_b200 import transcript as tr
from zkduel_b200.fields import get_field
from zkduel_b200.serve import ProofServer

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)


def _same(a, b):
    assert np.array_equal(a.round_polys_mont, b.round_polys_mont)
    assert np.array_equal(a.challenges_mont, b.challenges_mont)
    assert np.array_equal(a.finals_mont, b.finals_mont)
    assert np.array_equal(a.claim0_mont, b.claim0_mont)
    assert a.checksum == b.checksum


ZEROCHECK = ((1, ("qL", "w1", "fz1")), (1, ("qR", "w2", "fz1")), (1, ("qM", "w1", "w2", "fz1")),
             (-1, ("qO", "w3", "fz1")), (1, ("qC", "fz1")))
CASES = [
    (32, ((1, ("a", "b")),), 14),                              # round 1 takes g(1) from the claim
    (64, ZEROCHECK, 12),                                       # compile-time zerocheck shape
    (64, ((1, ("x", "y")),), 16),                              # rounds 1-3 from the claim
    (128, ((1, ("a", "b", "c")), (3, ("d", "e")), (-1, ("a",))), 9),
    (128, ((2, ("a", "b")),), 13),
    (256, ((1, ("a", "b", "c", "g")), (1, ("d", "e", "g"))), 8),  # compile-time g(abc + de) shape
    (256, ((1, ("a", "b")), (3, ("c",))), 10),                 # point-parallel 8-limb kernel
]


def _tables(spec, expr, n, seed, kinds=None):
    k = api.encode_expression(expr).num_vars
    kinds = [0] * k if kinds is None else kinds
    return api.generate_tables(spec, k, n, kinds, seed), kinds


@pytest.mark.parametrize("bw,expr,n", CASES)
def test_resume_at_every_boundary_equals_whole_proof(bw, expr, n):
    spec = get_field(bw)
    t, _ = _tables(spec, expr, n, 300 + n + bw)
    whole = api.prove_device(t, expr, spec, n, "sha3")
    for j in sorted({1, 2, n // 2, n - 1}):
        a = tr.prove_rounds(t, expr, spec, j, tr.start(expr, spec, n))
        assert a.rounds_done == j and not a.complete
        b = tr.prove_rounds(t, expr, spec, n, tr.Transcript.from_bytes(a.to_bytes()))
        assert b.complete
        _same(tr.result(b, expr, spec), whole)
    # chained segments, the whole proof in one segment
    t2 = tr.start(expr, spec, n)
    for stop in sorted({1, min(3, n), min(7, n), n}):
        t2 = tr.prove_rounds(t, expr, spec, stop, t2)
    _same(tr.result(t2, expr, spec), whole)
    _same(tr.result(tr.prove_rounds(t, expr, spec, n, tr.start(expr, spec, n)), expr, spec), whole)


def test_resume_large_proof_and_file_round_trip(tmp_path):
    spec = get_field(64)
    expr = ((1, ("a", "b", "c")),)
    n = 20
    t, _ = _tables(spec, expr, n, 77)
    whole = api.prove_device(t, expr, spec, n, "sha3")
    a = tr.prove_rounds(t, expr, spec, 10, tr.start(expr, spec, n))
    a.save(tmp_path / "proof.sctr")
    b = tr.prove_rounds(t, expr, spec, n, tr.Transcript.load(tmp_path / "proof.sctr"))
    _same(tr.result(b, expr, spec), whole)


def test_fixed_and_explicit_modes():
    spec = get_field(128)
    expr = ((1, ("a", "b")), (5, ("c",)))
    n = 11
    t, _ = _tables(spec, expr, n, 9)
    whole = api.prove_device(t, expr, spec, n, "fixed")
    a = tr.prove_rounds(t, expr, spec, 4, tr.start(expr, spec, n, "fixed"))
    _same(tr.result(tr.prove_rounds(t, expr, spec, n, a), expr, spec), whole)
    rng = random.Random(4)
    ch = [rng.randrange(spec.modulus) for _ in range(n)]
    whole = api.prove_device(t, expr, spec, n, "explicit", ch)
    a = tr.prove_rounds(t, expr, spec, 6, tr.start(expr, spec, n, "explicit"), ch)
    _same(tr.result(tr.prove_rounds(t, expr, spec, n, a, ch), expr, spec), whole)
    with pytest.raises(ValueError, match="differ"):  # the challenges already used must not change
        tr.prove_rounds(t, expr, spec, n, a, [ch[0] ^ 1] + ch[1:])


def test_transcripts_bind_to_field_expression_and_shape():
    spec = get_field(64)
    expr = ((1, ("a", "b")),)
    n = 8
    t, _ = _tables(spec, expr, n, 3)
    a = tr.prove_rounds(t, expr, spec, 3, tr.start(expr, spec, n))
    with pytest.raises(ValueError, match="another expression"):
        tr.prove_rounds(t, ((2, ("a", "b")),), spec, n, a)
    t32, _ = _tables(get_field(32), expr, n, 3)
    with pytest.raises(ValueError, match="another field"):
        tr.prove_rounds(t32, expr, get_field(32), n, a)
    with pytest.raises(ValueError, match="stop_round"):
        tr.prove_rounds(t, expr, spec, 3, a)
    with pytest.raises(ValueError):
        tr.Transcript(a.words[:-1])  # truncated
    with pytest.raises(_lib.SumcheckError, match="rounds"):
        tr.result(a, expr, spec)  # not complete
    done = tr.prove_rounds(t, expr, spec, n, a)
    with pytest.raises(ValueError, match="complete"):
        tr.prove_rounds(t, expr, spec, n, done)


# ---------------------------------------------------------------------------- served


def _alone(spec, expr, n, seed, mode="sha3"):
    t, _ = _tables(spec, expr, n, seed)
    return api.prove_device(t, expr, spec, n, mode)


SERVE_EXPRS = [((1, ("a", "b", "c")), (3, ("d",))), ((1, ("a", "b")),), ((1, ("a", "b", "c", "d", "e")), (2, ("b",)))]


def test_plain_transcripts_resume_on_a_server():
    spec = get_field(128)
    jobs = []
    for i, (expr, n, j) in enumerate([(SERVE_EXPRS[0], 12, 5), (SERVE_EXPRS[1], 21, 1), (SERVE_EXPRS[1], 19, 9),
                                      (SERVE_EXPRS[2], 9, 8), (SERVE_EXPRS[0], 14, 2)]):
        seed = 900 + i
        t, kinds = _tables(spec, expr, n, seed)
        a = tr.prove_rounds(t, expr, spec, j, tr.start(expr, spec, n, tables_tag=tr.tables_tag(kinds, seed)))
        jobs.append((expr, n, seed, kinds, a))
    for policy in ("continuous", "fifo_plain"):
        with ProofServer(spec, policy=policy) as srv:
            ids = [srv.submit(e, n, s, k, resume=a) for e, n, s, k, a in jobs]
            srv.drain(timeout_ms=120_000)
            for rid, (e, n, s, _k, _a) in zip(ids, jobs):
                _same(srv.result(rid), _alone(spec, e, n, s))


def _suspend_run(spec, specs, sleep_s, **server_kw):
    with ProofServer(spec, **server_kw) as srv:
        ids = [srv.submit(e, n, s) for e, n, s in specs]
        time.sleep(sleep_s)
        srv.suspend()
        srv.drain(timeout_ms=120_000)
        out = []
        for rid, job in zip(ids, specs):
            st = srv.wait(rid, timeout_ms=1000)
            out.append((job, st, srv.transcript(rid) if st == "suspended" else srv.result(rid)))
        stats = srv.stats()
    assert stats["suspended"] == sum(1 for _j, st, _x in out if st == "suspended")
    return out


def test_suspend_mid_proof_and_resume_anywhere():
    spec = get_field(128)
    specs = [(SERVE_EXPRS[i % 3], 17 if i < 4 else 8 + i, 50 + i) for i in range(10)]
    mid = []
    for attempt, sleep_s in enumerate((0.002, 0.006, 0.015)):
        out = _suspend_run(spec, specs, sleep_s, chunk_items=1, pairs_per_thread=1)
        resumed = []
        for (e, n, s), st, x in out:
            if st == "done":
                _same(x, _alone(spec, e, n, s))
                continue
            assert x.num_rounds == n and 0 <= x.rounds_done < n
            assert x.tables_tag == tr.tables_tag([0] * api.encode_expression(e).num_vars, s)
            resumed.append(((e, n, s), x))
            if 0 < x.rounds_done:
                mid.append(x)
        # half finish on another server, half on the plain path
        with ProofServer(spec) as srv:
            ids = [(srv.submit(e, n, s, resume=x), (e, n, s)) for (e, n, s), x in resumed[::2]]
            srv.drain(timeout_ms=120_000)
            for rid, (e, n, s) in ids:
                _same(srv.result(rid), _alone(spec, e, n, s))
        for (e, n, s), x in resumed[1::2]:
            t, _ = _tables(spec, e, n, s)
            _same(tr.result(tr.prove_rounds(t, e, spec, n, x), e, spec), _alone(spec, e, n, s))
        if mid:
            break
    assert mid, "no request was suspended between rounds"


def test_suspend_queued_requests_and_errors():
    spec = get_field(64)
    expr = SERVE_EXPRS[0]
    specs = [(expr, 10, 70 + i) for i in range(6)]
    out = _suspend_run(spec, specs, 0.0, policy="fifo_plain")
    assert any(st == "suspended" for _j, st, _x in out)
    with ProofServer(spec) as srv:
        for (e, n, s), st, x in out:
            if st != "suspended":
                continue
            assert x.rounds_done == 0  # FIFO suspends only requests not started
            with pytest.raises(ValueError, match="other tables"):
                srv.submit(e, n, s + 1, resume=x)
            rid = srv.submit(e, n, s, resume=x)
            assert srv.wait(rid, timeout_ms=60_000) == "done"
            _same(srv.result(rid), _alone(spec, e, n, s))
            with pytest.raises(ValueError, match="not suspended"):
                srv.transcript(rid)


@pytest.mark.parametrize("bw,expr,n,j", [
    (64, ((1, ("x", "y")),), 16, 2),          # generic 2-limb kernel
    (64, ZEROCHECK, 14, 1),                   # compile-time zerocheck shape
    (256, ((1, ("a", "b")), (3, ("c",))), 14, 1),  # point-parallel 8-limb kernel
])
def test_resume_checks_the_recorded_claim_against_the_tables(bw, expr, n, j):
    """A resumed segment whose first round would take g(1) from the recorded claim instead
    evaluates g(1) and checks g(0) + g(1) against that claim on the device: the untouched
    transcript resumes to the whole proof; an altered claim, or tables other than the ones
    the recorded rounds were proved on, fail with the device status (kStatusClaim = 1)."""
    spec = get_field(bw)
    t, _ = _tables(spec, expr, n, 900 + n)
    whole = api.prove_device(t, expr, spec, n, "sha3")
    a = tr.prove_rounds(t, expr, spec, j, tr.start(expr, spec, n))
    _same(tr.result(tr.prove_rounds(t, expr, spec, n, a), expr, spec), whole)
    bad = a.words.copy()
    bad[-spec.limbs] ^= 1  # the claim is the transcript's last L words
    with pytest.raises(_lib.SumcheckError, match="device status 1"):
        tr.prove_rounds(t, expr, spec, n, tr.Transcript(bad))
    other, _ = _tables(spec, expr, n, 901 + n)
    with pytest.raises(_lib.SumcheckError, match="device status 1"):
        tr.prove_rounds(other, expr, spec, n, a)
    # the context proves normally afterwards
    _same(api.prove_device(t, expr, spec, n, "sha3"), whole)
