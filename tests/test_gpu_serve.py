"""Served proving (GPU): continuous batching gives every request the result it gets alone.

"Alone" is ``prove_device`` on ``generate_tables`` with the request's seed; the oracle pins
a few requests directly. The mixes force the cases continuous batching must get right:
requests joining while others run, rounds sliced over several launches (small chunks), a
budget that holds requests back, and both degree classes of the 128-bit stream at once.
"""

from __future__ import annotations

import random

import numpy as np
import pytest

from helpers import assert_proof_equals_oracle, oracle_tables
from oracle import oracle as O
from zkduel_b200 import api
from zkduel_b200.fields import get_field
from zkduel_b200.serve import ProofServer, replay
from zkduel_b200.streams import served_stream

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)

SPEC = get_field(128)


def _alone(spec, s, mode="sha3"):
    t = api.generate_tables(spec, s.num_tables, s.num_vars, [0] * s.num_tables, s.seed)
    return api.prove_device(t, s.expression, spec, s.num_vars, mode)


def _same(a, b):
    assert np.array_equal(a.round_polys_mont, b.round_polys_mont)
    assert np.array_equal(a.challenges_mont, b.challenges_mont)
    assert np.array_equal(a.finals_mont, b.finals_mont)
    assert np.array_equal(a.claim0_mont, b.claim0_mont)
    assert a.checksum == b.checksum


def _stream(count, lo, hi, seed):
    """served_stream's expressions with num_vars redrawn in [lo, hi] (test-sized)."""
    rng = random.Random(seed)
    out = []
    for r in served_stream(count, rate_per_s=1e9, seed=seed):
        s = r.spec
        out.append(type(s)(s.index, s.bit_width, rng.randint(lo, hi), s.seed, s.expression))
    return out


@pytest.mark.parametrize("chunk", [0, 1, 3])
def test_burst_equals_proofs_alone(chunk):
    specs = _stream(32, 1, 14, 5 + chunk)
    with ProofServer(SPEC, chunk_items=chunk, pairs_per_thread=1) as srv:
        ids = [srv.submit(s.expression, s.num_vars, s.seed) for s in specs]
        srv.drain(timeout_ms=120_000)
        for rid, s in zip(ids, specs):
            _same(srv.result(rid), _alone(SPEC, s))
        st = srv.stats()
        assert st["completed"] == len(specs) and st["failed"] == 0
        assert st["peak_inflight"] >= 2  # the burst overlapped
        if chunk:
            assert st["ticks"] > max(s.num_vars for s in specs)  # rounds were sliced


def test_requests_joining_while_others_run():
    big = _stream(1, 18, 18, 21)[0]
    small = _stream(12, 4, 10, 22)
    with ProofServer(SPEC, chunk_items=4) as srv:
        rb = srv.submit(big.expression, big.num_vars, big.seed)
        ids = []
        for s in small:  # submitted one by one while the large proof is on the GPU
            ids.append(srv.submit(s.expression, s.num_vars, s.seed))
            srv.wait(ids[-1], timeout_ms=60_000)
        srv.wait(rb, timeout_ms=60_000)
        _same(srv.result(rb), _alone(SPEC, big))
        for rid, s in zip(ids, small):
            _same(srv.result(rid), _alone(SPEC, s))
        tb = srv.times(rb)
        # the small requests finished while the large one was still in flight
        assert any(srv.times(r).done_s < tb.done_s for r in ids)


def test_large_requests_on_their_lane_with_small_ones():
    large = _stream(3, 20, 21, 71)
    small = _stream(16, 3, 12, 72)
    with ProofServer(SPEC) as srv:
        ids_l = [srv.submit(s.expression, s.num_vars, s.seed) for s in large]
        ids_s = [srv.submit(s.expression, s.num_vars, s.seed) for s in small]
        srv.drain(timeout_ms=120_000)
        for rid, s in zip(ids_l + ids_s, large + small):
            _same(srv.result(rid), _alone(SPEC, s))
        # the small requests overtook the large ones submitted before them
        last_large = max(srv.times(r).done_s for r in ids_l)
        assert max(srv.times(r).done_s for r in ids_s) < last_large
        assert srv.stats()["peak_inflight"] >= 4


def test_served_results_match_oracle():
    specs = _stream(5, 2, 6, 31)
    with ProofServer(SPEC) as srv:
        ids = [srv.submit(s.expression, s.num_vars, s.seed) for s in specs]
        srv.drain(timeout_ms=60_000)
        for rid, s in zip(ids, specs):
            terms, k = O.indexed_terms(s.expression)
            res = O.prove(terms, k, SPEC.modulus, SPEC.limbs, oracle_tables(["uniform"] * k, s.seed, s.num_vars, SPEC),
                          "sha3")
            assert_proof_equals_oracle(srv.result(rid), res, SPEC)


def test_budget_holds_requests_back():
    first = _stream(1, 12, 12, 41)[0]
    specs = [type(first)(i, 128, 12, 1000 + i, first.expression) for i in range(10)]  # equal footprints
    with ProofServer(SPEC) as probe:
        fp = probe.footprint(first.expression, 12)
    budget = 2 * fp + 1
    with ProofServer(SPEC, budget_bytes=budget) as srv:
        ids = [srv.submit(s.expression, s.num_vars, s.seed) for s in specs]
        srv.drain(timeout_ms=60_000)
        st = srv.stats()
        assert st["peak_footprint"] <= budget
        assert st["peak_inflight"] == 2  # the budget, not the burst, limited the overlap
        for rid, s in zip(ids, specs):
            _same(srv.result(rid), _alone(SPEC, s))
        # beyond the budget: rejected at submit
        with pytest.raises(ValueError):
            srv.submit(specs[0].expression, 20, 1)


def test_fifo_plain_policy_and_fixed_mode():
    specs = _stream(8, 3, 12, 51)
    with ProofServer(SPEC, policy="fifo_plain") as srv:
        ids = [srv.submit(s.expression, s.num_vars, s.seed) for s in specs]
        srv.drain(timeout_ms=60_000)
        for rid, s in zip(ids, specs):
            _same(srv.result(rid), _alone(SPEC, s))
        assert srv.stats()["peak_inflight"] == 1
    with ProofServer(SPEC) as srv:
        ids = [srv.submit(s.expression, s.num_vars, s.seed, challenge_mode="fixed") for s in specs]
        srv.drain(timeout_ms=60_000)
        for rid, s in zip(ids, specs):
            _same(srv.result(rid), _alone(SPEC, s, "fixed"))


def test_other_fields_and_errors():
    for bw in (32, 64, 256):
        spec = get_field(bw)
        specs = _stream(6, 2, 9, 60 + bw)
        with ProofServer(spec, max_tables=8) as srv:
            ids = [srv.submit(s.expression, s.num_vars, s.seed) for s in specs]
            srv.drain(timeout_ms=60_000)
            for rid, s in zip(ids, specs):
                _same(srv.result(rid), _alone(spec, s))
    with ProofServer(SPEC, max_tables=2) as srv:
        with pytest.raises(ValueError):
            srv.submit(((1, ("a", "b", "c")),), 4, 1)  # three tables > max_tables
        with pytest.raises(ValueError):
            srv.submit(((1, ("a", "b")),), 4, 1, challenge_mode="explicit")
        rid = srv.submit(((1, ("a", "b")),), 18, 3)
        try:
            srv.result(rid)  # usually still pending here; a finished one reads normally
        except RuntimeError as e:
            assert "has not completed" in str(e)
        srv.wait(rid, timeout_ms=60_000)
        srv.result(rid)
        srv.release(rid)
        with pytest.raises(ValueError):
            srv.result(rid)


def test_replay_reports_latencies():
    reqs = served_stream(40, rate_per_s=2000.0, seed=3, min_vars=6, max_vars=12)
    with ProofServer(SPEC) as srv:
        rep, results = replay(srv, reqs, keep_results=True)
    s = rep.summary()
    assert s["requests"] == 40 and s["p50_ms"] > 0 and s["p99_ms"] >= s["p50_ms"]
    for i in (0, 17, 39):
        _same(results[i], _alone(SPEC, reqs[i].spec))
