"""Batched proving (GPU): every proof of a batch equals the same proof proved alone."""

from __future__ import annotations

import random

import numpy as np
import pytest

from helpers import assert_proof_equals_oracle, oracle_tables
from oracle import oracle as O
from zkduel_b200 import api
from zkduel_b200.batch import BatchProver
from zkduel_b200.fields import get_field
from zkduel_b200.streams import batched_stream

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)


def _tables(spec, s):
    return api.generate_tables(spec, s.num_tables, s.num_vars, [0] * s.num_tables, s.seed)


def _same(a, b):
    assert np.array_equal(a.round_polys_mont, b.round_polys_mont)
    assert np.array_equal(a.challenges_mont, b.challenges_mont)
    assert np.array_equal(a.finals_mont, b.finals_mont)
    assert np.array_equal(a.claim0_mont, b.claim0_mont)
    assert a.checksum == b.checksum


def _mixed(count, lo, hi, seed):
    rng = random.Random(seed)
    out = []
    for s in batched_stream(count, seed):
        n = rng.randint(lo, hi)
        out.append(type(s)(s.index, s.bit_width, n, s.seed, s.expression))
    return out


@pytest.mark.parametrize("tile", [None, {2: (64, 1), 8: (32, 1)}, {2: (256, 8), 8: (128, 4)}])
def test_small_mixed_batch_equals_single_proofs(tile):
    specs = _mixed(40, 1, 12, 7)
    items = [(s.expression, s.bit_width, s.num_vars, _tables(get_field(s.bit_width), s)) for s in specs]
    bp = BatchProver(items, tile=tile)
    bp.run()
    for i, s in enumerate(specs):
        spec = get_field(s.bit_width)
        alone = api.prove_device(items[i][3], s.expression, spec, s.num_vars, "sha3")
        _same(bp.result(i), alone)


def test_batch_matches_oracle():
    specs = _mixed(6, 2, 6, 3)
    items = [(s.expression, s.bit_width, s.num_vars, _tables(get_field(s.bit_width), s)) for s in specs]
    bp = BatchProver(items)
    bp.run()
    for i, s in enumerate(specs):
        spec = get_field(s.bit_width)
        terms, k = O.indexed_terms(s.expression)
        res = O.prove(terms, k, spec.modulus, spec.limbs, oracle_tables(["uniform"] * k, s.seed, s.num_vars, spec), "sha3")
        assert_proof_equals_oracle(bp.result(i), res, spec)


def test_stream_batch_replays_identically():
    specs = batched_stream(48, 11)
    items = [(s.expression, s.bit_width, s.num_vars, _tables(get_field(s.bit_width), s)) for s in specs]
    bp = BatchProver(items)
    bp.run()
    first = bp.results()
    bp.run()
    for a, b in zip(first, bp.results()):
        _same(a, b)
    for i in (0, 7, 23, 47):
        s = specs[i]
        _same(first[i], api.prove_device(items[i][3], s.expression, get_field(s.bit_width), s.num_vars, "sha3"))
    classes = bp.tick_times()
    assert sorted(i for c in classes for i in c["proofs"]) == list(range(len(specs)))
    for c in classes:
        assert len(c["ms"]) == max(specs[i].num_vars for i in c["proofs"])
        assert all(x > 0 for x in c["ms"])
        assert all(specs[i].degree <= c["degree_class"] for i in c["proofs"])


def test_fixed_mode_and_rejects_explicit():
    specs = _mixed(5, 3, 5, 1)
    items = [(s.expression, s.bit_width, s.num_vars, _tables(get_field(s.bit_width), s)) for s in specs]
    bp = BatchProver(items, challenge_mode="fixed")
    bp.run()
    for i, s in enumerate(specs):
        _same(bp.result(i), api.prove_device(items[i][3], s.expression, get_field(s.bit_width), s.num_vars, "fixed"))
    with pytest.raises(ValueError):
        BatchProver(items, challenge_mode="explicit")


def test_tuned_tiles_are_bit_identical():
    from zkduel_b200.autotune import TuneTable

    specs = _mixed(30, 2, 12, 13)
    items = [(s.expression, s.bit_width, s.num_vars, _tables(get_field(s.bit_width), s)) for s in specs]
    rng = random.Random(5)
    tune = TuneTable()
    for L in (2, 8):
        for dc in (2, 4, 7):
            tune.threads_by[(L, dc)] = rng.choice([32, 64, 128, 256])
            for r in range(4):
                tune.ppt_by[(L, dc, r)] = rng.choice([1, 2, 3, 8, 16])
    bp = BatchProver(items, tuning=tune)
    bp.run()
    for i, s in enumerate(specs):
        _same(bp.result(i), api.prove_device(items[i][3], s.expression, get_field(s.bit_width), s.num_vars, "sha3"))


def test_autotune_fills_its_table(tmp_path):
    from zkduel_b200 import autotune as A

    t = A.load_or_tune((64,), cache=tmp_path / "tune.json", proofs_per_range=2, reps=1)
    assert all(t.threads(2, dc) in A.THREADS for dc in A.CLASSES)
    assert all(t.pairs_per_thread(2, dc, n) in A.PAIRS_PER_THREAD for dc in A.CLASSES for n in (10, 14, 17, 19))
    again = A.load_or_tune((64,), cache=tmp_path / "tune.json")  # from the cache: no timing
    assert again.threads_by == t.threads_by and again.ppt_by == t.ppt_by


def test_tune_for_keeps_results_and_reports_timings():
    from zkduel_b200.autotune import tune_for

    specs = _mixed(16, 4, 12, 17)
    items = [(s.expression, s.bit_width, s.num_vars, _tables(get_field(s.bit_width), s)) for s in specs]
    t = tune_for(items, reps=1, ppt_candidates=(1, 4))
    assert t.timings["best"] <= t.timings["start"]
    bp = BatchProver(items, tuning=t)
    bp.run()
    for i, s in enumerate(specs):
        _same(bp.result(i), api.prove_device(items[i][3], s.expression, get_field(s.bit_width), s.num_vars, "sha3"))


@pytest.mark.parametrize("chunks", [1, 3, 7])
def test_host_batch_prover_equals_single_proofs(chunks):
    from zkduel_b200.batch import HostBatchProver

    specs = _mixed(30, 2, 14, 21)
    dev = [_tables(get_field(s.bit_width), s) for s in specs]
    host = [torch.from_numpy(api.download_tables(t, get_field(s.bit_width)).view(np.int32)).pin_memory()
            for s, t in zip(specs, dev)]
    hb = HostBatchProver([(s.expression, s.bit_width, s.num_vars) for s in specs], host, chunks=chunks)
    assert len(hb.chunks) == min(chunks, len(specs))
    for _ in range(2):  # the second run reuses the device tables
        res = hb.run()
        for s, t, p in zip(specs, dev, res):
            _same(p, api.prove_device(t, s.expression, get_field(s.bit_width), s.num_vars, "sha3"))
    hb.close()
