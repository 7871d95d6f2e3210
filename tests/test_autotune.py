"""Autotuner table logic (CPU): ranges, JSON round trip, the synthetic expressions' classes."""

from __future__ import annotations

import random

from zkduel_b200 import autotune as A
from zkduel_b200.batch import degree_class


def test_ranges_cover_every_num_vars():
    for n in range(1, 41):
        r = A._range_of(n)
        lo, hi = A.RANGES[r]
        assert lo <= n <= hi
    assert A._range_of(12) == 0 and A._range_of(13) == 1 and A._range_of(18) == 3


def test_sample_ranges_fall_in_their_ranges():
    for (lo, hi), (slo, shi) in zip(A.RANGES, A.SAMPLE_RANGES):
        assert lo <= slo <= shi <= hi


def test_table_round_trips_through_json():
    t = A.TuneTable()
    t.threads_by[(8, 7)] = 128
    t.threads_by[(2, 2)] = 64
    t.ppt_by[(8, 7, 3)] = 16
    t.ppt_by[(2, 2, 0)] = 1
    t.timings["x"] = 1.5
    u = A.TuneTable.from_json(t.to_json())
    assert u.threads_by == t.threads_by and u.ppt_by == t.ppt_by and u.timings == t.timings
    assert u.threads(8, 7) == 128 and u.threads(4, 4) == 0
    assert u.pairs_per_thread(8, 7, 20) == 16 and u.pairs_per_thread(2, 2, 5) == 1
    assert u.pairs_per_thread(2, 4, 5) == 0  # missing: default


def test_synthetic_expressions_land_in_their_class():
    rng = random.Random(3)
    for dc in A.CLASSES:
        for _ in range(200):
            e = A._expression(rng, dc)
            assert degree_class(max(len(f) for _c, f in e)) == dc
            assert all(len(set(f)) == len(f) for _c, f in e)
