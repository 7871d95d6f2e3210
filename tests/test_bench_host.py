"""bench.py's host-side helpers (CPU only): the fixed CPU sample and the busy-time union."""

from __future__ import annotations

import random

import pytest

import bench
from zkduel_b200.streams import batched_stream


def test_cpu_sample_is_fixed_and_stratified():
    """The same 32 proofs every run; every (field, size) stratum of the stream represented;
    about 1/16 of the stream's work (work of a proof ~ tables x 2^num_vars x limbs^2)."""
    a, b = bench.cpu_sample_specs(), bench.cpu_sample_specs()
    assert [s.index for s in a] == [s.index for s in b]
    assert len(a) == bench.STREAM_COUNT // bench.CPU_SAMPLE_STRIDE == 32
    assert {s.bit_width for s in a} == {64, 256}
    stream = batched_stream(bench.STREAM_COUNT, 0)
    for bw in (64, 256):
        sizes = sorted(s.num_vars for s in stream if s.bit_width == bw)
        picked = sorted(s.num_vars for s in a if s.bit_width == bw)
        assert picked[0] <= sizes[len(sizes) // 8] and picked[-1] >= sizes[-len(sizes) // 8]

    def work(s):
        return s.num_tables * (1 << s.num_vars) * (1 if s.bit_width == 64 else 16)

    frac = sum(work(s) for s in a) / sum(work(s) for s in stream)
    assert 1 / 24 < frac < 1 / 10
    assert [s.index for s in bench.cpu_sample_specs(3)] == [s.index for s in a[:3]]


@pytest.mark.parametrize("seed", range(5))
def test_busy_ms_is_the_union_of_intervals(seed):
    rng = random.Random(seed)
    iv = []
    for _ in range(40):
        a = rng.uniform(0, 100)
        iv.append((a, a + rng.uniform(0, 10)))
    # brute force on a fine grid
    step = 0.001
    covered = sum(step for k in range(int(115 / step)) if any(x <= k * step < y for x, y in iv))
    assert abs(bench.busy_ms(iv) - covered) < 0.05
    assert bench.busy_ms([]) == 0.0
    assert bench.busy_ms([(1.0, 2.0), (2.0, 3.0), (5.0, 6.0)]) == pytest.approx(3.0)
