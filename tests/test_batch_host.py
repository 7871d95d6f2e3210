"""Host logic of the batched paths without a GPU: the degree classes and the chunking of
HostBatchProver (consecutive runs of about equal bytes, none empty)."""

from __future__ import annotations

import random

import pytest

from zkduel_b200.batch import chunk_bounds, degree_class


def test_degree_classes():
    assert [degree_class(d) for d in range(1, 8)] == [2, 2, 4, 4, 7, 7, 7]


@pytest.mark.parametrize("chunks", [1, 2, 3, 8, 16, 100])
def test_chunk_bounds_cover_everything_in_order(chunks):
    rng = random.Random(chunks)
    sizes = [rng.choice([8, 32]) * 2 ** rng.randint(10, 20) * rng.randint(2, 8) for _ in range(64)]
    b = chunk_bounds(sizes, chunks)
    assert b[0] == 0 and b[-1] == len(sizes)
    assert all(x < y for x, y in zip(b, b[1:]))  # no empty chunk
    assert 1 <= len(b) - 1 <= min(chunks, len(sizes))
    if chunks <= 8:  # about equal bytes: no chunk beyond twice its share plus one proof
        share = sum(sizes) / (len(b) - 1)
        assert all(sum(sizes[x:y]) <= 2 * share + max(sizes) for x, y in zip(b, b[1:]))


def test_chunk_bounds_small_cases():
    assert chunk_bounds([5], 4) == [0, 1]
    assert chunk_bounds([1, 1, 1, 1], 2) == [0, 2, 4]
    assert chunk_bounds([100, 1, 1, 1], 2) == [0, 1, 4]
