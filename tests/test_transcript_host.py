"""Transcripts without a GPU: the header the library parses, the tables tag, and the byte
round trip of ``zkduel_b200.Transcript`` (the proving and resuming is in the GPU tests)."""

from __future__ import annotations

import numpy as np
import pytest

from zkduel_b200 import _lib
from zkduel_b200.transcript import HEADER_WORDS, MAGIC, Transcript, tables_tag


def _blob(L=2, n=6, K=3, d=3, mode=0, done=2):
    state = 4 + L * (9 * n + K + 3)
    w = np.zeros(HEADER_WORDS + state, dtype=np.uint32)
    w[:8] = [MAGIC, HEADER_WORDS, L, n, K, d, mode, done]
    w[8:14] = [1, 2, 3, 4, 0xDEADBEEF, 7]  # digests and tag (not checked without a proof)
    w[14] = state
    w[HEADER_WORDS + 4:] = np.arange(state - 4, dtype=np.uint32)
    return w


def test_header_parsed_by_the_library():
    t = Transcript(_blob())
    assert (t.num_rounds, t.rounds_done, t.challenge_mode, t.complete) == (6, 2, "sha3", False)
    assert t.tables_tag == 0x7_DEADBEEF
    assert Transcript(_blob(done=6, mode=1)).complete and Transcript(_blob(mode=1)).challenge_mode == "fixed"


@pytest.mark.parametrize("bad", [
    lambda w: w.__setitem__(0, 0),            # magic
    lambda w: w.__setitem__(2, 3),            # limbs
    lambda w: w.__setitem__(7, 7),            # rounds done > rounds
    lambda w: w.__setitem__(5, 8),            # degree > 7
    lambda w: w.__setitem__(14, 5),           # state size disagrees
])
def test_malformed_headers_rejected(bad):
    w = _blob()
    bad(w)
    with pytest.raises(ValueError):
        Transcript(w)


def test_truncated_rejected_and_bytes_round_trip(tmp_path):
    w = _blob()
    with pytest.raises(ValueError, match="shorter"):
        Transcript(w[:-1])
    t = Transcript(w)
    b = t.to_bytes()
    assert len(b) == 4 * w.size and b[:4] == MAGIC.to_bytes(4, "little")
    assert np.array_equal(Transcript.from_bytes(b).words, w)
    t.save(tmp_path / "t.sctr")
    assert np.array_equal(Transcript.load(tmp_path / "t.sctr").words, w)


def test_tables_tag():
    a = tables_tag([0, 1, 0], 5)
    assert a == tables_tag([0, 1, 0], 5)
    assert len({a, tables_tag([0, 1, 0], 6), tables_tag([0, 0, 0], 5), tables_tag([0, 1], 5)}) == 4
    with pytest.raises(ValueError):
        tables_tag([], 5)
    assert _lib.SC_SUSPENDED == 9
