"""The C oracle pinned against the Python oracle (CPU only)."""

from __future__ import annotations

import hashlib
import random

import numpy as np
import pytest

from helpers import oracle_tables
from oracle import c_oracle as C
from oracle import oracle as O
from zkduel_b200.configs import PLAIN_CONFIGS
from zkduel_b200.fields import from_limbs, get_field
from zkduel_b200.workloads import WORKLOADS


def test_sha3_matches_hashlib():
    rng = random.Random(0)
    for n in (0, 1, 21, 135, 136, 137, 281, 300):
        data = bytes(rng.randrange(256) for _ in range(n))
        assert C.sha3_256(data) == hashlib.sha3_256(data).digest()


@pytest.mark.parametrize("bw", [32, 64, 128, 256])
def test_generators_match(bw):
    f = get_field(bw)
    t = C.generate(f.modulus, f.limbs, [0, 1, 2 + 4], 8, 77)
    want = oracle_tables(["uniform", "bernoulli", "arith"], 77, 8, f, arith_index=[0, 0, 4])
    for k in range(3):
        assert [from_limbs(t[k, :, i].tolist()) for i in range(256)] == want[k]


CASES = [("poly_ab", 32, 5), ("vanilla_zerocheck_hp", 64, 5), ("poly_abcg_plus_deg", 256, 4),
         ("jellyfish_zerocheck_hp", 128, 3), ("witness_id_point_1", 64, 4), ("vanilla_permcheck_hp", 256, 3)]


@pytest.mark.parametrize("mode", ["sha3", "fixed", "explicit"])
@pytest.mark.parametrize("workload,bw,n", CASES, ids=[f"{w}-{b}-{n}" for w, b, n in CASES])
def test_c_prove_matches_python(workload, bw, n, mode):
    f = get_field(bw)
    expr = WORKLOADS[workload]
    terms, k = O.indexed_terms(expr)
    tables = C.generate(f.modulus, f.limbs, [0] * k, n, 5)
    canon = [[from_limbs(tables[kk, :, i].tolist()) for i in range(1 << n)] for kk in range(k)]
    ch = [random.Random(n).randrange(f.modulus) for _ in range(n)] if mode == "explicit" else None
    want = O.prove(terms, k, f.modulus, f.limbs, canon, mode, ch)
    got = C.prove(terms, k, f.modulus, f.limbs, tables, mode, ch, threads=3)
    dec = lambda v: f.decode_limbs(v.tolist())  # noqa: E731
    assert [[dec(v) for v in row] for row in got["round_polys"]] == want["round_polys"]
    assert [dec(v) for v in got["challenges"]] == want["challenges"]
    assert dec(got["finals"][0]) == want["final_claim"]
    assert [dec(v) for v in got["finals"][1:]] == want["final_values"]
    assert dec(got["claim0"]) == want["claim0"] and got["checksum"] == want["checksum"]


def test_c_prove_thread_count_invariant():
    cfg = PLAIN_CONFIGS["plain_goldilocks"]
    f = get_field(cfg.bit_width)
    terms, k = O.indexed_terms(cfg.expression)
    t = C.generate(f.modulus, f.limbs, [1 if x == "bernoulli" else 0 for x in cfg.table_kinds()], 12, 1)
    a = C.prove(terms, k, f.modulus, f.limbs, t, threads=1)
    b = C.prove(terms, k, f.modulus, f.limbs, t, threads=7)
    assert np.array_equal(a["round_polys"], b["round_polys"]) and a["checksum"] == b["checksum"]


@pytest.mark.parametrize("mode", ["sha3", "explicit"])
@pytest.mark.parametrize("workload,bw,n,kinds", [
    ("poly_ab", 32, 1, [0, 0]), ("poly_ab", 32, 9, [0, 1]), ("vanilla_zerocheck_hp", 64, 7, None),
    ("poly_abcg_plus_deg", 256, 5, None), ("poly_abc", 128, 6, [2 + 3, 0, 1])])
def test_seeded_prove_equals_table_prove(workload, bw, n, kinds, mode):
    """Round 0 generating its entries on the fly gives the proof of the generated tables."""
    f = get_field(bw)
    terms, k = O.indexed_terms(WORKLOADS[workload])
    kinds = kinds or [0] * k
    ch = [random.Random(n + 1).randrange(f.modulus) for _ in range(n)] if mode == "explicit" else None
    want = C.prove(terms, k, f.modulus, f.limbs, C.generate(f.modulus, f.limbs, kinds, n, 31), mode, ch, threads=2)
    got = C.prove_seeded(terms, k, f.modulus, f.limbs, n, kinds, 31, mode, ch, threads=3)
    for key in ("round_polys", "challenges", "finals", "claim0"):
        assert np.array_equal(got[key], want[key]), key
    assert got["checksum"] == want["checksum"]
