"""Parity of the CUDA prover with the oracle and the reference's golden data (GPU).

Everything goes through the C ABI (libsumcheck_b200.so via ctypes). Integer work, so the
bar is bit-exact equality everywhere: round polynomials, challenges, final claims and
checksum.
"""

from __future__ import annotations

import random

import numpy as np
import pytest

from conftest import load_jsonl
from helpers import assert_proof_equals_oracle, check_transcript_and_identities, oracle_tables
from oracle import oracle as O
from zkduel_b200 import api
from zkduel_b200.configs import PLAIN_CONFIGS
from zkduel_b200.fields import FIELD_SPECS, from_limbs, get_field, stress_value
from zkduel_b200.workloads import WORKLOADS, get_kernel_workload

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)

REGISTRY = load_jsonl("registry_checksums.jsonl")
OUTPUTS = load_jsonl("reference_outputs.jsonl")


@pytest.mark.parametrize("bw", [32, 64, 128, 256])
def test_device_arithmetic_matches_bigint(bw):
    import ctypes

    from zkduel_b200 import _lib

    spec = get_field(bw)
    p, L = spec.modulus, spec.limbs
    rng = random.Random(bw)
    n = 4096
    a = [stress_value(p, L, rng) for _ in range(n)]
    b = [stress_value(p, L, rng) for _ in range(n)]
    to_dev = lambda xs: torch.tensor(np.array([[(x >> (32 * i)) & 0xFFFFFFFF for i in range(L)] for x in xs],
                                              dtype=np.uint32).view(np.int32), device="cuda")
    da, db = to_dev(a), to_dev(b)
    out = torch.empty_like(da)
    ctx = api.get_context()
    fld = api.get_device_field(spec, ctx.device)
    r_inv = pow(1 << (32 * L), -1, p)
    for op, want in ((0, lambda x, y: x * y * r_inv % p), (1, lambda x, y: (x + y) % p), (2, lambda x, y: (x - y) % p)):
        rc = _lib.load().sc_field_apply(ctx.handle, fld.handle, op, ctypes.c_void_p(da.data_ptr()),
                                        ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(out.data_ptr()), n)
        _lib.check(rc, "sc_field_apply")
        got = out.cpu().numpy().view(np.uint32)
        for i in range(n):
            assert from_limbs(got[i].tolist()) == want(a[i], b[i]), (op, hex(a[i]), hex(b[i]))


@pytest.mark.parametrize("bw", [32, 64, 128, 256])
def test_generated_tables_match_oracle(bw):
    spec = get_field(bw)
    n = 10
    kinds = [api._lib.SC_TABLE_UNIFORM, api._lib.SC_TABLE_BERNOULLI, api._lib.SC_TABLE_ARITH + 5]
    t = api.generate_tables(spec, 3, n, kinds, seed=12345)
    got = api.download_tables(t, spec)
    want = oracle_tables(["uniform", "bernoulli", "arith"], 12345, n, spec, arith_index=[0, 0, 5])
    for k in range(3):
        vals = [from_limbs([int(got[k, l, i]) for l in range(spec.limbs)]) for i in range(1 << n)]
        assert vals == want[k], k


def _rid(r):
    return f"{r['workload']}-bw{r['bit_width']}-r{r['rounds']}-{r['challenge_mode']}"


@pytest.mark.parametrize("rec", REGISTRY, ids=[_rid(r) for r in REGISTRY])
def test_registry_golden_checksum(rec):
    """The reference's own golden checksums (all 32 workloads x 4 widths x 3 cases)."""
    w = get_kernel_workload(rec["workload"])
    proof = api.prove(w.expression, rec["bit_width"], rec["rounds"], rec["seed"],
                      table_kinds=["arith"] * w.num_vars, arith_index=w.table_index(),
                      challenge_mode=rec["challenge_mode"])
    assert rec["runs"] * proof.checksum == rec["checksum_x2"]


@pytest.mark.parametrize("case", OUTPUTS, ids=[o["case"] for o in OUTPUTS])
def test_sumcheck_api_matches_reference_outputs(case):
    """zkduel.sumcheck's call and return, checked against the reference's own outputs."""
    claim, evals = api.sumcheck(case["tables"], q=case["q"], expression=WORKLOADS[case["workload"]],
                                challenges=case["challenges"], num_rounds=case["num_rounds"],
                                bit_width=case["bit_width"])
    assert claim == case["claim0"]
    assert [[int(x) for x in row] for row in evals.tolist()] == case["evals"]


SHAPES = [
    ("poly_ab", 32), ("vanilla_zerocheck_hp", 64), ("poly_abcg_plus_deg", 256), ("jellyfish_zerocheck_hp", 128),
    ("poly_aabbc", 64), ("vanilla_permcheck_hp", 256), ("witness_non_id_point", 32), ("poly_a", 128),
]


@pytest.mark.parametrize("n", [1, 2, 3, 7])
@pytest.mark.parametrize("workload,bw", SHAPES, ids=[f"{w}-{b}" for w, b in SHAPES])
def test_prove_matches_oracle(workload, bw, n):
    spec = get_field(bw)
    expr = WORKLOADS[workload]
    terms, k = O.indexed_terms(expr)
    kinds = ["uniform"] * k
    if workload == "vanilla_zerocheck_hp":
        kinds = PLAIN_CONFIGS["plain_goldilocks"].table_kinds()
    proof = api.prove(expr, bw, n, seed=1000 + n, table_kinds=kinds)
    res = O.prove(terms, k, spec.modulus, spec.limbs, oracle_tables(kinds, 1000 + n, n, spec), "sha3")
    assert_proof_equals_oracle(proof, res, spec)


@pytest.mark.parametrize("mode", ["fixed", "explicit"])
def test_challenge_modes_match_oracle(mode):
    spec = get_field(64)
    expr = WORKLOADS["vanilla_zerocheck_hp"]
    terms, k = O.indexed_terms(expr)
    n = 6
    rng = random.Random(5)
    ch = [rng.randrange(spec.modulus) for _ in range(n)] if mode == "explicit" else None
    proof = api.prove(expr, 64, n, seed=9, challenge_mode=mode, challenges=ch)
    res = O.prove(terms, k, spec.modulus, spec.limbs, oracle_tables(["uniform"] * k, 9, n, spec), mode, ch)
    assert_proof_equals_oracle(proof, res, spec)


@pytest.mark.parametrize("name", ["plain_p32", "plain_goldilocks", "plain_bls"])
def test_multi_block_sizes_match_oracle(name):
    """Sizes where the grid has many blocks and threads loop (grid-stride)."""
    cfg = PLAIN_CONFIGS[name]
    n = {"plain_p32": 13, "plain_goldilocks": 9, "plain_bls": 8}[name]
    spec = get_field(cfg.bit_width)
    terms, k = O.indexed_terms(cfg.expression)
    kinds = cfg.table_kinds()
    proof = api.prove(cfg.expression, cfg.bit_width, n, seed=3, table_kinds=kinds)
    res = O.prove(terms, k, spec.modulus, spec.limbs, oracle_tables(kinds, 3, n, spec), "sha3")
    assert_proof_equals_oracle(proof, res, spec)


def _kind_codes(kinds):
    return [1 if x == "bernoulli" else 0 for x in kinds]


@pytest.mark.parametrize("name", ["plain_p32", "plain_goldilocks", "plain_bls"])
def test_full_size_config_matches_c_oracle(name):
    """Each plain configuration at its full size (n = 16 / 24 / 22), bit-exact against the C
    oracle: round polynomials, challenges, final claim and every f_k(r), claim0, checksum.
    Then the verifier-side identities, with f_k(r) taken from the oracle's fold of the
    tables (not from the proof), and determinism over two runs."""
    from oracle import c_oracle as C

    cfg = PLAIN_CONFIGS[name]
    spec = get_field(cfg.bit_width)
    terms, k = O.indexed_terms(cfg.expression)
    a = api.prove(cfg.expression, cfg.bit_width, cfg.num_vars, cfg.seed, table_kinds=cfg.table_kinds())
    res = C.prove_seeded(terms, k, spec.modulus, spec.limbs, cfg.num_vars, _kind_codes(cfg.table_kinds()), cfg.seed)
    assert np.array_equal(a.round_polys_mont, res["round_polys"])
    assert np.array_equal(a.challenges_mont, res["challenges"])
    assert np.array_equal(a.finals_mont, res["finals"])
    assert np.array_equal(a.claim0_mont, res["claim0"])
    assert a.checksum == res["checksum"]
    host_finals = [spec.decode_limbs([int(x) for x in v]) for v in res["finals"][1:]]
    check_transcript_and_identities(a, terms, spec, final_values=host_finals)
    b = api.prove(cfg.expression, cfg.bit_width, cfg.num_vars, cfg.seed, table_kinds=cfg.table_kinds())
    assert np.array_equal(a.round_polys_mont, b.round_polys_mont) and a.checksum == b.checksum
    assert np.array_equal(a.finals_mont, b.finals_mont)


def test_tables_past_2_31_entries_match_c_oracle():
    """a * b over 2^32 - 5 at n = 31: 2^31 entries per table, so table 1's plane starts at
    entry 2^31 and the last index of every plane is 2^31 - 1. 32-bit indexing past 2^31
    elements was the reference's one recorded bug (fixed by size_t indexing,
    cuda/src/field_sumcheck.cu:596,618). Everything is compared with the C oracle, which
    generates round 0's entries on the fly (host memory for the folded half only)."""
    from oracle import c_oracle as C

    n, seed = 31, 7
    expr = WORKLOADS["poly_ab"]
    spec = get_field(32)
    terms, k = O.indexed_terms(expr)
    free, _total = torch.cuda.mem_get_info()
    need = 2 * (1 << n) * 4 * 7 // 4  # tables + fold buffers
    if free < need + (4 << 30):
        pytest.skip(f"needs {need / 2**30:.0f} GiB of device memory")
    proof = api.prove(expr, 32, n, seed, table_kinds=["uniform", "uniform"])
    torch.cuda.empty_cache()
    res = C.prove_seeded(terms, k, spec.modulus, spec.limbs, n, [0, 0], seed)
    assert np.array_equal(proof.round_polys_mont, res["round_polys"])
    assert np.array_equal(proof.challenges_mont, res["challenges"])
    assert np.array_equal(proof.finals_mont, res["finals"])
    assert proof.checksum == res["checksum"]


def test_plain_p32_full_size_matches_oracle():
    """The config small enough for the Python oracle at full size: bit-exact everything."""
    cfg = PLAIN_CONFIGS["plain_p32"]
    spec = get_field(cfg.bit_width)
    terms, k = O.indexed_terms(cfg.expression)
    proof = api.prove(cfg.expression, cfg.bit_width, cfg.num_vars, cfg.seed, table_kinds=cfg.table_kinds())
    res = O.prove(terms, k, spec.modulus, spec.limbs, oracle_tables(cfg.table_kinds(), cfg.seed, cfg.num_vars, spec), "sha3")
    assert_proof_equals_oracle(proof, res, spec)


def test_sumcheck_accepts_short_challenge_list_and_rejects_bad_input():
    spec = FIELD_SPECS[256]
    expr = WORKLOADS["poly_ab"]
    tables = {"a": [1, 2, 3, 4], "b": [5, 6, 7, 8]}
    claim, evals = api.sumcheck(tables, q=spec.modulus, expression=expr, challenges=[3], num_rounds=2)
    ref_claim, ref_evals = O.sumcheck_reference(tables, q=spec.modulus, expression=expr, challenges=[3], num_rounds=2)
    assert claim == ref_claim and evals.tolist() == ref_evals.tolist()
    with pytest.raises(ValueError, match="has length"):
        api.sumcheck({"a": [1, 2, 3], "b": [1, 2, 3]}, q=spec.modulus, expression=expr, challenges=[1, 1], num_rounds=2)
    with pytest.raises(KeyError):
        api.sumcheck({"a": [1, 2, 3, 4]}, q=spec.modulus, expression=expr, challenges=[1, 1], num_rounds=2)
    with pytest.raises(ValueError, match="Unknown backend"):
        api.sumcheck(tables, q=spec.modulus, expression=expr, challenges=[1, 1], num_rounds=2, backend="reference")
    assert api.available_backends() == ["b200"]


def test_tail_launch_plan_and_timings():
    """Generic expressions: a launch per round up to the tail round, then one launch for the
    rest (sc_prove_launches), and the per-launch timings come in that number. The
    compile-time shapes keep a launch per round. Results are pinned by the oracle tests."""
    for name, tail_expected in (("plain_p32", True), ("plain_goldilocks", False), ("plain_bls", False)):
        cfg = PLAIN_CONFIGS[name]
        spec = get_field(cfg.bit_width)
        n = 14
        launches, tail = api.prove_launches(cfg.expression, spec, n)
        if tail_expected:
            assert 0 < tail < n - 1 and launches == tail + 1
        else:
            assert (launches, tail) == (n, n)
        ctx = api.get_context()
        ctx.launch_times()  # drop earlier records
        ctx.set_timing(True)
        try:
            api.prove(cfg.expression, cfg.bit_width, n, seed=5, table_kinds=cfg.table_kinds())
            times = ctx.launch_times()
        finally:
            ctx.set_timing(False)
        assert len(times) == launches and all(t > 0 for t in times)


@pytest.mark.parametrize("name,bw,n", [("plain_goldilocks", 64, 13), ("plain_goldilocks", 64, 16),
                                       ("plain_bls", 64, 15), ("plain_bls", 32, 14)])
def test_shape_kernels_match_c_oracle_at_larger_sizes(name, bw, n):
    """The compile-time shape kernels on rounds of 2^12 pairs and more (g(1) from the claim,
    many blocks, grid-stride loops), at 64 and 32 bits; bit-exact against the C oracle."""
    from oracle import c_oracle as C

    cfg = PLAIN_CONFIGS[name]
    spec = get_field(bw)
    kinds = cfg.table_kinds()
    proof = api.prove(cfg.expression, bw, n, seed=21, table_kinds=kinds)
    terms, k = O.indexed_terms(cfg.expression)
    tables = C.generate(spec.modulus, spec.limbs, [1 if x == "bernoulli" else 0 for x in kinds], n, 21)
    res = C.prove(terms, k, spec.modulus, spec.limbs, tables, "sha3")
    assert np.array_equal(proof.round_polys_mont, res["round_polys"])
    assert np.array_equal(proof.challenges_mont, res["challenges"])
    assert np.array_equal(proof.finals_mont, res["finals"])
    assert proof.checksum == res["checksum"]
