"""Helpers shared by the GPU parity tests: oracle-side tables and proof comparison."""

from __future__ import annotations

import hashlib

from oracle import oracle as O
from zkduel_b200.fields import from_limbs


def oracle_tables(kinds, seed, n, spec, arith_index=None):
    out = []
    for k, kind in enumerate(kinds):
        if kind == "uniform":
            out.append(O.uniform_table(seed, k, 1 << n, spec.modulus, spec.limbs))
        elif kind == "bernoulli":
            out.append(O.bernoulli_table(seed, k, 1 << n))
        else:
            v = k if arith_index is None else arith_index[k]
            out.append(O.arith_table(seed, v, 1 << n, spec.modulus))
    return out


def mont(x, spec):
    return spec.montgomery_limbs(x)


def assert_proof_equals_oracle(proof, res, spec):
    """Bit-exact: every output of the device proof equals the oracle's."""
    L = spec.limbs
    polys = [[list(map(int, v)) for v in row] for row in proof.round_polys_mont]
    assert polys == [[mont(x, spec) for x in row] for row in res["round_polys"]]
    assert [list(map(int, c)) for c in proof.challenges_mont] == [mont(x, spec) for x in res["challenges"]]
    assert list(map(int, proof.claim0_mont)) == mont(res["claim0"], spec)
    assert list(map(int, proof.finals_mont[0])) == mont(res["final_claim"], spec)
    assert [list(map(int, v)) for v in proof.finals_mont[1:]] == [mont(x, spec) for x in res["final_values"]]
    assert proof.checksum == res["checksum"]
    assert len(polys[0][0]) == L


def check_transcript_and_identities(proof, terms, spec, mode="sha3", final_values=None):
    """Size-independent checks of a proof of any size (verifier side, on the host).

    ``final_values``: f_k(r) recomputed on the host from the tables with the proof's
    challenges. The final-claim identity is then checked on those, not on the prover's own
    folded values, so a consistent proof of the wrong tables fails it."""
    p, L = spec.modulus, spec.limbs
    g = proof.round_polys
    ch = proof.challenges
    cs = 0
    for j, row in enumerate(g):
        limbs = [list(map(int, v)) for v in proof.round_polys_mont[j]]
        cs += sum((i + 1) * w for v in limbs for i, w in enumerate(v))
        if mode == "sha3":
            h = hashlib.sha3_256(b"zkduel:field-sweep:v1" + j.to_bytes(4, "little")
                                 + b"".join(w.to_bytes(4, "little") for v in limbs for w in v))
            assert ch[j] == int.from_bytes(h.digest(), "little") % p, f"round {j} challenge"
        if j:
            assert (row[0] + row[1]) % p == O.lagrange_eval(g[j - 1], ch[j - 1], p), f"round {j} identity"
    assert (g[0][0] + g[0][1]) % p == proof.claim0
    assert O.lagrange_eval(g[-1], ch[-1], p) == proof.final_claim
    if final_values is not None:
        assert list(final_values) == proof.final_values, "f_k(r) differs from the tables' own"
    values = proof.final_values if final_values is None else final_values
    assert O.evaluate_terms(terms, values, p) == proof.final_claim
    assert cs == proof.checksum
    assert all(from_limbs(list(map(int, v))) < p for row in proof.round_polys_mont for v in row)
