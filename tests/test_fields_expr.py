"""Host logic: the modulus guard, expressions, the workload registry (CPU only)."""

from __future__ import annotations

import random

import numpy as np
import pytest

from conftest import load_jsonl
from zkduel_b200 import expression as X
from zkduel_b200 import fields as F
from zkduel_b200.api import host_tables_to_limbs
from zkduel_b200.workloads import KERNEL_WORKLOADS, WORKLOADS, get_kernel_workload, get_workload

GUARD = load_jsonl("guard_cases.jsonl")


@pytest.mark.parametrize("case", GUARD, ids=[f"{c['modulus']:#x}-L{c['limbs']}" for c in GUARD])
def test_guard_matches_reference_decisions(case):
    """Same accept/reject decision as the reference's guard, and the same wording."""
    if case["accepted"]:
        F.check_montgomery_modulus(case["modulus"], case["limbs"], case["nprime"])
        return
    with pytest.raises(F.UnsafeModulusError) as ei:
        F.check_montgomery_modulus(case["modulus"], case["limbs"], case["nprime"])
    ref = case["error"]
    for phrase in ("does not support this modulus", "valid only when", "nprime", "odd modulus", "does not fit"):
        if phrase in ref:
            assert phrase in str(ei.value)
    assert isinstance(ei.value, ValueError)


def test_configured_fields():
    assert sorted(F.FIELD_SPECS) == [32, 64, 128, 256]
    for bw, f in F.FIELD_SPECS.items():
        assert f.limbs == bw // 32
        assert f.nprime == F.montgomery_nprime(f.modulus)
        assert F.cios_bound_holds(f.modulus, f.limbs)
        x = 123456789 % f.modulus
        assert f.decode_limbs(f.montgomery_limbs(x)) == x
    assert F.FIELD_SPECS[64].modulus == 2**64 - 2**32 + 1
    with pytest.raises(ValueError):
        F.get_field(48)


def test_goldilocks_is_on_the_bound():
    g = F.FIELD_SPECS[64].modulus
    assert F.cios_bound_holds(g, 2) and not F.cios_bound_holds(g + 2, 2)


def test_field_for_modulus():
    assert F.field_for_modulus(F.FIELD_SPECS[256].modulus, 256) is F.FIELD_SPECS[256]
    f = F.field_for_modulus((1 << 61) - 1, 64)
    assert f.limbs == 2
    with pytest.raises(ValueError):
        F.field_for_modulus(1 << 70, 64)
    with pytest.raises(F.UnsafeModulusError):
        F.field_for_modulus((1 << 64) - 59, 64)


def test_stress_values_in_range():
    rng = random.Random(3)
    for f in F.FIELD_SPECS.values():
        for _ in range(200):
            assert 0 <= F.stress_value(f.modulus, f.limbs, rng) < f.modulus


def test_expression_forms_and_errors():
    assert X.normalize_expression([["a", "b"], ["c"]]) == ((1, ("a", "b")), (1, ("c",)))
    assert X.normalize_expression([(3, ["a"]), (-1, ("b", "a"))]) == ((3, ("a",)), (-1, ("b", "a")))
    assert X.expression_vars([["b", "a"], ["a", "c"]]) == ["b", "a", "c"]
    assert X.expression_degree(WORKLOADS["jellyfish_zerocheck_hp"]) == 7
    with pytest.raises(TypeError):
        X.normalize_expression(["ab"])
    with pytest.raises(TypeError):
        X.normalize_expression([[1, 2]])
    with pytest.raises(ValueError):
        X.normalize_expression([])
    enc = X.encode_expression(WORKLOADS["vanilla_zerocheck_hp"])
    assert enc.num_vars == 9 and enc.degree == 4 and enc.coeffs == (1, 1, 1, -1, 1)
    assert enc.term_offsets == (0, 3, 6, 10, 13) and len(enc.flat) == 15


def test_registry_and_kernel_workloads():
    assert len([w for w in WORKLOADS if w.startswith("zkphire_")]) == 25
    with pytest.raises(KeyError):
        get_workload("nope")
    assert len(KERNEL_WORKLOADS) == 32
    assert sorted(w.ident for w in KERNEL_WORKLOADS) == list(range(1, 33))
    for w in KERNEL_WORKLOADS:
        assert sorted(w.table_order) == sorted(X.expression_vars(w.expression))
        assert sorted(w.table_index()) == list(range(w.num_vars))
    assert get_kernel_workload("zkphire_20").name == "zk_vanilla_zerocheck_hp"


def test_host_tables_to_limbs():
    f = F.FIELD_SPECS[64]
    vals = np.array([[0, 1, f.modulus - 1, 2**63], [5, 6, 7, 8]], dtype=np.uint64)
    out = host_tables_to_limbs(vals, f)
    assert out.shape == (2, 2, 4) and out.dtype == np.uint32
    back = [[int(out[k, 0, i]) | (int(out[k, 1, i]) << 32) for i in range(4)] for k in range(2)]
    assert back == [[int(v) % f.modulus for v in row] for row in vals.tolist()]
    f256 = F.FIELD_SPECS[256]
    big = [[f256.modulus + 3, -1]]
    out = host_tables_to_limbs(big, f256)
    assert F.from_limbs(out[0, :, 0].tolist()) == 3 and F.from_limbs(out[0, :, 1].tolist()) == f256.modulus - 1
