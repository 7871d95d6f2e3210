"""One proof split across ranks (GPU): every rank's proof equals the whole proof, bit for bit.

The ranks are emulated in one process on one GPU: the host runs each rank's round, gathers
the shares (the all-gather a cluster does with NCCL) and commits them on every rank; no
kernel waits on another rank's kernel.
"""

from __future__ import annotations

import numpy as np
import pytest

from zkduel_b200 import api
from zkduel_b200.fields import get_field
from zkduel_b200.split import SplitProver

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)


def _same(a, b):
    assert np.array_equal(a.round_polys_mont, b.round_polys_mont)
    assert np.array_equal(a.challenges_mont, b.challenges_mont)
    assert np.array_equal(a.finals_mont, b.finals_mont)
    assert np.array_equal(a.claim0_mont, b.claim0_mont)
    assert a.checksum == b.checksum


def _emulate(tables, expr, spec, n, world, mode="sha3"):
    C = (1 << n) // world
    chunks = [tables[:, :, r * C:(r + 1) * C].contiguous() for r in range(world)]
    ranks = [SplitProver(c, expr, spec, n, world, r, mode) for r, c in enumerate(chunks)]
    for j in range(ranks[0].local_rounds):
        shares = np.stack([p.round(j) for p in ranks])
        for p in ranks:
            p.commit(j, shares)
    if world > 1:
        entries = np.stack([p.last_entries() for p in ranks])
        for p in ranks:
            p.finish(entries)
    else:
        for p in ranks:
            p.finish(None)
    out = [p.result() for p in ranks]
    for p in ranks:
        p.close()
    return out


CASES = [
    (32, (("a", "b"),), 10),
    (64, ((1, ("qL", "w1", "fz1")), (1, ("qR", "w2", "fz1")), (1, ("qM", "w1", "w2", "fz1")),
          (-1, ("qO", "w3", "fz1")), (1, ("qC", "fz1"))), 14),
    (128, ((1, ("a", "b", "c")), (3, ("d", "e")), (-1, ("a",))), 9),
    (256, ((1, ("a", "b", "c", "g")), (1, ("d", "e", "g"))), 8),
    (64, ((1, ("x", "y")),), 16),  # chunk rounds with g(1) from the claim
]


@pytest.mark.parametrize("bw,expr,n", CASES)
@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_split_equals_whole_proof(bw, expr, n, world):
    spec = get_field(bw)
    enc = api.encode_expression(expr)
    t = api.generate_tables(spec, enc.num_vars, n, [0] * enc.num_vars, 1000 + n + bw)
    whole = api.prove_device(t, expr, spec, n, "sha3")
    for proof in _emulate(t, expr, spec, n, world):
        _same(proof, whole)


def test_split_fixed_mode_and_errors():
    spec = get_field(64)
    expr = ((1, ("a", "b", "c")),)
    t = api.generate_tables(spec, 3, 7, [0] * 3, 5)
    whole = api.prove_device(t, expr, spec, 7, "fixed")
    for proof in _emulate(t, expr, spec, 7, 4, "fixed"):
        _same(proof, whole)
    with pytest.raises(ValueError):
        SplitProver(t[:, :, :64].contiguous(), expr, spec, 7, 3, 0)  # world not a power of two
    with pytest.raises(ValueError):
        SplitProver(t[:, :, :1].contiguous(), expr, spec, 7, 128, 0)  # chunks of one entry
    p = SplitProver(t[:, :, :32].contiguous(), expr, spec, 7, 4, 0)
    with pytest.raises(ValueError):
        p.commit(0, np.zeros((4, 4 * 2), dtype=np.uint32))  # not run yet
    with pytest.raises(ValueError):
        p.round(1)  # out of order
    p.close()
