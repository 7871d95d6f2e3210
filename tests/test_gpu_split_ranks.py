"""One proof split across two processes (GPU): the real protocol driver over torch.distributed.

Two spawned ranks share cuda:0 (this run has one GPU). Each holds its chunk of every table,
proves its chunk rounds, and the shares and last entries travel through gloo all-gathers
(`zkduel_b200.split.torch_allgather`). No kernel waits on the other rank's kernels: the
host gathers the shares between launches. Both ranks' proofs must equal `prove_device` on
the whole tables.
"""

from __future__ import annotations

import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]
EXPR = ((1, ("a", "b", "c")), (3, ("d", "e")))
BW, N, SEED = 64, 15, 404


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out):
    sys.path[:0] = [str(ROOT), str(ROOT / "sumcheck-triton_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from zkduel_b200 import api
        from zkduel_b200.fields import get_field
        from zkduel_b200.split import prove_split, torch_allgather

        torch.cuda.set_device(0)
        spec = get_field(BW)
        k = api.encode_expression(EXPR).num_vars
        whole = api.generate_tables(spec, k, N, [0] * k, SEED, device="cuda:0")
        C = (1 << N) // world
        chunk = whole[:, :, rank * C:(rank + 1) * C].contiguous()
        p = prove_split(chunk, EXPR, spec, N, world, rank, torch_allgather(device=torch.device("cpu")))
        out[rank] = (p.round_polys_mont.copy(), p.challenges_mont.copy(), p.finals_mont.copy(), int(p.checksum))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_split_proof_over_two_processes():
    from zkduel_b200 import api
    from zkduel_b200.fields import get_field

    world = 2
    with mp.get_context("spawn").Manager() as m:  # no fork after CUDA is up in this process
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    spec = get_field(BW)
    k = api.encode_expression(EXPR).num_vars
    whole = api.prove_device(api.generate_tables(spec, k, N, [0] * k, SEED), EXPR, spec, N, "sha3")
    for r in range(world):
        polys, chals, finals, cs = res[r]
        assert np.array_equal(polys, whole.round_polys_mont)
        assert np.array_equal(chals, whole.challenges_mont)
        assert np.array_equal(finals, whole.finals_mont)
        assert cs == whole.checksum
