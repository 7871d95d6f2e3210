"""The split-proof protocol driver on two gloo ranks (CPU): the rounds, all-gathers and
commits happen in order, every rank commits the shares in rank order, and the chunk entries
are gathered once before the last rounds."""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


class FakeProver:
    """Stands in for SplitProver: shares and entries that name their rank and round."""

    def __init__(self, world, rank, local_rounds=3, width=4):
        self.world, self.rank, self.local_rounds, self.width = world, rank, local_rounds, width
        self.log = []

    def round(self, j):
        self.log.append(("round", j))
        return np.array([self.rank, j] + [7] * (self.width - 2), dtype=np.uint32)

    def commit(self, j, shares):
        self.log.append(("commit", j, np.asarray(shares).tolist()))

    def last_entries(self):
        self.log.append(("entries",))
        return np.array([100 + self.rank] * self.width, dtype=np.uint32)

    def finish(self, entries):
        self.log.append(("finish", None if entries is None else np.asarray(entries).tolist()))

    def result(self):
        return self.log


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    sys.path[:0] = [str(ROOT), str(ROOT / "sumcheck-triton_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from zkduel_b200.split import run_protocol, torch_allgather

    out[rank] = run_protocol(FakeProver(world, rank), torch_allgather())
    dist.destroy_process_group()


def test_two_ranks_run_the_protocol_in_order():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        logs = dict(out)
    for rank in range(world):
        log = logs[rank]
        steps = [e[0] for e in log]
        assert steps == ["round", "commit"] * 3 + ["entries", "finish"]
        for j in range(3):
            shares = log[2 * j + 1][2]
            assert [s[:2] for s in shares] == [[r, j] for r in range(world)]  # rank order
        assert log[-1][1] == [[100 + r] * 4 for r in range(world)]
