"""The N > 1 path of bench.py on CPU: two gloo ranks.

Proofs are independent, so N GPUs run N replicas (rank r proves the stream of master seed r)
and the only cross-rank steps are the barriers around the timed region and the reductions
of the timings: max over ranks for times, sum for throughputs. The reference arm runs on
rank 0 alone; the other ranks return at once.
"""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    sys.path[:0] = [str(ROOT), str(ROOT / "sumcheck-triton_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    import bench
    from zkduel_b200.streams import batched_stream

    r, w, local = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank) and dist.get_backend() == "gloo"
    bench.barrier(w)
    res = {
        "max": bench.max_over_ranks(10.0 + rank, w),
        "sum": bench.sum_over_ranks(1.5 * (rank + 1), w),
        "stream_seeds": [s.seed for s in batched_stream(8, rank)],
        "reference_arm": bench.reference_arm(None, rank, w) if rank != 0 else None,
        # e2e: if one rank cannot pin its host tables, every rank skips the measurement
        "all_ok": bench.all_ranks_ok(True, w),
        "one_fails": bench.all_ranks_ok(rank != 1, w),
    }
    bench.barrier(w)
    dist.destroy_process_group()
    out[rank] = res


def test_two_ranks_reduce_and_split_the_stream():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0]["max"] == res[1]["max"] == 11.0  # times: the slowest rank
    assert res[0]["sum"] == res[1]["sum"] == 4.5  # throughput: every rank's proofs
    assert res[0]["stream_seeds"] != res[1]["stream_seeds"]  # replicas prove different proofs
    assert res[1]["reference_arm"] == 0  # non-zero ranks do no reference work
    assert res[0]["all_ok"] and res[1]["all_ok"]
    assert not res[0]["one_fails"] and not res[1]["one_fails"]  # both ranks skip together


def _bench(args, **env_extra):
    import json
    import subprocess

    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_PORT")}
    env.update(CUDA_VISIBLE_DEVICES="", **env_extra)
    out = subprocess.run([sys.executable, str(ROOT / "bench.py")] + args, capture_output=True, text=True,
                         timeout=600, env=env, cwd=str(ROOT))
    lines = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
    return out.returncode, lines, out.stderr


def test_bench_gpus_2_launches_two_ranks():
    """`bench.py --gpus 2` without a launcher starts two ranks itself (torch.distributed.run,
    gloo here); rank 0 prints the one line, reporting both ranks."""
    rc, lines, err = _bench(["--gpus", "2", "--impl", "reference", "--steps", "1", "--warmup", "0",
                             "--cpu-sample", "1"])
    assert rc == 0, err[-2000:]
    assert len(lines) == 1, lines
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


def test_bench_rejects_gpus_other_than_world_size():
    """Under a launcher, a world size other than --gpus is an error, never a silent
    run on fewer GPUs."""
    rc, lines, _err = _bench(["--gpus", "4", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                             WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    assert rc == 2 and lines and "error" in lines[0]
