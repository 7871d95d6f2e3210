"""One proof split across ranks: the intra-proof multi-GPU path.

Each rank holds a contiguous chunk of every table (``world`` a power of two, chunk =
2^num_vars / world entries). Per round the rank proves its chunk to a share of g_j(0..d);
the shares are all-gathered -- (d + 1) L words per rank, one collective per round -- and
every rank sums them in rank order and derives the round's SHA3 challenge itself on the device,
so nothing is broadcast. The chunks are folded down to one entry per table, those are
all-gathered (K L words per rank), and every rank proves the last log2(world) rounds on the
gathered tables. Every rank's proof is bit-identical to ``prove_device`` on the whole tables.

``prove_split`` runs the protocol with any all-gather: ``torch_allgather()`` wraps
``torch.distributed`` (NCCL over NVLink between GPUs, or gloo); tests pass their own.
"""

from __future__ import annotations

import ctypes
from typing import Callable

import numpy as np

from . import _lib
from .api import CompiledExpression, Proof, get_context, get_device_field
from .expression import encode_expression
from .fields import FieldSpec


class SplitProver:
    """This rank's part of one split proof (``sc_split_*``).

    ``local_tables``: device tensor (K, L, 2^num_vars / world) of Montgomery limbs, this rank's
    chunk [rank C, (rank + 1) C) of every table; it must stay alive until ``result``.
    """

    def __init__(self, local_tables, expression, spec: FieldSpec, num_vars: int, world: int, rank: int,
                 challenge_mode: str = "sha3", device=None):
        lib = _lib.load()
        self.spec = spec
        self.ctx = get_context(device if device is not None else local_tables.device)
        fld = get_device_field(spec, self.ctx.device)
        self.expr = expression if isinstance(expression, CompiledExpression) else CompiledExpression(
            encode_expression(expression), spec.modulus)
        self.n, self.world, self.rank = int(num_vars), int(world), int(rank)
        self.K, self.L, self.d = self.expr.num_vars, spec.limbs, self.expr.degree
        want = (self.K, self.L, (1 << self.n) // max(1, self.world))
        if tuple(local_tables.shape) != want or not local_tables.is_contiguous():
            raise ValueError(f"local tables {tuple(local_tables.shape)}, expected contiguous {want}")
        self._tables = local_tables
        h = ctypes.c_void_p()
        rc = lib.sc_split_create(self.ctx.handle, fld.handle, self.expr.handle, self.n, self.world, self.rank,
                                 ctypes.c_void_p(local_tables.data_ptr()), _lib.CHALLENGE_MODES[challenge_mode],
                                 ctypes.byref(h))
        _lib.check(rc, "sc_split_create")
        self.handle = h
        self.local_rounds = lib.sc_split_local_rounds(h)

    @staticmethod
    def _p(a: np.ndarray):
        return a.ctypes.data_as(_lib.U32P)

    def round(self, j: int) -> np.ndarray:
        share = np.zeros((self.d + 1) * self.L, dtype=np.uint32)
        _lib.check(_lib.load().sc_split_round(self.handle, int(j), self._p(share)), "sc_split_round")
        return share

    def commit(self, j: int, shares) -> None:
        a = np.ascontiguousarray(np.asarray(shares, dtype=np.uint32).reshape(self.world, (self.d + 1) * self.L))
        _lib.check(_lib.load().sc_split_commit(self.handle, int(j), self._p(a)), "sc_split_commit")

    def last_entries(self) -> np.ndarray:
        out = np.zeros(self.K * self.L, dtype=np.uint32)
        _lib.check(_lib.load().sc_split_last_entries(self.handle, self._p(out)), "sc_split_last_entries")
        return out

    def finish(self, entries=None) -> None:
        if entries is None:
            _lib.check(_lib.load().sc_split_finish(self.handle, None), "sc_split_finish")
            return
        a = np.ascontiguousarray(np.asarray(entries, dtype=np.uint32).reshape(self.world, self.K * self.L))
        _lib.check(_lib.load().sc_split_finish(self.handle, self._p(a)), "sc_split_finish")

    def result(self) -> Proof:
        n, d, L, K = self.n, self.d, self.L, self.K
        polys = np.zeros((n, d + 1, L), dtype=np.uint32)
        chals = np.zeros((n, L), dtype=np.uint32)
        finals = np.zeros((1 + K, L), dtype=np.uint32)
        claim0 = np.zeros((L,), dtype=np.uint32)
        cs = ctypes.c_uint64(0)
        rc = _lib.load().sc_split_result(self.handle, self._p(polys), self._p(chals), self._p(finals),
                                         self._p(claim0), ctypes.byref(cs))
        _lib.check(rc, "sc_split_result")
        return Proof(self.spec, n, d, tuple(self.expr.encoded.var_names), polys, chals, finals, claim0, cs.value)

    def close(self) -> None:
        if getattr(self, "handle", None):
            _lib.load().sc_split_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


AllGather = Callable[[np.ndarray], np.ndarray]  # this rank's words -> (world, words) in rank order


def run_protocol(prover, allgather: AllGather) -> Proof:
    """The split protocol for one rank over any prover with SplitProver's methods."""
    for j in range(prover.local_rounds):
        prover.commit(j, allgather(prover.round(j)))
    if prover.world > 1:
        prover.finish(allgather(prover.last_entries()))
    else:
        prover.finish(None)
    return prover.result()


def prove_split(local_tables, expression, spec: FieldSpec, num_vars: int, world: int, rank: int,
                allgather: AllGather, challenge_mode: str = "sha3") -> Proof:
    p = SplitProver(local_tables, expression, spec, num_vars, world, rank, challenge_mode)
    try:
        return run_protocol(p, allgather)
    finally:
        p.close()


def torch_allgather(group=None, device=None) -> AllGather:
    """An all-gather over torch.distributed: uint32 words travel as int32 tensors (CUDA tensors
    for NCCL, CPU for gloo)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = device if device is not None else (torch.device("cuda", torch.cuda.current_device())
                                             if dist.get_backend(group) == "nccl" else torch.device("cpu"))

    def gather(words: np.ndarray) -> np.ndarray:
        t = torch.from_numpy(np.ascontiguousarray(words).view(np.int32)).to(dev)
        out = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(out, t, group=group)
        return np.stack([o.cpu().numpy().view(np.uint32) for o in out])

    return gather
