"""Batched proving: many independent proofs in one CUDA graph per field.

``BatchProver`` groups the proofs by field (modulus and limb count) and builds one native
batch (``sc_batch_create``) per group. Each batch runs on its own stream, so the groups
overlap on the device (a 64-bit group is memory-bound, a 256-bit group multiply-bound).
Within a group, round t of every proof runs in one persistent launch whose blocks pull
(proof, tile) items from a device work queue; the whole group is one CUDA graph.

Results are bit-identical to proving each proof alone (``prove_device``); the tests check
exactly that.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .api import CompiledExpression, Proof, get_context, get_device_field
from .expression import encode_expression
from .fields import FieldSpec, get_field


def degree_class(d: int) -> int:
    """The kernel class that proves degree d (its register arrays hold class + 1 points)."""
    return 2 if d <= 2 else (4 if d <= 4 else 7)


@dataclass
class _Group:
    spec: FieldSpec
    indices: list[int]
    exprs: list[CompiledExpression]
    handle: ctypes.c_void_p


class BatchProver:
    """Proves ``items`` = [(expression, bit_width, num_vars, tables), ...] together.

    ``tables`` are device tensors (K, L, 2^n) of Montgomery limbs (``generate_tables`` /
    ``upload_tables``); they must stay alive while the prover exists.
    ``tile`` maps a limb count to (threads per block, pairs per thread); None = defaults.
    ``tuning`` (an ``autotune.TuneTable``) chooses threads per (field, degree class) and pairs
    per thread per (field, degree class, num_vars); it overrides ``tile``.
    """

    def __init__(self, items: Sequence[tuple], device=None, challenge_mode: str = "sha3",
                 tile: dict[int, tuple[int, int]] | None = None, fields: Sequence[FieldSpec] | None = None,
                 tuning=None):
        lib = _lib.load()
        self.ctx = get_context(device)
        self.items = list(items)
        mode = _lib.CHALLENGE_MODES[challenge_mode]
        if mode == _lib.SC_CHALLENGE_EXPLICIT:
            raise ValueError("batches derive their challenges: 'sha3' or 'fixed'")
        self.mode = challenge_mode
        specs = list(fields) if fields is not None else [get_field(bw) for _e, bw, _n, _t in self.items]
        groups: dict[tuple[int, int], list[int]] = {}
        for i, spec in enumerate(specs):
            groups.setdefault((spec.modulus, spec.limbs), []).append(i)
        self.groups: list[_Group] = []
        self._keep = []
        for (_q, L), idx in groups.items():
            spec = specs[idx[0]]
            fld = get_device_field(spec, self.ctx.device)
            exprs = []
            for i in idx:
                e = self.items[i][0]
                exprs.append(e if isinstance(e, CompiledExpression) else CompiledExpression(encode_expression(e), spec.modulus))
            n = len(idx)
            expr_arr = (ctypes.c_void_p * n)(*[e.handle.value for e in exprs])
            rounds = (ctypes.c_int32 * n)(*[int(self.items[i][2]) for i in idx])
            tabs = (ctypes.c_void_p * n)(*[self.items[i][3].data_ptr() for i in idx])
            for i, e in zip(idx, exprs):
                t = self.items[i][3]
                want = (e.num_vars, L, 1 << int(self.items[i][2]))
                if tuple(t.shape) != want or not t.is_contiguous():
                    raise ValueError(f"proof {i}: tables {tuple(t.shape)}, expected contiguous {want}")
            threads, ppt = (tile or {}).get(L, (0, 0))
            cls_threads = [int(threads)] * 3
            proof_ppt = [int(ppt)] * n
            if tuning is not None:
                cls_threads = [tuning.threads(L, dc) for dc in (2, 4, 7)]
                proof_ppt = [tuning.pairs_per_thread(L, degree_class(e.degree), int(self.items[i][2]))
                             for i, e in zip(idx, exprs)]
            h = ctypes.c_void_p()
            rc = lib.sc_batch_create_tiled(self.ctx.handle, fld.handle, n, expr_arr, rounds, tabs, mode,
                                           (ctypes.c_int32 * 3)(*cls_threads), (ctypes.c_int32 * n)(*proof_ppt),
                                           ctypes.byref(h))
            _lib.check(rc, "sc_batch_create_tiled")
            self.groups.append(_Group(spec, idx, exprs, h))
            self._keep.append((expr_arr, rounds, tabs))

    def launch(self) -> None:
        """Enqueues one run of every group (asynchronous). Every group is launched before any
        is joined to the caller's stream, so the groups run concurrently on their own streams."""
        lib = _lib.load()
        for g in self.groups:
            _lib.check(lib.sc_batch_launch(g.handle), "sc_batch_launch")
        for g in self.groups:
            _lib.check(lib.sc_batch_join(g.handle), "sc_batch_join")

    def wait(self) -> None:
        lib = _lib.load()
        for g in self.groups:
            _lib.check(lib.sc_batch_wait(g.handle), "sc_batch_wait")

    def run(self) -> None:
        self.launch()
        self.wait()

    def tick_times(self) -> list[dict]:
        """Per (field group, degree class): the proof indices and each tick's start, end and
        duration (ms from the start of its group's last run; groups' origins differ)."""
        out = []
        lib = _lib.load()
        for g in self.groups:
            cnt = ctypes.c_int(0)
            _lib.check(lib.sc_batch_classes(g.handle, None, None, 0, ctypes.byref(cnt)), "sc_batch_classes")
            ncls = cnt.value
            dcls = (ctypes.c_int32 * max(1, ncls))()
            ticks = (ctypes.c_int32 * max(1, ncls))()
            _lib.check(lib.sc_batch_classes(g.handle, dcls, ticks, ncls, ctypes.byref(cnt)), "sc_batch_classes")
            _lib.check(lib.sc_batch_tick_times(g.handle, None, None, 0, ctypes.byref(cnt)), "sc_batch_tick_times")
            t0 = (ctypes.c_float * max(1, cnt.value))()
            t1 = (ctypes.c_float * max(1, cnt.value))()
            _lib.check(lib.sc_batch_tick_times(g.handle, t0, t1, cnt.value, ctypes.byref(cnt)), "sc_batch_tick_times")
            starts, ends = list(t0)[: cnt.value], list(t1)[: cnt.value]
            pos = 0
            for c in range(ncls):
                _lib.check(lib.sc_batch_class_proofs(g.handle, c, None, 0, ctypes.byref(cnt)), "sc_batch_class_proofs")
                idx = (ctypes.c_int32 * max(1, cnt.value))()
                _lib.check(lib.sc_batch_class_proofs(g.handle, c, idx, cnt.value, ctypes.byref(cnt)),
                           "sc_batch_class_proofs")
                sl = slice(pos, pos + ticks[c])
                out.append({"limbs": g.spec.limbs, "degree_class": int(dcls[c]),
                            "proofs": [g.indices[k] for k in list(idx)[: cnt.value]],
                            "start": starts[sl], "end": ends[sl],
                            "ms": [b - a for a, b in zip(starts[sl], ends[sl])]})
                pos += ticks[c]
        return out

    def result(self, i: int) -> Proof:
        """Outputs of proof ``i`` of the last run."""
        for g in self.groups:
            if i in g.indices:
                j = g.indices.index(i)
                e = g.exprs[j]
                L, n, d, K = g.spec.limbs, int(self.items[i][2]), e.degree, e.num_vars
                polys = np.zeros((n, d + 1, L), dtype=np.uint32)
                chals = np.zeros((n, L), dtype=np.uint32)
                finals = np.zeros((1 + K, L), dtype=np.uint32)
                claim0 = np.zeros((L,), dtype=np.uint32)
                cs = ctypes.c_uint64(0)
                p = lambda a: a.ctypes.data_as(_lib.U32P)  # noqa: E731
                rc = _lib.load().sc_batch_result(g.handle, j, p(polys), p(chals), p(finals), p(claim0), ctypes.byref(cs))
                _lib.check(rc, "sc_batch_result")
                return Proof(g.spec, n, d, e.encoded.var_names, polys, chals, finals, claim0, int(cs.value))
        raise IndexError(i)

    def results(self) -> list[Proof]:
        return [self.result(i) for i in range(len(self.items))]

    def close(self) -> None:
        for g in self.groups:
            if g.handle:
                _lib.load().sc_batch_destroy(g.handle)
                g.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
