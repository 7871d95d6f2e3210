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
        """Outputs of every proof of the last run: one native call per field group
        (``sc_batch_results``), each proof's arrays views into the group's buffers."""
        out: list[Proof | None] = [None] * len(self.items)
        lib = _lib.load()
        p = lambda a: a.ctypes.data_as(_lib.U32P)  # noqa: E731
        for g in self.groups:
            L = g.spec.limbs
            shapes = [(int(self.items[i][2]), e.degree, e.num_vars) for i, e in zip(g.indices, g.exprs)]
            polys = np.zeros(sum(n * (d + 1) * L for n, d, _k in shapes), dtype=np.uint32)
            chals = np.zeros(sum(n * L for n, _d, _k in shapes), dtype=np.uint32)
            finals = np.zeros(sum((1 + k) * L for _n, _d, k in shapes), dtype=np.uint32)
            claim0 = np.zeros(len(shapes) * L, dtype=np.uint32)
            cs = np.zeros(len(shapes), dtype=np.uint64)
            rc = lib.sc_batch_results(g.handle, p(polys), p(chals), p(finals), p(claim0),
                                      cs.ctypes.data_as(_lib.U64P))
            _lib.check(rc, "sc_batch_results")
            op = oc = of = 0
            for j, (i, e) in enumerate(zip(g.indices, g.exprs)):
                n, d, k = shapes[j]
                out[i] = Proof(g.spec, n, d, e.encoded.var_names,
                               polys[op:op + n * (d + 1) * L].reshape(n, d + 1, L), chals[oc:oc + n * L].reshape(n, L),
                               finals[of:of + (1 + k) * L].reshape(1 + k, L), claim0[j * L:(j + 1) * L],
                               int(cs[j]))
                op += n * (d + 1) * L
                oc += n * L
                of += (1 + k) * L
        return out

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


def chunk_bounds(sizes: Sequence[int], chunks: int) -> list[int]:
    """Cuts proofs of ``sizes`` bytes into at most ``chunks`` consecutive runs of about equal
    bytes: the boundaries [0, ..., len(sizes)], every run non-empty."""
    n = len(sizes)
    total, nch = sum(sizes), max(1, min(int(chunks), n))
    bounds, acc = [0], 0
    for i, b in enumerate(sizes):
        acc += b
        if len(bounds) < nch and acc >= total * len(bounds) / nch and i + 1 < n:
            bounds.append(i + 1)
    bounds.append(n)
    return bounds


class HostBatchProver:
    """Proves proofs whose tables live in host memory, end to end.

    ``items`` = [(expression, bit_width, num_vars), ...]; ``host_tables[i]`` is proof i's
    canonical tables, an int32 (K, L, 2^n) tensor of limbs in pinned host memory (read at
    every ``run``, so the caller may refill it between runs). Each ``run`` copies every
    proof's tables to the device, converts them to Montgomery form there, proves them and
    returns every proof's results on the host.

    The proofs are cut into ``chunks`` consecutive batches of about equal bytes, each a
    ``BatchProver``. The copies go out on ``copy_streams`` streams in chunk order and carry
    nothing else, so the transfer never waits for a kernel; chunk c's conversions and
    proving run on the caller's stream as soon as its own copies have landed. The later
    chunks' transfers overlap the earlier chunks' proving, so only the last chunk's
    proving adds to the PCIe time. Results are bit-identical to ``prove_device`` of each
    proof alone.

    Measured on one B200 with the 512-proof mixed stream (8.7 GB of tables a run, PCIe
    moving 54 GB/s): one chunk took 226 ms a run, 16 chunks on one copy stream 172 ms,
    within 7% of the transfer alone. More chunks or copy streams were slower (per-chunk
    launch and cross-stream event costs).
    """

    def __init__(self, items: Sequence[tuple], host_tables: Sequence, chunks: int = 16, copy_streams: int = 1,
                 device=None, tuning=None, challenge_mode: str = "sha3"):
        import torch

        from .api import empty_tables

        if len(items) != len(host_tables):
            raise ValueError(f"{len(items)} proofs, {len(host_tables)} host tables")
        if not items:
            raise ValueError("no proofs")
        self.ctx = get_context(device)
        dev = torch.device("cuda", self.ctx.device)
        self.stream = torch.cuda.current_stream(dev)
        self.host = list(host_tables)
        self.specs = [get_field(bw) for _e, bw, _n in items]
        self.dev_tables = []
        for (e, _bw, n), spec, h in zip(items, self.specs, self.host):
            t = empty_tables(spec, h.shape[0], int(n), self.ctx.device)
            if tuple(h.shape) != tuple(t.shape):
                raise ValueError(f"host tables {tuple(h.shape)}, expected {tuple(t.shape)}")
            self.dev_tables.append(t)
        sizes = [h.numel() * 4 for h in self.host]
        total = sum(sizes)
        bounds = chunk_bounds(sizes, chunks)
        self.chunks = []
        for a, b in zip(bounds[:-1], bounds[1:]):
            sub = [(items[i][0], items[i][1], items[i][2], self.dev_tables[i]) for i in range(a, b)]
            self.chunks.append((a, b, BatchProver(sub, device=device, challenge_mode=challenge_mode,
                                                  fields=self.specs[a:b], tuning=tuning)))
        self.copy_streams = [torch.cuda.Stream(dev) for _ in range(max(1, int(copy_streams)))]
        self.h2d_bytes = total

    def launch(self) -> None:
        """Enqueues one run (copies, conversions, every chunk's proving); asynchronous."""
        import torch

        lib = _lib.load()
        main = self.stream
        for st in self.copy_streams:
            st.wait_stream(main)  # the device tables are free again
        k = 0
        for a, b, bp in self.chunks:
            for i in range(a, b):
                with torch.cuda.stream(self.copy_streams[k % len(self.copy_streams)]):
                    self.dev_tables[i].copy_(self.host[i], non_blocking=True)
                k += 1
            for st in self.copy_streams:  # this chunk's copies, not the later ones
                ev = torch.cuda.Event()
                ev.record(st)
                main.wait_event(ev)
            for i in range(a, b):
                t = self.dev_tables[i]
                fld = get_device_field(self.specs[i], self.ctx.device)
                K, _L, N = t.shape
                _lib.check(lib.sc_tables_to_mont(self.ctx.handle, fld.handle, ctypes.c_void_p(t.data_ptr()),
                                                 ctypes.c_uint64(N), int(K)), "sc_tables_to_mont")
            bp.launch()

    def wait(self) -> None:
        for _a, _b, bp in self.chunks:
            bp.wait()

    def run(self) -> list[Proof]:
        self.launch()
        self.wait()
        return self.results()

    def results(self) -> list[Proof]:
        out = []
        for _a, _b, bp in self.chunks:
            out.extend(bp.results())
        return out

    def close(self) -> None:
        for _a, _b, bp in self.chunks:
            bp.close()
