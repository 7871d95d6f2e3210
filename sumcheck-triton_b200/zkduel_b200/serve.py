"""Served proving: a request loop with continuous batching under an HBM budget.

``ProofServer`` wraps ``sc_server_*``: a native worker thread that admits requests in
arrival order by their HBM footprint, keeps each admitted request's tables (generated on
the device from its seed), fold buffers and transcript state resident, and merges the
rounds of the in-flight requests into shared launches of the batched round kernel on
high-priority streams. A request whose first round is larger than one wave of the GPU runs
whole on a low-priority stream instead (one launch per round, one block per tile), so the
small requests' blocks take SMs as its blocks retire: requests that arrive while a large
proof runs overtake it instead of queueing behind it. Policy ``"fifo_plain"`` is the
baseline: one request at a time, in arrival order, through the plain per-round path.

A request's result is bit-identical to ``prove_device`` on ``generate_tables`` with the
same seed, alone or in any mix; the GPU tests check exactly that.

``suspend`` stops requests at their next round boundary and frees their device memory;
``transcript`` then gives each one's :class:`~zkduel_b200.transcript.Transcript`, which
``submit(..., resume=t)`` continues -- on this server, another one, or after a restart --
or ``transcript.prove_rounds`` finishes on the plain path, bit-identically either way.

``replay`` drives a server with an arrival trace (seconds from its start) and returns the
latency of every request: completion minus arrival, on the server's clock.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .api import CompiledExpression, Proof, get_device_field
from .expression import encode_expression
from .fields import FieldSpec, get_field
from .transcript import Transcript


@dataclass
class RequestTimes:
    submit_s: float
    admit_s: float
    done_s: float


class ProofServer:
    """A served prover for one field on one GPU.

    budget_bytes   HBM admission budget (sum of admitted footprints).
    max_inflight   admitted requests at most.
    max_tables     tables per request at most (sizes the kernel's shared memory).
    chunk_items    tiles of one request per launch (0: two waves of the grid).
    """

    def __init__(self, spec: FieldSpec | int, policy: str = "continuous", budget_bytes: int = 150 * 10**9,
                 max_inflight: int = 256, max_tables: int = 8, threads: int = 0, pairs_per_thread: int = 0,
                 chunk_items: int = 0, device: int = 0):
        lib = _lib.load()
        self.spec = get_field(spec) if isinstance(spec, int) else spec
        self.device = int(device)
        self.field = get_device_field(self.spec, self.device)
        if policy not in _lib.SERVE_POLICIES:
            raise ValueError(f"policy must be one of {sorted(_lib.SERVE_POLICIES)}")
        self.policy = policy
        h = ctypes.c_void_p()
        rc = lib.sc_server_create(self.device, self.field.handle, _lib.SERVE_POLICIES[policy], int(budget_bytes),
                                  int(max_inflight), int(max_tables), int(threads), int(pairs_per_thread),
                                  int(chunk_items), ctypes.byref(h))
        _lib.check(rc, "sc_server_create")
        self.handle = h
        self._meta: dict[int, tuple] = {}  # id -> (n, degree, num_tables, var names, compiled expression)
        self._exprs: dict = {}

    # -------------------------------------------------------------------- requests

    def _compiled(self, expression) -> CompiledExpression:
        if isinstance(expression, CompiledExpression):
            return expression
        key = expression if isinstance(expression, tuple) else None
        if key is not None and key in self._exprs:
            return self._exprs[key]
        ce = CompiledExpression(encode_expression(expression), self.spec.modulus)
        if key is not None:
            self._exprs[key] = ce
        return ce

    def reserve(self, nbytes: int) -> None:
        """Maps ``nbytes`` into the server's memory pool now, so admissions do not grow it later."""
        _lib.check(_lib.load().sc_server_reserve(self.handle, int(nbytes)), "sc_server_reserve")

    def footprint(self, expression, num_vars: int) -> int:
        ce = self._compiled(expression)
        out = ctypes.c_uint64(0)
        _lib.check(_lib.load().sc_server_footprint(self.handle, ce.handle, int(num_vars), ctypes.byref(out)),
                   "sc_server_footprint")
        return out.value

    def submit(self, expression, num_vars: int, seed: int, kinds: Sequence[int] | None = None,
               challenge_mode: str = "sha3", resume: Transcript | None = None) -> int:
        """Queues one request; returns its id at once. ``resume``: continue that transcript
        (same expression, num_vars, seed and kinds as its tables; its challenge mode)."""
        ce = self._compiled(expression)
        k = ce.num_vars
        kinds = [_lib.SC_TABLE_UNIFORM] * k if kinds is None else list(kinds)
        if len(kinds) != k:
            raise ValueError(f"{len(kinds)} table kinds for {k} tables")
        rid = ctypes.c_uint64(0)
        seed_c = ctypes.c_uint64(int(seed) & (2**64 - 1))
        if resume is not None:
            if resume.num_rounds != int(num_vars):
                raise ValueError(f"transcript has {resume.num_rounds} rounds, request {num_vars}")
            w = resume.words
            rc = _lib.load().sc_server_submit_resume(self.handle, ce.handle, _lib.i32_array(kinds), seed_c,
                                                     w.ctypes.data_as(_lib.U32P), w.size, ctypes.byref(rid))
            _lib.check(rc, "sc_server_submit_resume")
        else:
            mode = _lib.CHALLENGE_MODES[challenge_mode]
            rc = _lib.load().sc_server_submit(self.handle, ce.handle, int(num_vars), _lib.i32_array(kinds), seed_c,
                                              mode, ctypes.byref(rid))
            _lib.check(rc, "sc_server_submit")
        self._meta[rid.value] = (int(num_vars), ce.degree, k, tuple(ce.encoded.var_names), ce)
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1) -> str:
        """Waits for request ``rid``: "done" or "suspended" (raises if it failed or timed out)."""
        rc = _lib.load().sc_server_wait(self.handle, ctypes.c_uint64(rid), int(timeout_ms))
        if rc == _lib.SC_SUSPENDED:
            return "suspended"
        _lib.check(rc, "sc_server_wait")
        return "done"

    def suspend(self, rid: int | None = None) -> None:
        """Suspends request ``rid`` (None: every unfinished request) at its next round boundary."""
        _lib.check(_lib.load().sc_server_suspend(self.handle, ctypes.c_uint64(0 if rid is None else rid)),
                   "sc_server_suspend")

    def transcript(self, rid: int) -> Transcript:
        """The transcript of a suspended request."""
        if rid not in self._meta:
            raise ValueError(f"unknown request {rid}")
        n, _d, _k, _names, ce = self._meta[rid]
        lib = _lib.load()
        words = ctypes.c_uint64(0)
        _lib.check(lib.sc_transcript_words(self.field.handle, ce.handle, n, ctypes.byref(words)), "sc_transcript_words")
        w = np.zeros(words.value, dtype=np.uint32)
        _lib.check(lib.sc_server_transcript(self.handle, ctypes.c_uint64(rid), w.ctypes.data_as(_lib.U32P), w.size),
                   "sc_server_transcript")
        return Transcript(w)

    def drain(self, timeout_ms: int = -1) -> None:
        _lib.check(_lib.load().sc_server_drain(self.handle, int(timeout_ms)), "sc_server_drain")

    def result(self, rid: int) -> Proof:
        if rid not in self._meta:
            raise ValueError(f"unknown request {rid}")
        n, d, k, names, _ce = self._meta[rid]
        L = self.spec.limbs
        polys = np.zeros((n, d + 1, L), dtype=np.uint32)
        chals = np.zeros((n, L), dtype=np.uint32)
        finals = np.zeros((1 + k, L), dtype=np.uint32)
        claim0 = np.zeros((L,), dtype=np.uint32)
        cs = ctypes.c_uint64(0)
        u32 = lambda a: a.ctypes.data_as(_lib.U32P)  # noqa: E731
        rc = _lib.load().sc_server_result(self.handle, ctypes.c_uint64(rid), u32(polys), u32(chals), u32(finals),
                                          u32(claim0), ctypes.byref(cs))
        _lib.check(rc, "sc_server_result")
        return Proof(self.spec, n, d, names, polys, chals, finals, claim0, cs.value)

    def times(self, rid: int) -> RequestTimes:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.load().sc_server_times(self.handle, ctypes.c_uint64(rid), ctypes.byref(a), ctypes.byref(b),
                                               ctypes.byref(c)), "sc_server_times")
        return RequestTimes(a.value, b.value, c.value)

    def release(self, rid: int) -> None:
        _lib.check(_lib.load().sc_server_release(self.handle, ctypes.c_uint64(rid)), "sc_server_release")
        self._meta.pop(rid, None)

    def stats(self) -> dict:
        st = _lib.ServerStats()
        _lib.check(_lib.load().sc_server_stats_get(self.handle, ctypes.byref(st)), "sc_server_stats_get")
        return {name: getattr(st, name) for name, _t in _lib.ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            _lib.load().sc_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ReplayReport:
    ids: list[int]
    arrival_s: list[float]      # when each request was submitted, from the replay's start
    latency_ms: list[float]     # completion - submission
    makespan_s: float           # first submission to last completion
    stats: dict

    def percentile(self, q: float) -> float:
        return float(np.percentile(np.asarray(self.latency_ms), q))

    @property
    def proofs_per_s(self) -> float:
        return len(self.ids) / self.makespan_s if self.makespan_s > 0 else float("inf")

    def summary(self) -> dict:
        lat = np.asarray(self.latency_ms)
        return {
            "requests": len(self.ids),
            "proofs_per_s": self.proofs_per_s,
            "p50_ms": float(np.percentile(lat, 50)),
            "p90_ms": float(np.percentile(lat, 90)),
            "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()),
            "makespan_s": self.makespan_s,
            "busy_s": self.stats.get("busy_s"),
            "ticks": self.stats.get("ticks"),
            "worker_build_s": self.stats.get("build_s"),   # composing and issuing ticks
            "worker_wait_s": self.stats.get("wait_s"),     # blocked on the GPU
            "worker_alloc_s": self.stats.get("alloc_s"),   # pool allocations at admission
            "peak_inflight": self.stats.get("peak_inflight"),
            "peak_footprint_gb": self.stats.get("peak_footprint", 0) / 1e9,
        }


def replay(server: ProofServer, requests: Sequence, time_scale: float = 1.0, release: bool = True,
           keep_results=False) -> tuple[ReplayReport, dict]:
    """Submits ``requests`` (streams.Request: spec + arrival_s) at their arrival times
    (scaled by ``time_scale``), waits for all, and reports each latency.

    Returns the report and {request index: Proof} for the requests ``keep_results`` names
    (True: all; a set of indices: those)."""
    reqs = list(requests)
    ids = []
    t_sub = []
    base = time.perf_counter()
    server_base = None
    for r in reqs:
        target = base + r.arrival_s * time_scale
        while True:
            dt = target - time.perf_counter()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.002) if dt > 0.0005 else 0)
        kinds = None
        rid = server.submit(r.spec.expression, r.spec.num_vars, r.spec.seed, kinds)
        ids.append(rid)
    server.drain()
    results = {}
    lat = []
    first = last = None
    for i, rid in enumerate(ids):
        t = server.times(rid)
        if server_base is None:
            server_base = t.submit_s
        t_sub.append(t.submit_s - server_base)
        lat.append((t.done_s - t.submit_s) * 1e3)
        first = t.submit_s if first is None else min(first, t.submit_s)
        last = t.done_s if last is None else max(last, t.done_s)
        if keep_results is True or (keep_results and i in keep_results):
            results[i] = server.result(rid)
        if release:
            server.release(rid)
    rep = ReplayReport(ids, t_sub, lat, (last - first) if ids else 0.0, server.stats())
    return rep, results
