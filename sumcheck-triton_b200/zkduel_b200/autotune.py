"""Autotuner of the batched prover's launch shape.

For every field (limb count L) and degree class (<= 2, <= 4, <= 7) it picks the threads per
block of that class's tick kernel, and for every num_vars range the pairs per thread of a
proof's tiles (a work item is threads x pairs_per_thread pairs). Candidates are timed on the
GPU with CUDA events on seeded synthetic proofs of that (field, class, range), each batch
replayed several times after a warm-up; the fastest wins. The table is cached as JSON per GPU
model and library version, so a process tunes once.

Order of the search (coordinate descent, a few seconds per field):
  1. threads per block, over the whole (field, class) group, pairs per thread at 2;
  2. pairs per thread per num_vars range, with the chosen threads.

Tiling never changes a result: every candidate proves bit-identically (the batched kernel's
tests run with several tile shapes).
"""

from __future__ import annotations

import json
import os
import random
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

from . import _lib
from .batch import BatchProver, degree_class
from .fields import get_field

THREADS = (64, 128, 256)
PAIRS_PER_THREAD = (1, 2, 4, 8, 16)
RANGES = ((1, 12), (13, 15), (16, 17), (18, 40))  # num_vars ranges with their own tile
SAMPLE_RANGES = ((10, 12), (13, 15), (16, 17), (18, 20))  # num_vars of the timed proofs per range
CLASSES = (2, 4, 7)
DEFAULT_CACHE = Path(os.environ.get("ZKDUEL_B200_TUNE_CACHE", Path.home() / ".cache" / "zkduel_b200" / "tune.json"))


def _range_of(n: int) -> int:
    for i, (lo, hi) in enumerate(RANGES):
        if lo <= n <= hi:
            return i
    return len(RANGES) - 1


@dataclass
class TuneTable:
    """threads[(L, class)] and ppt[(L, class, range index)]; missing entries: defaults."""

    threads_by: dict = field(default_factory=dict)
    ppt_by: dict = field(default_factory=dict)
    timings: dict = field(default_factory=dict)

    def threads(self, L: int, dclass: int) -> int:
        return int(self.threads_by.get((L, dclass), 0))

    def pairs_per_thread(self, L: int, dclass: int, n: int) -> int:
        return int(self.ppt_by.get((L, dclass, _range_of(n)), 0))

    def to_json(self) -> dict:
        return {
            "threads": {f"{L}/{c}": t for (L, c), t in self.threads_by.items()},
            "pairs_per_thread": {f"{L}/{c}/{r}": v for (L, c, r), v in self.ppt_by.items()},
            "ranges": RANGES,
            "timings_ms": self.timings,
        }

    @classmethod
    def from_json(cls, d: dict) -> "TuneTable":
        t = cls()
        for k, v in d.get("threads", {}).items():
            L, c = map(int, k.split("/"))
            t.threads_by[(L, c)] = int(v)
        for k, v in d.get("pairs_per_thread", {}).items():
            L, c, r = map(int, k.split("/"))
            t.ppt_by[(L, c, r)] = int(v)
        t.timings = d.get("timings_ms", {})
        return t


def _expression(rng: random.Random, dclass: int) -> tuple:
    """A sum of 1-3 products of distinct tables whose degree falls in the class."""
    lo, hi = {2: (2, 2), 4: (3, 4), 7: (5, 6)}[dclass]
    k = rng.randint(hi, 8)
    terms = []
    for t in range(rng.randint(1, 3)):
        size = rng.randint(lo, hi) if t == 0 else rng.randint(2, hi)
        terms.append((1, tuple(rng.sample([f"t{i}" for i in range(k)], size))))
    return tuple(terms)


def _group(L_bits: int, dclass: int, n_range: tuple[int, int], count: int, seed: int, device):
    from . import api

    spec = get_field(L_bits)
    rng = random.Random(seed)
    items = []
    for _ in range(count):
        expr = _expression(rng, dclass)
        n = rng.randint(*n_range)
        enc = api.encode_expression(expr)
        t = api.generate_tables(spec, enc.num_vars, n, [_lib.SC_TABLE_UNIFORM] * enc.num_vars, rng.getrandbits(63), device)
        items.append((expr, L_bits, n, t))
    return items


def _time(items, tuning: TuneTable, reps: int, device) -> float:
    import torch

    bp = BatchProver(items, device=device, tuning=tuning)
    try:
        bp.run()
        stream = torch.cuda.current_stream(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        a.record(stream)
        for _ in range(reps):
            bp.launch()
        b.record(stream)
        bp.wait()
        torch.cuda.synchronize(device)
        return a.elapsed_time(b) / reps
    finally:
        bp.close()


def autotune(bit_widths: Sequence[int] = (64, 256), classes: Sequence[int] = CLASSES, device=None,
             proofs_per_range: int = 12, reps: int = 3, seed: int = 7) -> TuneTable:
    """Times the candidates on the current GPU and returns the table (no cache)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    table = TuneTable()
    for bw in bit_widths:
        L = get_field(bw).limbs
        for dc in classes:
            groups = [_group(bw, dc, rg, proofs_per_range, seed + 101 * i + 7 * dc + bw, dev)
                      for i, rg in enumerate(SAMPLE_RANGES)]
            every = [it for g in groups for it in g]
            best = None
            for th in THREADS:
                if L >= 8 and th > 128:
                    continue  # the 8-limb kernels are compiled for 128-thread blocks
                trial = TuneTable(dict(table.threads_by), dict(table.ppt_by))
                trial.threads_by[(L, dc)] = th
                for r in range(len(RANGES)):
                    trial.ppt_by[(L, dc, r)] = 2
                ms = _time(every, trial, reps, dev)
                table.timings[f"{L}/{dc}/threads={th}"] = ms
                if best is None or ms < best[0]:
                    best = (ms, th)
            table.threads_by[(L, dc)] = best[1]
            for r, g in enumerate(groups):
                bestp = None
                for ppt in PAIRS_PER_THREAD:
                    trial = TuneTable(dict(table.threads_by), dict(table.ppt_by))
                    trial.ppt_by[(L, dc, r)] = ppt
                    ms = _time(g, trial, reps, dev)
                    table.timings[f"{L}/{dc}/{r}/ppt={ppt}"] = ms
                    if bestp is None or ms < bestp[0]:
                        bestp = (ms, ppt)
                table.ppt_by[(L, dc, r)] = bestp[1]
            del groups, every
            torch.cuda.empty_cache()
    return table


def tune_for(items, device=None, reps: int = 2, min_gain: float = 0.01, start: TuneTable | None = None,
             ppt_candidates: Sequence[int] = (1, 2, 4, 8)) -> TuneTable:
    """Tunes on the batch itself: ``items`` as for ``BatchProver``. Coordinate descent over
    threads per (field, degree class), then pairs per thread per (field, class, num_vars
    range), each candidate timed as the whole batch (best of ``reps`` replays after one warm-up);
    a change is kept when it beats the current best by ``min_gain``."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    present = sorted({(get_field(bw).limbs, degree_class(_degree(e)), _range_of(int(n))) for e, bw, n, _t in items})
    table = TuneTable(dict(start.threads_by), dict(start.ppt_by)) if start else TuneTable()

    def measure(t: TuneTable) -> float:
        return min(_time(items, t, 1, dev) for _ in range(reps))

    timings: dict = {}
    best = measure(table)
    timings["start"] = best
    for L, dc in sorted({(L, dc) for L, dc, _r in present}):
        for th in THREADS:
            if (L >= 8 and th > 128) or th == table.threads(L, dc):
                continue
            trial = TuneTable(dict(table.threads_by), dict(table.ppt_by))
            trial.threads_by[(L, dc)] = th
            ms = measure(trial)
            timings[f"{L}/{dc}/threads={th}"] = ms
            if ms < best * (1 - min_gain):
                best, table = ms, trial
    for L, dc, r in present:
        for ppt in ppt_candidates:
            if ppt == (table.pairs_per_thread(L, dc, RANGES[r][0]) or 2):
                continue
            trial = TuneTable(dict(table.threads_by), dict(table.ppt_by))
            trial.ppt_by[(L, dc, r)] = ppt
            ms = measure(trial)
            timings[f"{L}/{dc}/{r}/ppt={ppt}"] = ms
            if ms < best * (1 - min_gain):
                best, table = ms, trial
    timings["best"] = best
    table.timings = timings
    return table


def _degree(e) -> int:
    """Degree of a CompiledExpression or of an expression in the reference's term format."""
    if hasattr(e, "degree"):
        return int(e.degree)
    from .expression import normalize_expression

    return max(len(f) for _c, f in normalize_expression(e))


def cache_key(device=None) -> str:
    import torch

    name = torch.cuda.get_device_name(device)
    return f"{name}|lib{_lib.load().sc_version()}"


def load_or_tune(bit_widths: Sequence[int] = (64, 256), device=None, cache: Path | None = DEFAULT_CACHE,
                 retune: bool = False, **kw) -> TuneTable:
    """The cached table for this GPU model and library version, tuning (and caching) it first
    when absent, incomplete or ``retune``."""
    key = cache_key(device)
    data = {}
    if cache is not None and cache.exists():
        try:
            data = json.loads(cache.read_text())
        except (OSError, ValueError):
            data = {}
    want = {get_field(bw).limbs for bw in bit_widths}
    if not retune and key in data:
        t = TuneTable.from_json(data[key])
        if all((L, c) in t.threads_by for L in want for c in CLASSES):
            return t
    t = autotune(bit_widths, device=device, **kw)
    if cache is not None:
        data[key] = t.to_json()
        try:
            cache.parent.mkdir(parents=True, exist_ok=True)
            cache.write_text(json.dumps(data, indent=1))
        except OSError:
            pass
    return t


def degree_class_of(expression) -> int:
    return degree_class(max(len(f) for _c, f in expression))
