"""Benchmark: SumCheck proofs/s on the mixed 512-proof stream, one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--path batched|plain]

A step proves the whole stream once: 512 independent proofs, num_vars uniform in {10..20},
64- or 256-bit field by coin flip, random sum-of-products expressions of degree 2-6 over
2-8 uniform tables (zkduel_b200.streams.batched_stream, master seed 0; rank r uses master
seed r, so per-GPU work is fixed: weak scaling, no collective on the data path).

Prints one JSON line (rank 0):
  value      proofs/s over all ranks, tables resident in HBM before the timed region,
             timed with CUDA events on the proving stream, max over ranks;
  e2e        the same through the host-buffer API (zkduel_b200.batch.HostBatchProver): every
             step copies each proof's tables from pinned host memory, in chunks whose copies
             overlap the proving of the chunks before, and reads each proof's results back;
             reported with the measured PCIe host-to-device rate that bounds it;
  plain      the same stream proved one proof at a time (the denominator of the batched
             speed-up);
  roofline   the dominant round kernel (by time) against its bound: integer multiply-adds
             against the measured IMAD rate (256-bit) or bytes against measured HBM GB/s;
  cpu_baseline  the C oracle (all host threads) on a fixed stratified sample of the same
             stream (32 proofs, about 1/16 of its work; see cpu_sample_specs);
  plain_configs  the three plain configurations at full size, one proof at a time;
  reference_cuda  the reference's own CUDA executable (built from its source into
             oracle/_ref) beside this library's drop-in of it, same arguments, checksums compared;
  served     the served stream (zkduel_b200.streams.served_stream: 20,000 requests over
             2^127 - 1, num_vars log-uniform 12..24, degree 3-7 over up to 8 tables, Poisson
             arrivals at the rate that keeps the FIFO-plain server 80% busy, measured first)
             replayed in real time through the continuous-batching server and through the
             FIFO-plain server, 150 GB admission budget: proofs/s and p50/p90/p99 latency
             (host-observed completion minus submission) for both; then the capacity sweep
             (offered rates beyond FIFO's capacity, and a burst) and a burst of requests up to
             num_vars 26 where the budget binds.
--impl reference times that CPU port alone on the same fixed sample (the reference's own
prover is Python-only and its source does not travel here; the port restates it and is
pinned against it, and reference.py itself was timed at full size where its source is).
--gpus N runs one rank per GPU: under a launcher the world size must equal N; without one the
bench re-runs itself under torch.distributed.run with N ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "sumcheck-triton_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "sumcheck_proofs_per_s_mixed_stream"
WORKLOAD = "batched_512"
STREAM_COUNT = 512
PEAKS = ROOT / "MEASURED_PEAKS.json"
SERVED_COUNT = 20000
SERVED_LOAD = 0.8
SERVED_BUDGET = 150 * 10**9
CAPACITY_MULTIPLES = (1.0, 1.1, 1.2, 1.3, 1.5, 2.0)  # offered rate / FIFO-plain capacity (1 / E[service])
CAPACITY_P99_MS = 100.0  # a rate is sustained when throughput >= 95% of it and p99 stays under this
CPU_SAMPLE_STRIDE = 16
CPU_SAMPLE_PROOFS = STREAM_COUNT // CPU_SAMPLE_STRIDE  # proofs 0, 16, ..., 496 of the stream


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--path", choices=["batched", "plain"], default="batched")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain-configs", action="store_true",
                    help="skip the three plain configs' latency (GPU) and CPU-port timings")
    ap.add_argument("--e2e-chunks", type=int, default=16,
                    help="host-buffer path: batches whose copies overlap the proving of the ones before")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE_PROOFS,
                    help="proofs in the fixed CPU sample (every 16th proof of the stream, from proof 0)")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes instead of the autotuned ones")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference CUDA executable comparison")
    ap.add_argument("--served", type=int, default=SERVED_COUNT,
                    help="requests in the served stream (0: skip the served measurement)")
    ap.add_argument("--capacity-requests", type=int, default=3000,
                    help="served capacity: requests per offered rate (0: skip the capacity sweep)")
    ap.add_argument("--budget-requests", type=int, default=300,
                    help="served: a burst of requests with num_vars up to 26, where the HBM budget binds (0: skip)")
    ap.add_argument("--case", default=None,
                    help="profile mode: prove one plain config (plain_p32|plain_goldilocks|plain_bls) twice and exit")
    ap.add_argument("--case-vars", type=int, default=None, help="num_vars for --case (default: the config's)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="profile mode: build the mixed stream (--stream-count proofs), run the batch twice, exit")
    ap.add_argument("--stream-count", type=int, default=STREAM_COUNT, help="proofs in the stream (profile mode)")
    ap.add_argument("--profile-field", type=int, default=0, choices=[0, 64, 256],
                    help="profile mode: only the proofs of this field width (0: both)")
    ap.add_argument("--profile-split", action="store_true",
                    help="profile mode: plain_goldilocks at num_vars 22 proved as 2 emulated ranks (the host "
                         "gathers the shares), twice, then exit")
    ap.add_argument("--profile-served", action="store_true",
                    help="profile mode: a burst of 120 requests of the served stream (num_vars 12..18) through "
                         "the continuous server, then exit")
    ap.add_argument("--profile-aux", action="store_true",
                    help="profile mode: the plain path's generic kernels (point-parallel 8-limb, 2-limb generic, "
                         "tail launch), a resume refold and a host-table conversion, each twice, then exit")
    return ap.parse_args()


def profile_batch(args) -> int:
    """The batched path on a (smaller) mixed stream, twice; for ncu captures."""
    import torch

    from zkduel_b200.batch import BatchProver

    work = Workload(master_seed=0, device=torch.device("cuda", 0), count=args.stream_count)
    bp = BatchProver([(e, s.bit_width, s.num_vars, t) for s, _f, e, t in work.items
                      if args.profile_field in (0, s.bit_width)])
    for _ in range(2):
        bp.run()
    torch.cuda.synchronize()
    print(json.dumps({"profile_batch": args.stream_count, "field": args.profile_field, "table_bytes": work.table_bytes(),
                      "checksum0": bp.result(bp.groups[0].indices[0]).checksum}))
    return 0


def profile_split(args) -> int:
    """One proof split over 2 ranks, emulated in this process on one GPU: each rank's round
    kernel (ext_out) on its chunk, the host gathers the shares, each rank's commit kernel
    (split_commit_kernel) finalises the round; twice, the first warms up. plain_goldilocks at
    num_vars 22: 9 tables x 2^22 x 8 B = 302 MB in two 151 MB chunks (> L2)."""
    import numpy as np
    import torch

    from zkduel_b200 import api
    from zkduel_b200.configs import PLAIN_CONFIGS
    from zkduel_b200.fields import get_field
    from zkduel_b200.split import SplitProver

    cfg = PLAIN_CONFIGS["plain_goldilocks"]
    n, world = 22, 2
    spec = get_field(cfg.bit_width)
    enc = api.encode_expression(cfg.expression)
    kinds = [api._lib.SC_TABLE_BERNOULLI if k == "bernoulli" else api._lib.SC_TABLE_UNIFORM for k in cfg.table_kinds()]
    t = api.generate_tables(spec, enc.num_vars, n, kinds, cfg.seed)
    C = (1 << n) // world
    chunks = [t[:, :, r * C:(r + 1) * C].contiguous() for r in range(world)]
    for _ in range(2):
        ranks = [SplitProver(c, cfg.expression, spec, n, world, r) for r, c in enumerate(chunks)]
        for j in range(ranks[0].local_rounds):
            shares = np.stack([p.round(j) for p in ranks])
            for p in ranks:
                p.commit(j, shares)
        entries = np.stack([p.last_entries() for p in ranks])
        for p in ranks:
            p.finish(entries)
        out = [p.result() for p in ranks]
        for p in ranks:
            p.close()
    torch.cuda.synchronize()
    print(json.dumps({"profile_split": world, "num_vars": n, "checksum": out[0].checksum,
                      "ranks_equal": out[0].checksum == out[1].checksum}))
    return 0


def profile_case(args) -> int:
    """One plain proof, twice (first warms up); for ncu captures of the round kernel."""
    import torch

    from zkduel_b200 import api
    from zkduel_b200.configs import PLAIN_CONFIGS
    from zkduel_b200.fields import get_field

    cfg = PLAIN_CONFIGS[args.case]
    n = args.case_vars or cfg.num_vars
    spec = get_field(cfg.bit_width)
    enc = api.encode_expression(cfg.expression)
    kinds = [api._lib.SC_TABLE_BERNOULLI if k == "bernoulli" else api._lib.SC_TABLE_UNIFORM for k in cfg.table_kinds()]
    t = api.generate_tables(spec, enc.num_vars, n, kinds, cfg.seed)
    expr = api.CompiledExpression(enc, spec.modulus)
    times = []
    for _ in range(2):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        p = api.prove_device(t, expr, spec, n, "sha3")
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    print(json.dumps({"case": args.case, "num_vars": n, "ms": times, "checksum": p.checksum}))
    return 0


# ------------------------------------------------------------------------------ helpers


def measured_peaks() -> dict:
    try:
        return json.loads(PEAKS.read_text())
    except (OSError, ValueError):
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def relaunch_ranks(n_gpus: int) -> int | None:
    """One process per GPU. Under a launcher (WORLD_SIZE set) the world must be --gpus;
    without one, --gpus N > 1 re-runs this command under torch.distributed.run with N ranks
    on this node and returns its exit code. None: go on in this process."""
    world = os.environ.get("WORLD_SIZE")
    if world is not None:
        if int(world) != n_gpus:
            print(json.dumps({"error": f"--gpus {n_gpus} but WORLD_SIZE={world}: launch one rank per GPU"}),
                  flush=True)
            return 2
        return None
    if n_gpus <= 1:
        return None
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n_gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd)


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n_gpus:
        raise SystemExit(f"--gpus {n_gpus} but WORLD_SIZE={world}")
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if _cuda_ok() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def _cuda_ok() -> bool:
    import torch

    return torch.cuda.is_available()


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def profiled_traffic_ratio(L: int):
    """DRAM bytes / algorithmic bytes of the L-limb ticks, from the committed ncu summary."""
    import re

    f = ROOT / "profiles" / "batch_round_kernel_mixed_stream_64.md"
    if L != 8 or not f.exists():
        return None
    m = re.search(r"traffic_ratio_L8:\s*([0-9.]+)", f.read_text())
    return float(m.group(1)) if m else None


def busy_ms(intervals) -> float:
    """Length of the union of [start, end] intervals (ms)."""
    iv = sorted(intervals)
    busy, a0, b0 = 0.0, None, None
    for a, b in iv:
        if b0 is None or a > b0:
            if b0 is not None:
                busy += b0 - a0
            a0, b0 = a, b
        else:
            b0 = max(b0, b)
    return busy + (b0 - a0 if b0 is not None else 0.0)


def group_alone_rooflines(work, batch_items, work_per_round, tuning, device, hbm_peak: float,
                          imad_rate: float) -> dict:
    """Each field group of the stream proved alone (its own BatchProver, the same tiles),
    outside the timed region: its ticks' busy time (CUDA events inside the graph, last of 3
    timed runs), and its algorithmic bytes and IMAD over that time against the group's own
    bound -- HBM for the 2-limb group, the IMAD rate for the 8-limb group. In the timed step
    the two groups share the SMs, so their by-class rates there are not rooflines."""
    from zkduel_b200.batch import BatchProver

    out = {}
    for bw in sorted({s.bit_width for s, _f, _e, _t in work.items}):
        idx = [i for i, (s, _f, _e, _t) in enumerate(work.items) if s.bit_width == bw]
        bp = BatchProver([batch_items[i] for i in idx], device=device, tuning=tuning)
        for _ in range(2):
            bp.run()
        ms = timed(bp.run, 3, 1, device) / 3
        cls = bp.tick_times()
        bp.close()
        L = cls[0]["limbs"]
        busy = busy_ms([iv for c in cls for iv in zip(c["start"], c["end"])])
        b = sum(w[1] for i in idx for w in work_per_round[i])
        im = sum(w[2] for i in idx for w in work_per_round[i])
        e = {"proofs": len(idx), "ms_per_step": ms, "busy_ms": busy, "GB/s": b / (busy / 1e3) / 1e9,
             "TIMAD/s": im / (busy / 1e3) / 1e12}
        if L >= 4:
            e.update(bound="imad", frac=e["TIMAD/s"] / (imad_rate / 1e12))
        else:
            e.update(bound="hbm", frac=e["GB/s"] / hbm_peak)
        out[f"L{L}"] = e
    return out


def all_ranks_ok(ok: bool, world: int) -> bool:
    """True on every rank when every rank passes ok (one collective, the same on all ranks)."""
    return max_over_ranks(0.0 if ok else 1.0, world) == 0.0


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------------------ workload


class Workload:
    """The stream's proofs with their tables resident on the device."""

    def __init__(self, master_seed: int, device, count: int = STREAM_COUNT):
        import torch

        from zkduel_b200 import api
        from zkduel_b200.fields import get_field
        from zkduel_b200.streams import batched_stream

        self.specs = batched_stream(count, master_seed)
        self.items = []
        for s in self.specs:
            spec = get_field(s.bit_width)
            enc = s.encoded()
            expr = api.CompiledExpression(enc, spec.modulus)
            tables = api.generate_tables(spec, enc.num_vars, s.num_vars, [api._lib.SC_TABLE_UNIFORM] * enc.num_vars,
                                         s.seed, device)
            self.items.append((s, spec, expr, tables))
        torch.cuda.synchronize(device)

    def table_bytes(self) -> int:
        return sum(t.numel() * 4 for _s, _f, _e, t in self.items)


def run_plain(work: Workload):
    from zkduel_b200 import api

    out = []
    for s, spec, expr, tables in work.items:
        out.append(api.prove_device(tables, expr, spec, s.num_vars, "sha3"))
    return out


def timed(fn, steps: int, world: int, device):
    import torch

    barrier(world)
    torch.cuda.synchronize(device)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        fn()
    end.record()
    torch.cuda.synchronize(device)
    barrier(world)
    return start.elapsed_time(end)


# ------------------------------------------------------------------------------ CPU port


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_sample_specs(proofs: int = CPU_SAMPLE_PROOFS, master_seed: int = 0):
    """A fixed, stratified sample of the stream: the proofs sorted by (field width,
    num_vars, index), then every 16th of that order from the 8th on -- so each size class of
    the stream is represented in proportion and the sample holds about 1/16 of the stream's
    work (the work of a proof grows as 2^num_vars, so an unsorted every-16th sample is
    dominated by whichever few large proofs it happens to hit)."""
    from zkduel_b200.streams import batched_stream

    specs = sorted(batched_stream(STREAM_COUNT, master_seed), key=lambda s: (s.bit_width, s.num_vars, s.index))
    return specs[CPU_SAMPLE_STRIDE // 2::CPU_SAMPLE_STRIDE][:max(1, proofs)]


def cpu_port_sample(proofs: int = CPU_SAMPLE_PROOFS, master_seed: int = 0):
    """The C oracle with every host thread on the fixed stratified sample
    (``cpu_sample_specs``), the same proofs every run. Table generation is outside the
    timed region, as it is for the GPU. Returns (proofs/s, proofs, seconds, threads): with
    the whole sample (1/16 of the stream's proofs and about 1/16 of its work), proofs/s
    estimates the rate over the whole stream."""
    from oracle import c_oracle as C
    from oracle import oracle as O
    from zkduel_b200.fields import get_field

    threads = os.cpu_count() or 1
    specs = cpu_sample_specs(proofs, master_seed)
    spent = 0.0
    for s in specs:
        f = get_field(s.bit_width)
        terms, k = O.indexed_terms(s.expression)
        t = C.generate(f.modulus, f.limbs, [0] * k, s.num_vars, s.seed)
        t0 = time.perf_counter()
        C.prove(terms, k, f.modulus, f.limbs, t, "sha3", threads=threads)
        spent += time.perf_counter() - t0
    return len(specs) / spent, len(specs), spent, threads


def cpu_sample_text(done: int) -> str:
    return (f"{done} proofs: the 512-proof stream (master seed 0) sorted by (field, num_vars), every "
            f"{CPU_SAMPLE_STRIDE}th from the {CPU_SAMPLE_STRIDE // 2}th (stratified, about 1/{CPU_SAMPLE_STRIDE} "
            f"of the stream's work), the same every run")


def reference_arm(args, rank: int, world: int):
    """The reference's CPU prover path, restated in C (the reference's own prover is pure
    Python and its source does not travel with this repository), on every host thread.
    A step proves the fixed sample once; rank 0 alone runs it."""
    if rank != 0:
        return 0
    per_step = []
    done, threads = 0, 1
    for i in range(args.warmup + args.steps):
        rate, done, spent, threads = cpu_port_sample(args.cpu_sample)
        if i >= args.warmup:
            per_step.append(spent)
    total = sum(per_step)
    value = done * len(per_step) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(per_step),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (Montgomery)",
        "data": "synthetic", "config": {"workload": WORKLOAD, "proofs_per_step": done, "sample": cpu_sample_text(done)},
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                         "sample": cpu_sample_text(done)},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------ main


def main() -> int:
    args = parse()
    if args.case:
        return profile_case(args)
    if args.profile_batch:
        return profile_batch(args)
    if args.profile_aux:
        return profile_aux(args)
    if args.profile_served:
        return profile_served(args)
    if args.profile_split:
        return profile_split(args)
    rc = relaunch_ranks(args.gpus)
    if rc is not None:
        return rc
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch

    from zkduel_b200 import api, roofline
    from zkduel_b200.fields import get_field

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    work = Workload(master_seed=rank, device=device)
    ctx = api.get_context(device)
    imad_rate = api.calibrate_imad(ctx)

    from zkduel_b200.batch import BatchProver

    tuning = None
    batch_items = [(e, s.bit_width, s.num_vars, t) for s, _f, e, t in work.items]
    if not args.no_tune:
        from zkduel_b200.autotune import tune_for

        tuning = tune_for(batch_items, device=device)  # on this stream, before the timed region
    batcher = BatchProver(batch_items, device=device, tuning=tuning)
    steps_fn = {"batched": batcher.run, "plain": lambda: run_plain(work)}

    def measure(path, steps):
        for _ in range(args.warmup):
            steps_fn[path]()
        if path == "plain":
            ctx.set_timing(True)
        with ClockSampler(local) as clk:
            ms = timed(steps_fn[path], steps, world, device)
        launch_ms = ctx.launch_times() if path == "plain" else None
        if path == "plain":
            ctx.set_timing(False)
        return max_over_ranks(ms / steps, world), launch_ms, clk

    path = args.path
    ms_step, launch_ms, clocks = measure(path, args.steps)
    value = world * STREAM_COUNT / (ms_step / 1e3)
    other = "plain" if path == "batched" else "batched"
    ms_other, launch_other, _clk = measure(other, max(1, min(args.steps, 3)))
    if path == "batched":
        ms_plain, plain_launch_ms = ms_other, launch_other
    else:
        ms_plain, plain_launch_ms = ms_step, launch_ms

    # roofline of the dominant kernel class: algorithmic work per launch over CUDA-event
    # durations. Batched: the tick times of the last run of the timed region (events inside
    # the graph); plain: every launch of its timed region.
    per_class = {}

    def add(L, ms, b, im, launches=1):
        c = per_class.setdefault(L, {"ms": 0.0, "bytes": 0, "imad": 0, "launches": 0})
        c["ms"] += ms
        c["bytes"] += b
        c["imad"] += im
        c["launches"] += launches

    work_per_round = []
    for s, spec, _e, _t in work.items:
        enc = s.encoded()
        M = roofline.products_per_point(s.expression)
        work_per_round.append([(spec.limbs, roofline.launch_bytes(enc.num_vars, spec.limbs, s.num_vars, j),
                                roofline.launch_imad(enc.num_vars, spec.limbs, enc.degree, M, s.num_vars, j))
                               for j in range(s.num_vars)])
    if path == "batched":
        # Degree classes of one field run concurrently on their own streams: a field's
        # kernel time is the union of its ticks' [start, end] intervals (busy time).
        # a class's work is every round of its proofs (the last tick of a proof also proves its
        # tail rounds, so ticks and rounds do not map one to one)
        classes = batcher.tick_times()
        spans = {}
        for c in classes:
            b = sum(w[1] for i in c["proofs"] for w in work_per_round[i])
            im = sum(w[2] for i in c["proofs"] for w in work_per_round[i])
            add(c["limbs"], 0.0, b, im, launches=len(c["start"]))
            for a, b_ in zip(c["start"], c["end"]):
                spans.setdefault(c["limbs"], []).append((a, b_))
        for L, iv in spans.items():
            iv.sort()
            busy, cur_a, cur_b = 0.0, None, None
            for a, b_ in iv:
                if cur_b is None or a > cur_b:
                    if cur_b is not None:
                        busy += cur_b - cur_a
                    cur_a, cur_b = a, b_
                else:
                    cur_b = max(cur_b, b_)
            busy += cur_b - cur_a
            per_class[L]["ms"] = busy
        gpu_launches = sum(len(c["ms"]) for c in classes) * args.steps
    else:
        # one launch per round up to a proof's tail round, then one launch for the rest
        from zkduel_b200 import api

        flat = []
        for (s, spec, e, _t), rounds in zip(work.items, work_per_round):
            _n, tail = api.prove_launches(e, spec, s.num_vars, device)
            flat.extend(rounds[:tail])
            if tail < len(rounds):
                flat.append((spec.limbs, sum(w[1] for w in rounds[tail:]), sum(w[2] for w in rounds[tail:])))
        for i, t in enumerate(launch_ms):
            L, b, im = flat[i % len(flat)]
            add(L, t, b, im)
        gpu_launches = len(launch_ms)
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    roof = None
    if per_class:
        L, c = max(per_class.items(), key=lambda kv: kv[1]["ms"])
        if L >= 4:
            ach = c["imad"] / (c["ms"] / 1e3) / 1e12
            pk = imad_rate / 1e12
            kname = f"batch_round_kernel<{L}, *, *>" if path == "batched" else f"round_kernel<{L}, *, *>"
            roof = {"bound": "imad", "kernel": kname, "achieved": ach, "peak": pk,
                    "unit": "TIMAD/s", "frac": ach / pk, "traffic": None,
                    "peak_source": "sc_calibrate_imad probe (measured live)"}
        else:
            ach = c["bytes"] / (c["ms"] / 1e3) / 1e9
            kname = f"batch_round_kernel<{L}, *, *>" if path == "batched" else f"round_kernel<{L}, *, *>"
            roof = {"bound": "hbm", "kernel": kname, "achieved": ach, "peak": hbm_peak,
                    "unit": "GB/s", "frac": ach / hbm_peak, "traffic": None,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback"}
        ratio = profiled_traffic_ratio(L) if path == "batched" else None
        if ratio is not None:
            roof["traffic"] = ratio * c["bytes"] / max(1, c["launches"])
            roof["traffic_unit"] = "bytes per launch"
            roof["traffic_source"] = (f"dram__bytes_read.sum + dram__bytes_write.sum of every {L}-limb tick of the "
                                      f"64-proof cut (profiles/), {ratio:.3f} x the algorithmic bytes, applied to "
                                      f"this run's algorithmic bytes per launch")
        if path == "batched" and len(per_class) > 1:
            roof["note"] = ("the field groups run concurrently on their own streams; a class's launch "
                            "durations include the other group's use of the SMs")
        roof["by_class"] = {f"L{k}": {"busy_ms": v["ms"], "launches": v["launches"],
                                      "GB/s": v["bytes"] / (v["ms"] / 1e3) / 1e9,
                                      "TIMAD/s": v["imad"] / (v["ms"] / 1e3) / 1e12} for k, v in per_class.items()}
        if path == "batched":
            roof["alone"] = group_alone_rooflines(work, batch_items, work_per_round, tuning, device, hbm_peak,
                                                  imad_rate)

    line = {
        "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 limbs (Montgomery; 64- and 256-bit fields)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "path": path, "proofs_per_step_per_gpu": STREAM_COUNT,
                   "table_bytes_per_gpu": work.table_bytes(),
                   "l2": "inputs larger than L2 (tables total > 126 MB); no flush", "parallelism": f"replicas x{world}"},
        "plain": {"value": world * STREAM_COUNT / (ms_plain / 1e3), "unit": "proofs/s", "ms_per_step": ms_plain,
                  "path": "one proof at a time (sc_prove per proof)"},
        "speedup_vs_plain": ms_plain / ms_step if path == "batched" else 1.0,
        "gpu_launches": gpu_launches,
        "tuning": None if tuning is None else {"threads": tuning.to_json()["threads"],
                                               "pairs_per_thread": tuning.to_json()["pairs_per_thread"],
                                               "untuned_ms": tuning.timings.get("start"),
                                               "tuned_ms": tuning.timings.get("best")},
        "clocks": clocks.summary(),
        "imad_peak_tera_per_s": imad_rate / 1e12,
    }
    if roof:
        line["roofline"] = roof

    if not args.no_e2e:  # every rank: its own host buffers and PCIe link, max time over ranks
        resident = batcher.results() if path == "batched" else run_plain(work)
        e2e = e2e_measure(work, args, device, path == "batched", tuning, world, expect=resident)
        if rank == 0:
            line["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, done, spent, threads = cpu_port_sample(args.cpu_sample)
        line["cpu_baseline"] = {"value": rate, "unit": "proofs/s", "cores": threads, "kind": "port",
                                "sample": f"{cpu_sample_text(done)}; {spent:.1f} s", "cpu_model": cpu_model()}
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        line["reference_cuda"] = reference_cuda_compare()
    if rank == 0 and world == 1 and not args.no_plain_configs:
        line["plain_configs"] = plain_configs_measure(device, cpu=not args.no_cpu, hbm_peak=hbm_peak,
                                                      imad_rate=imad_rate)
    if args.served > 0:
        del batcher, steps_fn, work
        torch.cuda.empty_cache()
        line["served"] = served_measure(args, device, rank, world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


REF_BIN = ROOT / "oracle" / "_ref" / "field_sumcheck_cuda"
CLI_BIN = ROOT / "sumcheck-triton_b200" / "bin" / "field_sumcheck_b200"
PLAIN_CASES = (("poly_ab", 16, 32), ("zk_vanilla_zerocheck_hp", 24, 64), ("poly_abcg_plus_deg", 22, 256))


def profile_served(args) -> int:
    """A burst of served requests (2^127 - 1, num_vars 12..18, degree 3-7) through the
    continuous server: its ticks (4-limb batched kernel), tail rounds, lane launches and
    table generation."""
    from zkduel_b200.fields import get_field
    from zkduel_b200.serve import ProofServer, replay
    from zkduel_b200.streams import served_stream

    reqs = served_stream(120, rate_per_s=1e9, seed=5, min_vars=12, max_vars=18)
    with ProofServer(get_field(128)) as srv:
        rep, _ = replay(srv, reqs)
    print(json.dumps({"profile_served": len(reqs), "p50_ms": rep.summary()["p50_ms"]}))
    return 0


def profile_aux(args) -> int:
    """Kernels outside the plain configs and the batch, on inputs larger than L2, twice each
    (the first warms up): a generic 256-bit proof at n = 21 (point-parallel kernel, tail
    launch), a generic 64-bit proof at n = 22 (generic round kernel), the refold of a 64-bit
    n = 22 transcript resumed at round 10 (fold_kernel), the Montgomery conversion of
    host tables (convert_tables_kernel), and the IMAD-rate probe (imad_probe_kernel)."""
    import torch

    from zkduel_b200 import api
    from zkduel_b200 import transcript as tr
    from zkduel_b200.fields import get_field

    f256, f64 = get_field(256), get_field(64)
    e256 = ((1, ("a", "b")), (3, ("c",)))
    e64 = ((1, ("a", "b", "c")), (5, ("d",)))
    t256 = api.generate_tables(f256, 3, 21, [0] * 3, 1)
    t64 = api.generate_tables(f64, 4, 22, [0] * 4, 2)
    host = api.download_tables(t64, f64)
    half = tr.prove_rounds(t64, e64, f64, 10, tr.start(e64, f64, 22))
    ctx = api.get_context()
    for _ in range(2):
        api.prove_device(t256, e256, f256, 21, "sha3")
        api.prove_device(t64, e64, f64, 22, "sha3")
        tr.prove_rounds(t64, e64, f64, 22, half)
        api.upload_tables(host, f64)
        api.calibrate_imad(ctx)  # imad_probe_kernel
    torch.cuda.synchronize()
    print(json.dumps({"profile_aux": True, "bytes_256": t256.numel() * 4, "bytes_64": t64.numel() * 4}))
    return 0


def plain_configs_measure(device, cpu: bool = True, cpu_vars: int = 20, hbm_peak: float | None = None,
                          imad_rate: float | None = None) -> dict:
    """The three plain configs one proof at a time at full size, tables resident: per-proof
    device time (CUDA events) as p50 / p99 and proofs/s. Beside it the C port of the
    reference's CPU prover (every host thread) on the same tables: at full size for the
    32-bit config; for the others at num_vars = cpu_vars, the time scaled by 2^(n - cpu_vars)
    (the work is linear in the table size), with the GPU checksum compared at that size."""
    import torch

    from oracle import c_oracle as C
    from oracle import oracle as O
    from zkduel_b200 import api, roofline
    from zkduel_b200.configs import PLAIN_CONFIGS
    from zkduel_b200.fields import get_field

    out = {}
    for name, cfg in PLAIN_CONFIGS.items():
        spec = get_field(cfg.bit_width)
        enc = api.encode_expression(cfg.expression)
        kinds = [api._lib.SC_TABLE_BERNOULLI if k == "bernoulli" else api._lib.SC_TABLE_UNIFORM
                 for k in cfg.table_kinds()]
        expr = api.CompiledExpression(enc, spec.modulus)
        n = cfg.num_vars
        t = api.generate_tables(spec, enc.num_vars, n, kinds, cfg.seed, device)
        for _ in range(3):
            api.prove_device(t, expr, spec, n, "sha3")
        reps = 200 if n <= 16 else 40
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            p = api.prove_device(t, expr, spec, n, "sha3")
            b.record()
            torch.cuda.synchronize(device)
            ms.append(a.elapsed_time(b))
        del t
        ms.sort()
        entry = {"num_vars": n, "gpu": {"p50_ms": ms[len(ms) // 2], "p99_ms": ms[min(len(ms) - 1, int(0.99 * len(ms)))],
                                        "proofs_per_s": 1e3 * len(ms) / sum(ms), "proofs": len(ms),
                                        "timer": "CUDA events around each prove_device (results on the host)"}}
        # the whole proof against its bound (canonical counts, zkduel_b200.roofline): HBM for
        # the 64-bit zerocheck, the IMAD rate for 256 bits; the 32-bit config is L2-resident
        p50_s = entry["gpu"]["p50_ms"] / 1e3
        if spec.limbs == 2 and hbm_peak:
            b = roofline.proof_bytes(enc.num_vars, spec.limbs, n)
            entry["roofline"] = {"bound": "hbm", "algorithmic_bytes": b, "achieved": b / p50_s / 1e9,
                                 "peak": hbm_peak, "unit": "GB/s", "frac": b / p50_s / 1e9 / hbm_peak}
        elif spec.limbs == 8 and imad_rate:
            im = roofline.proof_imad(enc.num_vars, spec.limbs, enc.degree, sum(t - 1 for t in enc.term_lens), n)
            entry["roofline"] = {"bound": "imad", "algorithmic_imad": im, "achieved": im / p50_s / 1e12,
                                 "peak": imad_rate / 1e12, "unit": "TIMAD/s", "frac": im / p50_s / imad_rate}
        else:
            entry["roofline"] = {"bound": "latency", "note": "tables resident in L2 (2 x 256 KiB): p50 / p99 latency"}
        if cpu:
            nc = n if n <= 16 else cpu_vars
            terms, k = O.indexed_terms(cfg.expression)
            ct = C.generate(spec.modulus, spec.limbs, kinds, nc, cfg.seed)
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            res = C.prove(terms, k, spec.modulus, spec.limbs, ct, "sha3", threads=threads)
            sec = time.perf_counter() - t0
            gt = api.generate_tables(spec, enc.num_vars, nc, kinds, cfg.seed, device)
            gp = api.prove_device(gt, expr, spec, nc, "sha3")
            entry["cpu_port"] = {"ms_per_proof": sec * 1e3 * (1 << (n - nc)), "threads": threads,
                                 "sample": "full size" if nc == n else f"num_vars {nc}, time x 2^{n - nc}",
                                 "checksum_equal_gpu": gp.checksum == res["checksum"]}
        out[name] = entry
    return out


def reference_cuda_compare() -> dict:
    """The three plain configs through the reference's own CUDA executable (built from its
    source for sm_100a into oracle/_ref) and through this library's drop-in of that executable,
    same arguments and inputs (the reference's table fill): median ms of 10 runs after 2
    warm-ups, and whether the checksums agree."""
    import csv as _csv
    import tempfile

    if not REF_BIN.exists() or not CLI_BIN.exists():
        return {"unavailable": "reference CUDA executable not built (oracle/Makefile.ref)"}
    out = {"args": "--challenge-mode sha3 --point-mode specialized --warmups 2 --repeats 10 (host timer, median)"}
    with tempfile.TemporaryDirectory() as td:
        for wl, n, bw in PLAIN_CASES:
            row = {}
            for name, binary in (("reference", REF_BIN), ("b200", CLI_BIN)):
                csv_path = Path(td) / f"{name}_{wl}.csv"
                subprocess.run([str(binary), "--workloads", wl, "--rounds", str(n), "--bit-widths", str(bw),
                                "--challenge-mode", "sha3", "--point-mode", "specialized", "--warmups", "2",
                                "--repeats", "10", "--out", str(csv_path)], check=True, stdout=subprocess.DEVNULL,
                               timeout=600)
                r = list(_csv.DictReader(csv_path.open()))[-1]
                row[name] = {"median_ms": float(r["median_ms"]), "checksum": int(r["checksum"])}
            row["speedup"] = row["reference"]["median_ms"] / row["b200"]["median_ms"]
            row["checksums_equal"] = row["reference"]["checksum"] == row["b200"]["checksum"]
            out[f"{wl} n={n} {bw}-bit"] = row
    return out


def served_measure(args, device, rank: int, world: int) -> dict:
    """The served stream through both server policies (one server per rank, own stream)."""
    import torch

    from zkduel_b200 import api
    from zkduel_b200.fields import get_field
    from zkduel_b200.serve import ProofServer, replay
    from zkduel_b200.streams import served_stream

    spec = get_field(128)
    dev = device.index
    reserve = 32 << 30
    # E[plain service time]: a burst through the FIFO-plain server (busy time / requests)
    cal = served_stream(1000, rate_per_s=1e9, seed=1000 + rank)
    with ProofServer(spec, policy="fifo_plain", budget_bytes=SERVED_BUDGET, device=dev) as srv:
        srv.reserve(reserve)
        replay(srv, sorted(cal[:100], key=lambda r: r.spec.num_vars))
        b0 = srv.stats()["busy_s"]
        replay(srv, cal)
        service_s = (srv.stats()["busy_s"] - b0) / len(cal)
    rate = SERVED_LOAD / service_s
    reqs = served_stream(args.served, rate_per_s=rate, seed=1 + rank)
    check = {0, len(reqs) // 2, len(reqs) - 1}
    out = {"requests_per_gpu": len(reqs), "field": "2^127-1 (4 limbs)", "load": SERVED_LOAD,
           "arrival_rate_per_s": rate, "plain_service_ms": service_s * 1e3, "budget_bytes": SERVED_BUDGET,
           "latency": "host-observed completion minus submission"}
    for pol in ("continuous", "fifo_plain"):
        with ProofServer(spec, policy=pol, budget_bytes=SERVED_BUDGET, device=dev) as srv:
            srv.reserve(reserve)
            replay(srv, served_stream(50, rate_per_s=rate, seed=99))
            srv.reserve(reserve)
            # every size once, largest last, so no scratch grows inside the timed replay
            warm = sorted(served_stream(400, rate_per_s=1e9, seed=98), key=lambda r: r.spec.num_vars)
            seen = {}
            for r in warm:
                seen[(r.spec.num_vars, r.spec.degree > 4)] = r
            replay(srv, list(seen.values()))
            rep, kept = replay(srv, reqs, keep_results=check)
        summ = rep.summary()
        # bit-exactness on a sample: the served result equals the proof alone
        for i in sorted(check):
            s = reqs[i].spec
            t = api.generate_tables(spec, s.num_tables, s.num_vars, [0] * s.num_tables, s.seed, device)
            alone = api.prove_device(t, s.expression, spec, s.num_vars, "sha3")
            got = kept[i]
            assert (got.checksum == alone.checksum and (got.round_polys_mont == alone.round_polys_mont).all()
                    and (got.finals_mont == alone.finals_mont).all()), f"served request {i} differs from its proof alone"
            del t
        summ["bit_exact_sample"] = sorted(check)
        if world > 1:
            summ["proofs_per_s"] = sum_over_ranks(summ["proofs_per_s"], world)
            for k in ("p50_ms", "p90_ms", "p99_ms", "mean_ms"):
                summ[k] = max_over_ranks(summ[k], world)
        out[pol] = summ
    c, f = out["continuous"], out["fifo_plain"]
    out["p50_speedup_vs_fifo"] = f["p50_ms"] / c["p50_ms"]
    out["p99_speedup_vs_fifo"] = f["p99_ms"] / c["p99_ms"]
    if args.capacity_requests > 0:
        out["capacity"] = served_capacity(args, spec, dev, service_s, rank, world)
    if args.budget_requests > 0:
        out["budget_binding"] = served_budget_binding(args, spec, dev, device, rank, world)
    torch.cuda.synchronize(device)
    return out


def served_capacity(args, spec, dev: int, service_s: float, rank: int, world: int) -> dict:
    """Offered load beyond what FIFO-plain can serve: the served distribution replayed at
    CAPACITY_MULTIPLES x FIFO-plain's capacity (1 / E[plain service]) through both policies,
    and once as a burst (every request at time 0: the policy's saturated throughput). A
    rate is sustained when the throughput keeps up with it (>= 95%) and p99 stays under
    CAPACITY_P99_MS; each policy's capacity is the highest sustained rate."""
    from zkduel_b200.serve import ProofServer, replay
    from zkduel_b200.streams import served_stream

    fifo_cap = 1.0 / service_s
    out = {"fifo_capacity_per_s": fifo_cap, "requests_per_point": args.capacity_requests,
           "p99_bound_ms": CAPACITY_P99_MS, "rule": "sustained: proofs/s >= 0.95 x offered and p99 <= bound"}
    for pol in ("continuous", "fifo_plain"):
        pts = []
        with ProofServer(spec, policy=pol, budget_bytes=SERVED_BUDGET, device=dev) as srv:
            srv.reserve(32 << 30)
            replay(srv, served_stream(50, rate_per_s=1e9, seed=97))
            for mult in CAPACITY_MULTIPLES:
                rate = mult * fifo_cap
                rep, _ = replay(srv, served_stream(args.capacity_requests, rate_per_s=rate,
                                                   seed=700 + int(10 * mult) + 100 * rank))
                s = rep.summary()
                pts.append({"offered_x_fifo": mult, "offered_per_s": rate, "proofs_per_s": s["proofs_per_s"],
                            "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"]})
            rep, _ = replay(srv, served_stream(args.capacity_requests, rate_per_s=1e9, seed=799 + 100 * rank))
        ok = [p["offered_per_s"] for p in pts
              if p["proofs_per_s"] >= 0.95 * p["offered_per_s"] and p["p99_ms"] <= CAPACITY_P99_MS]
        entry = {"points": pts, "sustained_per_s": max(ok) if ok else 0.0, "burst_proofs_per_s": rep.proofs_per_s}
        if world > 1:
            entry["sustained_per_s"] = sum_over_ranks(entry["sustained_per_s"], world)
            entry["burst_proofs_per_s"] = sum_over_ranks(entry["burst_proofs_per_s"], world)
        out[pol] = entry
    c, f = out["continuous"], out["fifo_plain"]
    out["sustained_ratio_vs_fifo"] = c["sustained_per_s"] / f["sustained_per_s"] if f["sustained_per_s"] else None
    out["burst_ratio_vs_fifo"] = c["burst_proofs_per_s"] / f["burst_proofs_per_s"]
    return out


def served_budget_binding(args, spec, dev: int, device, rank: int, world: int) -> dict:
    """A burst of the served distribution with num_vars up to 26 (up to ~15 GB a request)
    through the continuous server: the requests' footprints add up to more than the
    150 GB budget, so admission holds requests back. Reports throughput, latency, the peak
    admitted footprint (never above the budget) and whether the largest proof equals proving
    it alone, bit for bit (`largest_bit_exact`)."""
    from zkduel_b200 import api
    from zkduel_b200.serve import ProofServer, replay
    from zkduel_b200.streams import served_stream

    reqs = served_stream(args.budget_requests, rate_per_s=1e9, seed=900 + rank, max_vars=26)
    big = max(range(len(reqs)), key=lambda i: reqs[i].spec.num_vars)
    with ProofServer(spec, policy="continuous", budget_bytes=SERVED_BUDGET, device=dev) as srv:
        fp = sum(srv.footprint(r.spec.expression, r.spec.num_vars) for r in reqs)
        rep, kept = replay(srv, reqs, keep_results={big})
    s = rep.summary()
    sb = reqs[big].spec
    t = api.generate_tables(spec, sb.num_tables, sb.num_vars, [0] * sb.num_tables, sb.seed, device)
    alone = api.prove_device(t, sb.expression, spec, sb.num_vars, "sha3")
    del t
    got = kept[big]
    exact = bool(got.checksum == alone.checksum and (got.round_polys_mont == alone.round_polys_mont).all())
    return {"requests": len(reqs), "max_num_vars": max(r.spec.num_vars for r in reqs),
            "sum_footprints_gb": fp / 1e9, "budget_gb": SERVED_BUDGET / 1e9,
            "peak_footprint_gb": s["peak_footprint_gb"], "proofs_per_s": s["proofs_per_s"], "p50_ms": s["p50_ms"],
            "p99_ms": s["p99_ms"], "makespan_s": s["makespan_s"], "largest_bit_exact": exact,
            "largest_num_vars": sb.num_vars}


def e2e_measure(work: Workload, args, device, batched: bool, tuning=None, world: int = 1, expect=None) -> dict:
    """Host-buffer path: per step, every proof's canonical tables go from pinned host memory
    to the device and are converted to Montgomery form there; the proofs run (batched, or
    one sc_prove per proof); every proof's results are read back to the host. With several
    ranks each proves its own stream from its own host buffers; the step time is the
    slowest rank's, and the bytes and proofs are the whole job's. ``expect``: the resident
    path's proofs; the last timed step's proofs must equal them (round polynomials,
    challenges, final values, checksum) or the measurement is reported unavailable."""
    import torch

    from zkduel_b200 import api
    from zkduel_b200.batch import HostBatchProver

    host, why = [], ""
    try:
        for s, spec, _e, t in work.items:
            canon = api.download_tables(t, spec)
            host.append(torch.from_numpy(canon.view("int32")).pin_memory())
    except (RuntimeError, MemoryError) as e:  # pinned host memory is a per-node resource
        why = f"pinning {len(host)}/{len(work.items)} proofs' tables failed: {str(e)[:160]}"
    if not all_ranks_ok(not why, world):  # every rank takes the same path
        return {"unavailable": why or "another rank could not pin its host tables"}
    h2d = sum(h.numel() * 4 for h in host)

    if batched:
        # the public host-buffer batch API: copies in chunks overlapped with the proving
        hb = HostBatchProver([(e, spec.bit_width, s.num_vars) for s, spec, e, _t in work.items], host,
                             chunks=args.e2e_chunks, copy_streams=int(os.environ.get("E2E_COPY_STREAMS", "1")),
                             device=device, tuning=tuning)
        step = hb.run
    else:
        def step():
            return [api.prove_host(h, e, spec, s.num_vars, "sha3", device=device)
                    for (s, spec, e, _t), h in zip(work.items, host)]

    step()
    torch.cuda.synchronize(device)
    steps = max(1, min(args.steps, 3))
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        res = step()
    torch.cuda.synchronize(device)
    dt = max_over_ranks((time.perf_counter() - t0) / steps, world)
    d2h = sum(p.round_polys_mont.nbytes + p.challenges_mont.nbytes + p.finals_mont.nbytes + p.claim0_mont.nbytes + 8
              for p in res)
    import numpy as np

    bad = [] if expect is None else [
        i for i, (a, b) in enumerate(zip(res, expect))
        if not (a.checksum == b.checksum and np.array_equal(a.round_polys_mont, b.round_polys_mont)
                and np.array_equal(a.challenges_mont, b.challenges_mont) and np.array_equal(a.finals_mont, b.finals_mont))]
    if expect is not None and len(res) != len(expect):
        bad.append(-1)
    if not all_ranks_ok(not bad, world):
        return {"unavailable": f"host-buffer proofs differ from the resident path's (proofs {bad[:8]})"
                if bad else "another rank's host-buffer proofs differ from its resident path's"}
    pcie = h2d_bandwidth(device)
    return {"value": world * STREAM_COUNT / dt, "unit": "proofs/s", "h2d_bytes_per_step": world * h2d,
            "d2h_bytes_per_step": world * d2h, "ms_per_step": dt * 1e3, "ranks": world,
            "path": (f"batched, {args.e2e_chunks} chunks" if batched else "plain") + " (host buffers)",
            "steps": steps, "timer": "host wall clock around synchronised steps",
            # the bound of this path: the step's host-to-device bytes at the measured copy rate
            "pcie_h2d_gbs": pcie, "h2d_frac": (h2d / dt / 1e9) / pcie if pcie else None,  # per rank
            "results_equal_resident": expect is not None}


def h2d_bandwidth(device, nbytes: int = 1 << 30) -> float:
    """Pinned host-to-device copy rate (GB/s): best of 3 copies of 1 GiB, host timer around
    synchronised copies."""
    import torch

    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device=device)
    best = 0.0
    for _ in range(3):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        d.copy_(h, non_blocking=True)
        torch.cuda.synchronize(device)
        best = max(best, nbytes / (time.perf_counter() - t0) / 1e9)
    del h, d
    return best


if __name__ == "__main__":
    sys.exit(main())
