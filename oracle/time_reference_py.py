"""Times the reference's own CPU prover (``src/zkduel/reference.py:44-110``,
``sumcheck_reference``) single-threaded on the three plain configurations -- TEST
INFRASTRUCTURE ONLY (a measurement recipe; nothing in the product imports it).

The reference is pure Python and cannot travel to the GPU host, so it is timed where its
source tree is (``SUMCHECK_REFERENCE`` must name the reference checkout; there is no
default). For each configuration:

1. the seeded tables are generated by the C oracle (the same seeded generator the GPU
   path uses), converted to Python ints;
2. the C oracle proves them with SHA3 challenges; its challenges, decoded from Montgomery
   form, are the challenges ``sumcheck_reference`` consumes (it derives none itself);
3. ``sumcheck_reference`` runs once, timed with ``time.perf_counter`` around the call
   only (table conversion excluded), on one thread;
4. its ``(claim0, round evaluations)`` are compared with the C oracle's, decoded from
   Montgomery form -- a full-size pin of the C oracle against the reference itself.

Two stream samples (``stream_batched``, ``stream_served``) time the same function on a
seeded, stratified sample of the batched and the served proof streams: every proof of the
sample runs in a ``multiprocessing`` pool (spawn) with one worker per host core; each worker
times ``sumcheck_reference`` around the call alone, on its one thread. Reported: the sum of
those per-proof times (the sample proved on one thread), the pool's wall time (the sample
proved on every core), proofs/s for both, and whether every proof equals the C oracle's.
The batched sample is the bench's CPU sample (32 proofs, every 16th of the 512-proof stream
sorted by field and size, about 1/16 of its work); the served sample is every 1000th of the
20,000-request stream (seed 1) sorted by size, from the 500th on.

Writes ``oracle/reference_py_timings.json`` (host, CPU model, nproc, seconds, match).

    SUMCHECK_REFERENCE=<reference checkout> python oracle/time_reference_py.py [config ...]
"""

from __future__ import annotations

import json
import os
import platform
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sumcheck-triton_b200"))

OUT = HERE / "reference_py_timings.json"

# the three plain configurations, cheapest first
CONFIGS = ("plain_p32", "plain_bls", "plain_goldilocks")


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def from_mont(limbs, p: int, L: int) -> int:
    x = sum(int(w) << (32 * i) for i, w in enumerate(limbs))
    return x * pow(1 << (32 * L), -1, p) % p


def run(name: str, ref_src: Path) -> dict:
    sys.path.insert(0, str(ref_src))
    from zkduel.reference import sumcheck_reference  # the reference's own code
    from zkduel.workloads import WORKLOADS
    from zkduel._expr import expression_vars

    from oracle import c_oracle
    from oracle.oracle import indexed_terms

    from zkduel_b200.configs import PLAIN_CONFIGS
    from zkduel_b200.fields import get_field

    cfg = PLAIN_CONFIGS[name]
    spec = get_field(cfg.bit_width)
    workload, p, L, n, bern = cfg.workload, spec.modulus, spec.limbs, cfg.num_vars, cfg.bernoulli
    expr = WORKLOADS[workload]  # the reference's own expression
    names = expression_vars(expr)
    kinds = [1 if v in bern else 0 for v in names]  # SC_TABLE_BERNOULLI / SC_TABLE_UNIFORM
    tables = c_oracle.generate(p, L, kinds, n, cfg.seed)
    terms, k = indexed_terms(expr, names)
    t0 = time.perf_counter()
    want = c_oracle.prove(terms, k, p, L, tables, "sha3")
    c_s = time.perf_counter() - t0
    chals = [from_mont(want["challenges"][j], p, L) for j in range(n)]
    shifts = [1 << (32 * l) for l in range(L)]
    py_tables = {}
    for i, v in enumerate(names):
        acc = [0] * (1 << n)
        for l in range(L):
            plane = tables[i, l].tolist()
            s = shifts[l]
            acc = [a + w * s for a, w in zip(acc, plane)] if l else plane
        py_tables[v] = acc
    del tables
    t0 = time.perf_counter()
    claim0, evals = sumcheck_reference(py_tables, q=p, expression=expr, challenges=chals, num_rounds=n)
    ref_s = time.perf_counter() - t0
    got = [[int(x) for x in row] for row in evals]
    exp = [[from_mont(want["round_polys"][j][t], p, L) for t in range(want["round_polys"].shape[1])]
           for j in range(n)]
    match = got == exp and int(claim0) == from_mont(want["claim0"], p, L)
    return {"config": name, "workload": workload, "num_vars": n, "limbs": L, "tables": k,
            "reference_py_s": round(ref_s, 2), "reference_py_threads": 1,
            "c_oracle_s": round(c_s, 3), "c_oracle_threads": os.cpu_count(),
            "outputs_equal_c_oracle": bool(match)}


STREAMS = ("stream_batched", "stream_served")


def stream_sample(name: str):
    """(spec, bit width) of every proof in the named stream sample."""
    from zkduel_b200.streams import served_stream

    if name == "stream_batched":
        import bench  # the bench's own fixed CPU sample

        return [(sp, sp.bit_width) for sp in bench.cpu_sample_specs()]
    reqs = sorted(served_stream(20000, rate_per_s=1.0, seed=1), key=lambda r: (r.spec.num_vars, r.spec.index))
    return [(r.spec, 128) for r in reqs[500::1000]]


def _stream_worker(job):
    """One proof of a stream sample in a pool worker: C-oracle tables and SHA3 challenges,
    then the reference's ``sumcheck_reference`` timed alone; returns (index, seconds, equal)."""
    ref_src, spec, bw = job
    if ref_src not in sys.path:
        sys.path.insert(0, ref_src)
    from zkduel.reference import sumcheck_reference  # the reference's own code

    from oracle import c_oracle
    from oracle.oracle import indexed_terms
    from zkduel_b200.fields import get_field

    f = get_field(bw)
    p, L, n = f.modulus, f.limbs, spec.num_vars
    names = spec.var_names
    terms, k = indexed_terms(spec.expression, names)
    tables = c_oracle.generate(p, L, [0] * k, n, spec.seed)
    want = c_oracle.prove(terms, k, p, L, tables, "sha3", threads=1)
    chals = [from_mont(want["challenges"][j], p, L) for j in range(n)]
    shifts = [1 << (32 * l) for l in range(L)]
    py_tables = {}
    for i, v in enumerate(names):
        acc = tables[i, 0].tolist()
        for l in range(1, L):
            acc = [a + w * shifts[l] for a, w in zip(acc, tables[i, l].tolist())]
        py_tables[v] = acc
    del tables
    t0 = time.perf_counter()
    claim0, evals = sumcheck_reference(py_tables, q=p, expression=spec.expression, challenges=chals, num_rounds=n)
    sec = time.perf_counter() - t0
    got = [[int(x) for x in row] for row in evals]
    exp = [[from_mont(want["round_polys"][j][t], p, L) for t in range(want["round_polys"].shape[1])]
           for j in range(n)]
    return spec.index, sec, bool(got == exp and int(claim0) == from_mont(want["claim0"], p, L))


def run_stream(name: str, ref_src: Path) -> dict:
    import multiprocessing as mp

    sample = stream_sample(name)
    cores = os.cpu_count() or 1
    jobs = [(str(ref_src), sp, bw) for sp, bw in sorted(sample, key=lambda x: -x[0].num_vars)]  # longest first
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_stream_worker, jobs, chunksize=1)
    wall = time.perf_counter() - t0
    one = sum(sec for _i, sec, _ok in res)
    sizes = sorted(sp.num_vars for sp, _bw in sample)
    return {"config": name, "proofs": len(sample), "num_vars": [sizes[0], sizes[-1]],
            "fields": sorted({bw for _sp, bw in sample}),
            "reference_py_one_thread_s": round(one, 2), "reference_py_one_thread_proofs_per_s": len(sample) / one,
            "reference_py_pool_s": round(wall, 2), "reference_py_pool_proofs_per_s": len(sample) / wall,
            "pool_processes": cores, "host_cpu": cpu_model(), "nproc": cores,
            "timing": "per proof: sumcheck_reference alone in a pool worker (one thread); pool: wall time of the "
                      "whole sample including the C oracle's table generation and challenges",
            "outputs_equal_c_oracle": all(ok for _i, _s, ok in res)}


def main() -> int:
    ref = os.environ.get("SUMCHECK_REFERENCE")
    if not ref:
        print("set SUMCHECK_REFERENCE to the reference checkout", file=sys.stderr)
        return 2
    names = sys.argv[1:] or list(CONFIGS)
    doc = json.loads(OUT.read_text()) if OUT.exists() else {}
    doc.update({"host_cpu": cpu_model(), "nproc": os.cpu_count(), "python": platform.python_version(),
                "note": "reference.py timed single-threaded where the reference source lives (not the GPU host)"})
    results = doc.setdefault("configs", {})
    for name in names:
        r = run_stream(name, Path(ref) / "src") if name in STREAMS else run(name, Path(ref) / "src")
        results[name] = r
        OUT.write_text(json.dumps(doc, indent=1) + "\n")
        print(json.dumps(r), flush=True)
    return 0 if all(r["outputs_equal_c_oracle"] for r in results.values()) else 1


if __name__ == "__main__":
    sys.exit(main())
