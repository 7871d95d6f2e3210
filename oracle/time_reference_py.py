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
        r = run(name, Path(ref) / "src")
        results[name] = r
        OUT.write_text(json.dumps(doc, indent=1) + "\n")
        print(json.dumps(r), flush=True)
    return 0 if all(r["outputs_equal_c_oracle"] for r in results.values()) else 1


if __name__ == "__main__":
    sys.exit(main())
