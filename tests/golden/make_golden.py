"""Regenerates the golden fixtures of this directory from the reference itself.

Run in a container that has the reference tree (it is read, never modified):

    python tests/golden/make_golden.py --reference <reference checkout>

It writes three files; the tests only read them:

* ``registry_checksums.jsonl`` -- every distinct golden record of the reference's
  validation runs (``experiments/h100/validation/*.jsonl``): workload, width, rounds,
  challenge mode and the reference checksum of two runs. Duplicates across files are
  checked for agreement.
* ``reference_outputs.jsonl`` -- ``(claim0, round_evals)`` of the reference's own
  ``sumcheck_reference`` (``src/zkduel/reference.py``) on explicit seeded tables and
  challenges, for all 32 kernel workloads at every field width, plus the reference's
  own pytest cases (``tests/test_zkduel.py``: tables from ``random.Random(seed)``).
* ``guard_cases.jsonl`` -- moduli the reference's guard accepts or rejects
  (``src/zkduel/fields.py``), with the exception text.
"""

from __future__ import annotations

import argparse
import glob
import json
import random
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "sumcheck-triton_b200"))

from zkduel_b200.workloads import KERNEL_WORKLOADS  # noqa: E402


def registry_records(ref: Path) -> list[dict]:
    seen: dict[tuple, dict] = {}
    for f in sorted(glob.glob(str(ref / "experiments/h100/validation/*.jsonl"))):
        for line in open(f):
            line = line.strip()
            if not line:
                continue
            r = json.loads(line)
            if r.get("match") is not True:
                continue
            key = (r["workload"], int(r["bit_width"]), int(r["rounds"]), r["challenge_mode"])
            val = int(r["reference_checksum"])
            if key in seen:
                assert seen[key]["checksum_x2"] == val, (key, f)
                seen[key]["sources"].append(Path(f).name)
            else:
                seen[key] = {
                    "workload": key[0],
                    "bit_width": key[1],
                    "rounds": key[2],
                    "challenge_mode": key[3],
                    "seed": 1 + key[2],
                    "runs": 2,
                    "checksum_x2": val,
                    "sources": [Path(f).name],
                }
    return [seen[k] for k in sorted(seen)]


def reference_outputs(ref_mod, fields_mod) -> list[dict]:
    out = []
    rng = random.Random(20261203)
    for bw in (32, 64, 128, 256):
        q = fields_mod.get_field(bw).modulus
        for w in KERNEL_WORKLOADS:
            expr = ref_mod_workload(w.registry_name)
            names = ref_vars(expr)
            n = 3 if (bw <= 64 and len(names) <= 12) else 2
            tables = {v: [rng.randrange(q) for _ in range(1 << n)] for v in names}
            chals = [rng.randrange(q) for _ in range(n)]
            claim, evals = ref_mod.sumcheck_reference(
                tables, q=q, expression=expr, challenges=chals, num_rounds=n
            )
            out.append(
                {
                    "case": f"{w.name}_bw{bw}_n{n}",
                    "workload": w.registry_name,
                    "bit_width": bw,
                    "q": q,
                    "num_rounds": n,
                    "tables": tables,
                    "challenges": chals,
                    "claim0": int(claim),
                    "evals": [[int(x) for x in row] for row in evals.tolist()],
                }
            )
    # larger cases for the hot shapes, and the reference's own pytest cases
    for name, bw, n in (("poly_ab", 32, 8), ("vanilla_zerocheck_hp", 64, 6),
                        ("poly_abcg_plus_deg", 256, 6), ("jellyfish_zerocheck_hp", 128, 4)):
        q = fields_mod.get_field(bw).modulus
        expr = ref_mod_workload(name)
        tables = {v: [rng.randrange(q) for _ in range(1 << n)] for v in ref_vars(expr)}
        chals = [rng.randrange(q) for _ in range(n)]
        claim, evals = ref_mod.sumcheck_reference(
            tables, q=q, expression=expr, challenges=chals, num_rounds=n
        )
        out.append(
            {"case": f"{name}_bw{bw}_n{n}", "workload": name, "bit_width": bw, "q": q,
             "num_rounds": n, "tables": tables, "challenges": chals, "claim0": int(claim),
             "evals": [[int(x) for x in row] for row in evals.tolist()]}
        )
    ladder = ["poly_a", "poly_ab", "poly_ab_plus_c", "poly_abc", "poly_aabbc",
              "poly_abc_plus_de", "poly_abcg_plus_deg"]
    q = fields_mod.get_field(256).modulus
    for name in ladder:
        for rounds, seed in ((4, 11), (2, 256)):
            expr = ref_mod_workload(name)
            r1 = random.Random(seed)
            tables = {v: [r1.randrange(q) for _ in range(1 << rounds)] for v in ref_vars(expr)}
            r2 = random.Random(seed + 99)
            chals = [r2.randrange(q) for _ in range(rounds)]
            claim, evals = ref_mod.sumcheck_reference(
                tables, q=q, expression=expr, challenges=chals, num_rounds=rounds
            )
            out.append(
                {"case": f"pytest_{name}_r{rounds}_s{seed}", "workload": name, "bit_width": 256,
                 "q": q, "num_rounds": rounds, "tables": tables, "challenges": chals,
                 "claim0": int(claim), "evals": [[int(x) for x in row] for row in evals.tolist()]}
            )
    return out


def guard_cases(fields_mod) -> list[dict]:
    cases = []
    trial = [
        (0xFFFFFFFB, 1), (0xFFFFFFFF00000001, 2), ((1 << 127) - 1, 4),
        (fields_mod.get_field(256).modulus, 8), ((1 << 31) - 1, 1), ((1 << 61) - 1, 2),
        ((1 << 89) - 1, 3), ((1 << 255) - 19, 8), ((1 << 64) - 59, 2), ((1 << 128) - 159, 4),
        (0xFFFFFFFF00000001 + 2, 2), ((1 << 61) - 2, 2), ((1 << 64) + 13, 2),
    ]
    for p, L in trial:
        nprime = fields_mod.montgomery_nprime(p) if p % 2 else 1
        try:
            fields_mod.check_montgomery_modulus(p, L, nprime)
            cases.append({"modulus": p, "limbs": L, "nprime": nprime, "accepted": True})
        except fields_mod.UnsafeModulusError as exc:
            cases.append({"modulus": p, "limbs": L, "nprime": nprime, "accepted": False,
                          "error": str(exc)})
    p = (1 << 61) - 1
    try:
        fields_mod.check_montgomery_modulus(p, 2, 0x12345)
    except fields_mod.UnsafeModulusError as exc:
        cases.append({"modulus": p, "limbs": 2, "nprime": 0x12345, "accepted": False,
                      "error": str(exc)})
    return cases


_REF = {}


def ref_mod_workload(name):
    return _REF["workloads"].get_workload(name)


def ref_vars(expr):
    return _REF["expr"].expression_vars(expr)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True, help="the reference checkout")
    args = ap.parse_args()
    sys.path.insert(0, str(args.reference / "src"))
    import zkduel._expr as ref_expr
    import zkduel.fields as ref_fields
    import zkduel.reference as ref_reference
    import zkduel.workloads as ref_workloads

    _REF.update(workloads=ref_workloads, expr=ref_expr)
    with open(HERE / "registry_checksums.jsonl", "w") as f:
        for r in registry_records(args.reference):
            f.write(json.dumps(r) + "\n")
    with open(HERE / "reference_outputs.jsonl", "w") as f:
        for r in reference_outputs(ref_reference, ref_fields):
            f.write(json.dumps(r) + "\n")
    with open(HERE / "guard_cases.jsonl", "w") as f:
        for r in guard_cases(ref_fields):
            f.write(json.dumps(r) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
