"""The command-line drop-in (GPU): the reference's validator invocation, checksums against the
reference's golden records.

``experiments/h100/tools/validate_cuda_vs_registry.py`` runs the executable with
``--warmups 0 --repeats 1`` per challenge mode and compares each CSV row's checksum (two runs
summed) with the registry; this test does the same with the golden records in tests/golden.
"""

from __future__ import annotations

import csv
import subprocess
from pathlib import Path

import pytest

CLI = Path(__file__).resolve().parents[1] / "sumcheck-triton_b200" / "bin" / "field_sumcheck_b200"

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)

WORKLOADS = ["poly_ab", "poly_aabbc", "poly_abcg_plus_deg", "zk_spartan_1", "zkphire_20", "zk_vanilla_permcheck_hp",
             "zk_jellyfish_zerocheck_hp", "zk_opencheck"]
ALIAS = {"zkphire_20": "zk_vanilla_zerocheck_hp"}


@pytest.mark.parametrize("mode", ["fixed", "sha3"])
@pytest.mark.parametrize("layout,point_mode", [("element", "specialized"), ("limb", "generic")])
def test_validator_invocation_matches_golden_checksums(mode, layout, point_mode, registry_records, tmp_path):
    assert CLI.exists(), "build sumcheck-triton_b200 first"
    names = {ALIAS.get(w, w) for w in WORKLOADS}
    ref = {(r["workload"], r["bit_width"], r["rounds"]): r["checksum_x2"] for r in registry_records
           if r["challenge_mode"] == mode and r["workload"] in names}
    rounds = sorted({k[2] for k in ref})
    out = tmp_path / "cuda.csv"
    subprocess.run([str(CLI), "--workloads", *WORKLOADS, "--bit-widths", "32", "64", "128", "256",
                    "--rounds", *map(str, rounds), "--warmups", "0", "--repeats", "1", "--challenge-mode", mode,
                    "--point-mode", point_mode, "--layout", layout, "--out", str(out)],
                   check=True, stdout=subprocess.DEVNULL)
    rows = list(csv.DictReader(out.open()))
    seen = 0
    for row in rows:
        key = (row["workload"], int(row["bit_width"]), int(row["rounds"]))
        assert row["status"] == "ok" and row["challenge_mode"] == mode
        assert int(row["limbs"]) * 32 >= int(row["bit_width"]) - 1
        if key in ref:
            assert int(row["checksum"]) == ref[key], key
            seen += 1
    assert seen == len(ref) and seen > 0


def test_csv_columns_and_timing_modes(tmp_path):
    out = tmp_path / "o.csv"
    subprocess.run([str(CLI), "--workloads", "poly_ab", "--bit-widths", "64", "--rounds", "12", "--warmups", "1",
                    "--repeats", "3", "--timing-mode", "round-sum", "--out", str(out)], check=True,
                   stdout=subprocess.DEVNULL)
    rows = list(csv.DictReader(out.open()))
    assert list(rows[0].keys()) == (
        "workload,polynomial,backend,field,arithmetic,layout,point_mode,bit_width,limbs,modulus_hex,rounds,N,vars,"
        "degree,terms,warmups,repeats,timing_mode,challenge_mode,first_ms,median_ms,eval_median_ms,"
        "challenge_median_ms,fold_median_ms,total_median_ms,input_mib,checksum,status").split(",")
    r = rows[0]
    assert r["field"] == "p64_goldilocks" and r["N"] == str(1 << 12) and r["vars"] == "2" and r["degree"] == "2"
    assert float(r["median_ms"]) > 0 and float(r["eval_median_ms"]) == float(r["median_ms"])
    assert float(r["input_mib"]) == pytest.approx(2 * 2 * 4 * (1 << 12) / 2**20)
