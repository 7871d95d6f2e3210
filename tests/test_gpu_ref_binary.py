"""Full-size parity against the reference's own CUDA executable (GPU).

``oracle/Makefile.ref`` builds the reference's ``cuda/src/field_sumcheck.cu`` for sm_100a into
``oracle/_ref``. Where that binary is present, this test runs it and this library's drop-in
(``field_sumcheck_b200``) with the same arguments: both fill the tables with the reference's
arithmetic progressions, so their CSV checksums -- the sum over every run of the round
polynomials' Montgomery limbs -- must be equal, here at sizes far beyond the golden records.
"""

from __future__ import annotations

import csv
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "oracle" / "_ref" / "field_sumcheck_cuda"
CLI = ROOT / "sumcheck-triton_b200" / "bin" / "field_sumcheck_b200"

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a GPU", allow_module_level=True)


def _run(binary, args, out):
    subprocess.run([str(binary), *args, "--out", str(out)], check=True, stdout=subprocess.DEVNULL, timeout=900)
    return {(r["workload"], r["bit_width"], r["rounds"]): r["checksum"] for r in csv.DictReader(out.open())}


@pytest.mark.skipif(not REF.exists(), reason="reference executable not built (make -f oracle/Makefile.ref)")
@pytest.mark.parametrize("mode", ["sha3", "fixed"])
def test_checksums_equal_the_reference_executable(mode, tmp_path):
    args = ["--workloads", "poly_ab", "poly_abcg_plus_deg", "zk_vanilla_zerocheck_hp", "zk_jellyfish_permcheck_hp",
            "zk_opencheck", "--rounds", "14", "18", "--bit-widths", "32", "64", "128", "256", "--warmups", "1",
            "--repeats", "2", "--challenge-mode", mode, "--point-mode", "specialized"]
    ref = _run(REF, args, tmp_path / "ref.csv")
    ours = _run(CLI, args, tmp_path / "ours.csv")
    assert len(ref) == 5 * 2 * 4
    assert ours == ref
