"""The reference executable's command line (CPU side): argument errors exit 2 before any
device work, as cuda/src/field_sumcheck.cu:1108-1176 does."""

from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

CLI = Path(__file__).resolve().parents[1] / "sumcheck-triton_b200" / "bin" / "field_sumcheck_b200"

pytestmark = pytest.mark.skipif(not CLI.exists(), reason="command-line tool not built (sumcheck-triton_b200/build.py)")


@pytest.mark.parametrize("argv", [
    ["--bogus"],
    ["--block", "3"],
    ["--block", "0"],
    ["--timing-mode", "sometimes"],
    ["--challenge-mode", "random"],
    ["--layout", "diagonal"],
    ["--point-mode", "cubic"],
    ["--timer", "sundial"],
    ["--warmups"],
    ["--rounds", "x"],
    ["--rounds", "0"],
])
def test_bad_arguments_exit_2(argv, tmp_path):
    r = subprocess.run([str(CLI), *argv, "--out", str(tmp_path / "o.csv")], capture_output=True, text=True)
    assert r.returncode == 2, (r.returncode, r.stderr)
    assert r.stderr.strip()
