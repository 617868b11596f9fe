"""The device plan's shape tables checked on the host (tests/cpp/plan_tables.cpp): scanned and
expanded as the plan kernels do, they give exactly the node list, launch lists and size-1
positions of a direct per-bucket expansion of the RecSplit trees (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "shockhash_b200", "csrc")


def test_plan_tables_match_direct_expansion(tmp_path):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "plan_tables")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                    "-x", "cu", os.path.join(ROOT, "tests", "cpp", "plan_tables.cpp"),
                    "-x", "cu", os.path.join(CSRC, "shg_plan.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
