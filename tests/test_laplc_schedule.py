"""The single-launch laplc's work order (mpg_laplc_schedule, host C++), compiled here with the
library's own setup.cpp and checked on doubly periodic column grids: every item once, every
gradient item a divergence item reads inside its ranges and earlier in the order (the condition
under which the kernel's waits always end)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc for the CUDA vector types")
def test_laplc_schedule_orders_dependencies(tmp_path):
    exe = tmp_path / "laplc_schedule_check"
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-x", "cu", os.path.join(HERE, "native", "laplc_schedule_check.cpp"),
                    os.path.join(ROOT, "src_b200", "csrc", "setup.cpp"), "-o", str(exe)],
                   check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0, r.stdout[-2000:]
    assert len(lines) == 4 * 4 * 2 * 2 and all(ln.endswith(" ok") for ln in lines)
