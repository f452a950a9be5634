"""The Stage-1 producer's persistent worker pool (calig.cpp WorkerPool, behind
pool_run): back-to-back jobs of varied sizes, each task run exactly once and
before its job returns.  Built with g++ from the product's own source."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cgbdsm_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_pool_runs_every_task_once(tmp_path):
    exe = str(tmp_path / "pool_stress")
    subprocess.run(
        ["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
         os.path.join(ROOT, "tests", "native", "pool_stress.cpp"), os.path.join(CSRC, "calig.cpp"),
         "-o", exe],
        check=True)
    out = subprocess.run([exe, "50000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad=0" in out.stdout
