"""Native pieces of the Stage-1 producer, built with g++ from the product's
own source: the persistent worker pool (calig.cpp WorkerPool, behind
pool_run: back-to-back jobs of varied sizes, each task run exactly once and
before its job returns) and the batched sorted-set edits (insert_run,
erase_run) against the standard library's set algorithms, and the task-queue
dedupe at 1, 3 and 8 threads against sort + unique."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cgbdsm_b200", "csrc")


def _build(tmp_path, name, *sources):
    exe = str(tmp_path / name)
    subprocess.run(
        ["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
         os.path.join(ROOT, "tests", "native", name + ".cpp"), *sources, "-o", exe],
        check=True)
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_pool_runs_every_task_once(tmp_path):
    exe = _build(tmp_path, "pool_stress", os.path.join(CSRC, "calig.cpp"))
    out = subprocess.run([exe, "50000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad=0" in out.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_sorted_set_runs_match_set_algorithms(tmp_path):
    exe = _build(tmp_path, "sorted_runs")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad=0" in out.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_serving_staging_ring(tmp_path):
    """The serving loop's staging ring (FIFO allocate / release of edge-pair
    blocks, wrapping at the end): live blocks inside the ring and disjoint,
    all space back when every block is released."""
    exe = _build(tmp_path, "staging_ring")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad=0" in out.stdout and "wraps=0" not in out.stdout
