"""Index maps of the pitched SoA layout, checked on the CPU: tests/index_check.cu
includes the kernels' header, is built by nvcc as a host program and compares
CellMap (interior cell -> pitched index, multiply-high division) and soa_index
(dense padded cell -> pitched index) with plain loops."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_pitched_index_maps_match_plain_loops(tmp_path):
    exe = str(tmp_path / "index_check")
    src = os.path.join(ROOT, "tests", "index_check.cu")
    inc = ["-I", os.path.join(ROOT, "verona_b200", "csrc"), "-I", os.path.join(ROOT, "include")]
    r = subprocess.run([_nvcc(), "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-gencode",
                        "arch=compute_100a,code=sm_100a", *inc, src, "-o", exe], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
