"""Device helpers checked on the CPU: each check includes the kernels' headers,
is built by nvcc as a host program and prints "ok".
- tests/index_check.cu: the index maps of the pitched SoA layout, CellMap
  (interior cell -> pitched index, multiply-high division) and soa_index
  (dense padded cell -> pitched index), against plain loops.
- tests/c2pw_check.cu: the W Newton of the learned guess (c2p_w) and its
  bracketed fallback, against P -> U -> P round trips.
- tests/qdiv_check.cu: the FP64 zero-dividend forms (qdiv, qdiv_pos, qsqrt)
  against the IEEE divide and square root (also run on the device)."""
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


def _build_and_run(tmp_path, name, *args):
    exe = str(tmp_path / name)
    src = os.path.join(ROOT, "tests", name + ".cu")
    inc = ["-I", os.path.join(ROOT, "verona_b200", "csrc"), "-I", os.path.join(ROOT, "include")]
    r = subprocess.run([_nvcc(), "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-gencode",
                        "arch=compute_100a,code=sm_100a", *inc, src, "-o", exe], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([exe, *args], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_pitched_index_maps_match_plain_loops(tmp_path):
    _build_and_run(tmp_path, "index_check")


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_w_newton_and_its_bracketed_fallback_recover_the_state(tmp_path):
    """The bracketed phase alone (max_newton = 0) must solve every cell; an
    earlier form evaluated its residual with a loop counter in place of
    (gamma - 1) / gamma and missed the root by up to 5e-4 of U."""
    _build_and_run(tmp_path, "c2pw_check")


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_zero_dividend_forms_match_ieee_on_the_host(tmp_path):
    """qdiv / qdiv_pos / qsqrt (the FP64 divide and square root with a zero
    kept out of the IEEE sequence) equal a / b and sqrt(a) bit for bit over
    signed zeros, subnormals, infinities and NaN, apart from the documented
    zero over a divisor of magnitude at most 2^-1024."""
    _build_and_run(tmp_path, "qdiv_check")


@pytest.mark.gpu
@pytest.mark.skipif(_nvcc() is None, reason="nvcc not found")
def test_zero_dividend_forms_match_ieee_on_the_device(tmp_path):
    """The same comparisons in a kernel: the GPU's IEEE divide and square
    root against the forms with the opaque move that the device code uses."""
    _build_and_run(tmp_path, "qdiv_check", "device")
