"""The reference arm of bench.py runs on host cores only: its JSON line keeps
the benchmark contract (one line, the headline metric and unit, the CPU
baseline it timed, an e2e object with no host-device traffic)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-seconds", "0.5"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("zone-updates/s") and d["unit"] == "zone-updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_tensor_roofline_of_the_learned_kernel():
    sys.path.insert(0, ROOT)
    import bench

    r = bench.tensor_roofline(512**3, 16.1, 8.6, True)
    assert r["bound"] == "tensor" and r["flop_per_cell"] == 17024
    assert abs(r["kernel_ms_per_launch"] - 7.5) < 1e-9
    assert abs(r["achieved"] - 17024 * 512**3 / 7.5e-3 / 1e12) < 1e-6
    assert 0 < r["frac"] < 1
    assert bench.tensor_roofline(512**3, 16.1, 8.6, False) is None
    assert bench.tensor_roofline(512**3, 8.0, 8.6, True) is None
