"""The benchmark's JSON contract, checked on the CPU: the reference arm
(`bench.py --impl reference`, the CPU oracle frame on the host cores, no GPU)
prints one line with every key the contract names, and the helpers the GPU
arm uses for its roofline read the committed profiles."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

REQUIRED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config")


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in REQUIRED:
        assert k in d, k
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    assert d["higher_is_better"] is True and d["unit"] == "frames/s" and d["value"] > 0
    assert d["config"]["workload"] == bench.WORKLOAD and d["config"]["gaussians"] == 3_000_000
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    rc = d["reference_cpu_cull_sort"]
    assert ("ms" in rc and rc["ms"] > 0 and rc["visible"] > 0) or "unavailable" in rc


def test_roofline_traffic_from_profiles():
    t = bench.profiled_traffic("cull_visible_kernel", "cull_project_kernel")
    assert isinstance(t, int) and t > 0
    assert bench.profiled_traffic("cull_visible_kernel", "no_such_kernel") is None


def test_peaks_file():
    hbm, tflops, src = bench.load_peaks()
    assert hbm > 1000 and tflops > 100 and src in ("measured", "fallback")


@pytest.mark.parametrize("n", [10_000])
def test_reference_cull_sort_figure(n):
    from helpers import small_cam, small_rows

    r = bench.reference_cull_sort(small_rows(n, seed=5), small_cam(320, 180))
    assert ("ms" in r and r["threads"] == 1) or "unavailable" in r
