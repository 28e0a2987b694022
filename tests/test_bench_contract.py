"""The benchmark's JSON contract, checked on the CPU: the reference arm
(`bench.py --impl reference`, the CPU oracle frame on the host cores, no GPU)
prints one line with every key the contract names and the same `config` as
the GPU arm, without loading libgs_cuda.so; its rows and cameras (made by the
reference's own loader and camera code) equal the GPU arm's; and the helpers
the GPU arm uses for its roofline read the committed profiles."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

REQUIRED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config")


# Runs bench.py as __main__ and then lists the shared objects of this repository
# that the process mapped: the reference arm must not load libgs_cuda.so.
_WRAP = """
import runpy, sys
sys.argv = ["bench.py"] + sys.argv[1:]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("MAPPED", sorted({l.split()[-1].rsplit("/", 1)[-1] for l in maps.splitlines() if l.endswith(".so")}))
"""


def test_reference_arm_line():
    out = subprocess.run([sys.executable, "-c", _WRAP, "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    mapped = [l for l in out.stdout.splitlines() if l.startswith("MAPPED")]
    assert mapped and "libgs_cuda.so" not in mapped[0], mapped
    d = json.loads(lines[0])
    assert d["config"] == bench.bench_config(3_000_000, 1)
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


def test_reference_inputs_equal_ours():
    """The reference arm's rows (gaussian_load_ply + pack_gpu_gaussians) and
    orbit cameras (src/camera.cpp + src/main.cpp:1264-1281, compiled from the
    reference sources) are bit-identical to the GPU arm's."""
    from oracle import oracle as O

    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    rows_ref, cams_ref = bench.reference_inputs(20_000)
    rows = bench.make_rows(20_000)
    assert np.array_equal(rows_ref.view(np.uint32), rows.view(np.uint32))
    cams = bench.orbit_cameras()
    assert len(cams) == len(cams_ref)
    for a, b in zip(cams, cams_ref):
        assert np.array_equal(np.asarray(a, np.float32).view(np.uint32), b.view(np.uint32))
