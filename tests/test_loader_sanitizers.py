"""The host loaders (gs_hosthelpers.cpp, gs_gsanim.cpp, gs_sog.cpp,
gs_webp.cpp) built with AddressSanitizer and UndefinedBehaviorSanitizer and
fed seeded mutations of valid PLY, SOG, gsanim and WebP files and of raw
archive bytes (tests/loader_fuzz.py): no sanitizer report, no crash.  CPU
only; skipped where g++ or the sanitizer runtimes are missing."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "gamesplat_b200" / "csrc"
SOURCES = ["gs_hosthelpers.cpp", "gs_gsanim.cpp", "gs_sog.cpp", "gs_webp.cpp"]


def runtime(name):
    try:
        out = subprocess.run(["g++", f"-print-file-name={name}"], capture_output=True, text=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    path = out.stdout.strip()
    return path if os.path.isabs(path) and os.path.exists(path) else None


@pytest.fixture(scope="module")
def sanitized_lib(tmp_path_factory):
    if shutil.which("g++") is None or not runtime("libasan.so") or not runtime("libubsan.so"):
        pytest.skip("g++ with ASan/UBSan runtimes not available")
    out = tmp_path_factory.mktemp("asan") / "libgs_host_asan.so"
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-fno-omit-frame-pointer", "-fPIC", "-shared", *[str(CSRC / s) for s in SOURCES], "-lz", "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]
    return out


@pytest.mark.parametrize("seed", [7, 8])
def test_loaders_under_sanitizers(sanitized_lib, seed):
    env = dict(os.environ)
    env["LD_PRELOAD"] = f"{runtime('libasan.so')}:{runtime('libubsan.so')}"
    env["ASAN_OPTIONS"] = "detect_leaks=0:abort_on_error=1"
    env["UBSAN_OPTIONS"] = "print_stacktrace=1:halt_on_error=1"
    res = subprocess.run([sys.executable, str(ROOT / "tests" / "loader_fuzz.py"), str(sanitized_lib), str(seed),
                          "1000"], capture_output=True, text=True, env=env, timeout=900)
    report = res.stderr[-4000:]
    assert res.returncode == 0, report
    assert "AddressSanitizer" not in res.stderr and "runtime error" not in res.stderr, report
    assert "accepted" in res.stdout
