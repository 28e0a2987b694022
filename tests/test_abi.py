"""CPU tests of the C ABI boundary: the library loads without a GPU, exports
every function include/gs_api.h declares, and its host-only helpers and
error paths behave (no compute calls here)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from gamesplat_b200 import _lib as L

HEADER = Path(__file__).resolve().parents[1] / "include" / "gs_api.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = L.lib()
    decl = declared_functions()
    assert len(decl) >= 20
    missing = [f for f in decl if not hasattr(lib, f)]
    assert not missing, missing
    assert set(decl) == set(L.EXPORTS)


def test_struct_layouts_match_header():
    assert C.sizeof(L.GsCamera) == 160
    assert C.sizeof(L.GsKnobs) == 64
    assert C.sizeof(L.GsStats) == 4 * (4 + 8 + 12)


def test_status_strings():
    lib = L.lib()
    for s in range(-9, 1):
        assert lib.gs_status_str(s) != b"unknown status"
    assert lib.gs_status_str(-99) == b"unknown status"


def test_create_without_gpu_reports_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    ctx = C.c_void_p()
    st = L.lib().gs_create(C.byref(ctx), 0, None)
    assert st == L.GS_ERR_NO_DEVICE and not ctx


def test_null_arguments_rejected():
    lib = L.lib()
    assert lib.gs_render(None, None, None) == L.GS_ERR_BAD_ARG
    assert lib.gs_upload_rows(None, None, 0) == L.GS_ERR_BAD_ARG
    assert lib.gs_set_gps_budget(None, 5) == L.GS_ERR_BAD_ARG
    lib.gs_destroy(None)
    assert lib.gs_pack_raw(None, 3, None) == L.GS_ERR_BAD_ARG
    assert lib.gs_load_ply(b"/nonexistent.ply", None, 0) == L.GS_ERR_BAD_ARG
    assert lib.gs_sort_pairs(None, None, None, None, 10, 0, 32, None, 0, None) == L.GS_ERR_BAD_ARG
    assert lib.gs_sort_pairs(None, None, None, None, 0, 0, 32, None, 0, None) == L.GS_OK


def test_every_context_entry_rejects_a_null_context():
    """No entry point dereferences a null context or handle (CPU: none of
    these reach the device)."""
    lib = L.lib()
    bad = L.GS_ERR_BAD_ARG
    calls = {
        "gs_render_host": (None, None, None), "gs_render_host_submit": (None, None, None),
        "gs_render_host_wait": (None, None), "gs_upload_rows_device": (None, None, 0),
        "gs_upload_rows_range": (None, None, 0, 0), "gs_upload_anim": (None, None, 0, None),
        "gs_set_anim_state": (None, 0, 0, 0.0), "gs_upload_layers": (None, None, 0),
        "gs_set_layer_weights": (None, None, 0), "gs_get_knobs": (None, None), "gs_set_knobs": (None, None),
        "gs_set_mode": (None, 0), "gs_reset_accumulation": (None,), "gs_set_display_lut": (None, None, 0, 0.0, 1.0),
        "gs_display": (None, None, None, 1, 1, 0.0), "gs_read_stats": (None, None),
        "gs_debug_read": (None, 0, None, 0), "gs_profile_enable": (None, 1),
        "gs_stage_times": (None, None, None, 0, 0), "gs_debug_wait_probe": (None, 0, 1),
        "gs_gsanim_load": (b"x.gsanim", None), "gs_gsanim_get_info": (None, None), "gs_gsanim_rows": (None, None),
        "gs_gsanim_deltas": (None, None, None), "gs_gsanim_layer_data": (None, None),
        "gs_gsanim_display_lut": (None, None), "gs_gsanim_layer_name": (None, 0, None, 0),
        "gs_gsanim_sample": (None, 0.0, None, None, None), "gs_gsanim_layer_weights": (None, 0.0, None),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(*args) == bad, name
    assert lib.gs_last_error(None) == b"null context"
    lib.gs_gsanim_free(None)


def test_sort_scratch_size_grows_with_n():
    lib = L.lib()
    a, b = lib.gs_sort_pairs_scratch_bytes(1000), lib.gs_sort_pairs_scratch_bytes(1_000_000)
    assert 0 < a < b and b >= 8 * 1_000_000


def test_malformed_ply_rejected(tmp_path):
    p = tmp_path / "bad.ply"
    p.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\nend_header\n1\n2\n")
    assert L.lib().gs_load_ply(str(p).encode(), None, 0) == L.GS_ERR_BAD_ARG
    p.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 2\nproperty float y\nend_header\n")
    assert L.lib().gs_load_ply(str(p).encode(), None, 0) == L.GS_ERR_BAD_ARG
    p.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\nproperty float y\n"
                  b"property float z\nend_header\n" + np.zeros(3, np.float32).tobytes())
    rows = np.empty((4, 64), np.float32)
    assert L.lib().gs_load_ply(str(p).encode(), rows.ctypes.data, 4) == L.GS_ERR_BAD_ARG   # short read


C_CONSUMER = r"""
#include <stdio.h>
#include <stdlib.h>
#include "gs_api.h"

int main(int argc, char** argv) {
    gs_gsanim* a = NULL;
    if (gs_gsanim_load(argv[1], &a) != GS_OK) return 10;
    gs_gsanim_info info;
    if (gs_gsanim_get_info(a, &info) != GS_OK) return 11;
    float* rows = (float*)malloc((size_t)info.gaussian_count * 64 * sizeof(float));
    if (gs_gsanim_rows(a, rows) != GS_OK) return 12;
    int32_t sa, sb;
    float w;
    gs_gsanim_sample(a, 2.75, &sa, &sb, &w);
    printf("%u %u %u %d %d %.9g %.9g %zu\n", info.version, info.gaussian_count, info.state_count, sa, sb,
           (double)w, (double)rows[4], sizeof(gs_gsanim_info));
    gs_gsanim_free(a);
    int64_t n = gs_load_sog(argv[2], NULL, 0);
    if (n <= 0) return 13;
    float* srows = (float*)malloc((size_t)n * 64 * sizeof(float));
    if (gs_load_sog(argv[2], srows, (uint64_t)n) != n) return 14;
    printf("%lld %.9g\n", (long long)n, (double)srows[8]);
    printf("%d\n", gs_gsanim_load("/nonexistent.gsanim", &a));
    free(rows);
    free(srows);
    return 0;
}
"""


def test_c_consumer_of_the_header(tmp_path):
    """The header is plain C: a C99 program includes it, links the library
    and reads a gsanim and a SOG archive through the host entry points."""
    import shutil
    import subprocess

    from tests import gsanim_fixture as F
    from tests import sog_fixture as S

    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    m, b, s, d = F.v01_asset(n=4, states=3, seed=30, interpolation="linear")
    ga = F.pack(tmp_path / "a.gsanim", F.entries_v01(m, b, s, d))
    meta, imgs = S.sog_asset(5, seed=31)
    so = S.pack(tmp_path / "a.sog", S.entries(meta, imgs))
    src = tmp_path / "consumer.c"
    src.write_text(C_CONSUMER)
    exe = tmp_path / "consumer"
    lib_dir = L.LIB_PATH.parent
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(HEADER.parent), str(src), "-o", str(exe),
                    "-L", str(lib_dir), "-lgs_cuda", f"-Wl,-rpath,{lib_dir}"], check=True)
    out = subprocess.run([str(exe), str(ga), str(so)], capture_output=True, text=True, check=True).stdout.split("\n")
    from gamesplat_b200 import load_gsanim, load_sog

    a = load_gsanim(ga)
    version, n, states, sa, sb, w, scale0, info_size = out[0].split()
    assert (int(version), int(n), int(states)) == (1, 4, 3)
    assert (int(sa), int(sb), np.float32(w)) == tuple(a.sample(2.75)[:2]) + (np.float32(a.sample(2.75)[2]),)
    assert np.float32(scale0) == a.rows[0, 4]
    assert int(info_size) == C.sizeof(L.GsGsanimInfo)
    n_sog, q0 = out[1].split()
    rows = load_sog(so)
    assert int(n_sog) == rows.shape[0] and np.float32(q0) == rows[0, 8]
    assert int(out[2]) == L.GS_ERR_FORMAT
    a.close()


def test_asset_example_compiles(tmp_path):
    """The asset-loading example (tests/examples/load_asset.cpp, the host
    code the integration notes show) compiles against gs_api.h."""
    import shutil
    import subprocess

    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    src = Path(__file__).resolve().parent / "examples" / "load_asset.cpp"
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I", str(HEADER.parent),
                    str(src)], check=True)
