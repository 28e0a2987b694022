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
    for s in range(-8, 1):
        assert lib.gs_status_str(s)
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
