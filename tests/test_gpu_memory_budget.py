"""GPU: the memory-budget refusals of renderer_upload_gaussians
(src/renderer.cpp:739-763) and renderer_set_gps_work_budget (:1080-1092).
Uploads beyond gpu_budget_mb or beyond 4/5 of the free device memory are
refused with GS_ERR_TOO_LARGE before anything is allocated, and the resident
scene, animation and GPS buffer stay usable; the same context then renders
within the alpha-path gate of the CPU oracle."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L

from helpers import image_gate, oracle_alpha, small_cam, small_rows

pytestmark = pytest.mark.gpu

W, H = 320, 180
N = 100_000


def refused(fn, *args, status=L.GS_ERR_TOO_LARGE):
    with pytest.raises(L.GsError) as e:
        fn(*args)
    assert e.value.status == status, e.value
    return str(e.value)


def test_gpu_budget_cap():
    rows = small_rows(N)
    cam = small_cam(W, H)
    ref_img, _ = oracle_alpha(rows, cam, W, H)
    need = L.lib().gs_scene_device_bytes(N, 16 << 20)
    assert need % (1 << 20) != 0
    mb = need >> 20
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1, gpu_budget_mb=mb)
        msg = refused(r.upload_gaussians, rows)
        assert "budget" in msg
        refused(r.draw_frame, cam, status=L.GS_ERR_NO_SCENE)

        r.set(gpu_budget_mb=mb + 1)
        r.upload_gaussians(rows)
        img = r.draw_frame(cam)
        assert image_gate(img, ref_img)["ok"]

        # a larger scene is refused and the resident one stays
        refused(r.upload_gaussians, small_rows(2 * N, seed=1))
        assert np.array_equal(r.draw_frame(cam).view(np.uint16), img.view(np.uint16))

        # animation and layers beyond the cap are refused
        deltas = np.zeros((2, N, 48), np.int8)
        scales = np.ones(48, np.float32)
        refused(r.upload_animation, deltas, scales)
        refused(r.upload_layers, np.zeros((1, N, 48), np.uint16))

        # a larger GPS work buffer is refused, a smaller one accepted
        assert r.set_gps_work_budget(32 << 20) is False
        assert r.set_gps_work_budget(8 << 20) is True
        assert np.array_equal(r.draw_frame(cam).view(np.uint16), img.view(np.uint16))

        # without the cap all of them fit
        r.set(gpu_budget_mb=0)
        r.upload_animation(deltas, scales)
        r.upload_layers(np.zeros((1, N, 48), np.uint16))
        assert r.set_gps_work_budget(32 << 20) is True
        assert image_gate(r.draw_frame(cam), ref_img)["ok"]


def test_free_memory_budget():
    """2^30 - 1 Gaussians need ~530 GB, beyond 4/5 of any B200's free memory:
    refused before any allocation (the row pointer is never read)."""
    need = L.lib().gs_scene_device_bytes((1 << 30) - 1, 16 << 20)
    assert need > 500e9
    tiny = np.zeros((1, 64), np.float32)
    with Renderer(0) as r:
        st = L.lib().gs_upload_rows(r._ctx, tiny.ctypes.data, (1 << 30) - 1)
        assert st == L.GS_ERR_TOO_LARGE
        assert b"budget" in L.lib().gs_last_error(r._ctx)
        r.set(splat_render_mode="alpha", black_background=1)
        rows = small_rows(20_000, seed=3)
        r.upload_gaussians(rows)
        cam = small_cam(W, H)
        ref_img, _ = oracle_alpha(rows, cam, W, H)
        assert image_gate(r.draw_frame(cam), ref_img)["ok"]
