"""GPU parity of the sorted-alpha path through the C ABI (libgs_cuda.so):
cull/SH/project records, depth keys, cull mask and diagnostics bit-exact;
depth-sort permutation bit-exact; RGBA16F image within max-abs 2^-9 per
channel and PSNR >= 55 dB of the CPU oracle (FP32 composite, rounded once)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L
from gamesplat_b200 import renderer as RR
from gamesplat_b200 import scene
from oracle import oracle as O

from helpers import image_gate, oracle_alpha, small_cam, small_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    rows = small_rows()
    cam = small_cam()
    ref_img, ref = oracle_alpha(rows, cam, 1280, 720)
    return rows, cam, ref_img, ref


def make_renderer(rows, **knobs):
    r = Renderer(0)
    r.set(splat_render_mode="alpha", black_background=1, **knobs)
    r.upload_gaussians(rows)
    return r


def test_cull_records_keys_mask_bit_exact(small):
    rows, cam, _, ref = small
    with make_renderer(rows, write_invisible_records=1, splat_diagnostics_enabled=1) as r:
        r.draw_frame(cam)
        n = rows.shape[0]
        ids = r.debug_read(L.GS_DEBUG_IDS, n)
        keys = r.debug_read(L.GS_DEBUG_KEYS, n)
        proj = r.debug_read(L.GS_DEBUG_PROJECTED, n * 16, np.float32, (n, 16))
        st = r.stats()
    assert st.visible_count == ref["vc"]
    assert np.array_equal(ids, ref["ids"])
    assert np.array_equal(keys, ref["keys"])
    assert np.array_equal(proj.view(np.uint32), ref["proj"].view(np.uint32))
    assert list(st.diagnostics) == list(ref["diag"])


def test_depth_sort_permutation_bit_exact(small):
    rows, cam, _, ref = small
    with make_renderer(rows) as r:
        r.draw_frame(cam)
        n = rows.shape[0]
        si = r.debug_read(L.GS_DEBUG_SORTED_IDS, n)
        sk = r.debug_read(L.GS_DEBUG_SORTED_KEYS, n)
    ks, _ = O.sort_pairs(ref["keys"], ref["ids"])
    assert np.array_equal(si, ref["sorted_ids"])
    assert np.array_equal(sk, ks)


def test_alpha_image_parity_small(small):
    rows, cam, ref_img, _ = small
    with make_renderer(rows) as r:
        img = r.draw_frame(cam)
        img2 = r.draw_frame(cam)
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate
    assert np.array_equal(img.view(np.uint16), img2.view(np.uint16)), "frames must be deterministic"


@pytest.mark.parametrize("w,h", [(1, 1), (17, 9), (333, 211)])
def test_alpha_odd_sizes(w, h):
    rows = small_rows(20_000, seed=5)
    cam = small_cam(w, h)
    ref_img, _ = oracle_alpha(rows, cam, w, h)
    with make_renderer(rows) as r:
        img = r.draw_frame(cam)
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate


def test_alpha_4k_more_tiles_than_13_bits():
    """3840x2160: 32 400 tiles (15-bit tile ids: the tile sort's second pass
    has 7 bits), tile order over all of them."""
    w, h = 3840, 2160
    rows = small_rows(60_000, seed=9)
    cam = small_cam(w, h)
    ref_img, _ = oracle_alpha(rows, cam, w, h)
    with make_renderer(rows) as r:
        img = r.draw_frame(cam)
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate


def test_alpha_sh_degrees_and_grey_background():
    rows = small_rows(30_000, seed=9)
    cam = small_cam(320, 240)
    for deg in (0, 1, 2):
        ref_img, _ = oracle_alpha(rows, cam, 320, 240, black=False, sh_degree=deg)
        r = Renderer(0)
        r.set(splat_render_mode="alpha", black_background=0, sh_degree=deg)
        r.upload_gaussians(rows)
        img = r.draw_frame(cam)
        r.destroy()
        gate = image_gate(img, ref_img)
        assert gate["ok"], (deg, gate)


def test_nothing_visible():
    rows = small_rows(10_000, seed=1)
    cam = RR.camera_uniforms((0.0, 0.0, 3.0), 0.0, 0.0, 64, 48)   # looking away from the cloud
    with make_renderer(rows) as r:
        img = r.draw_frame(cam)
        st = r.stats()
    assert st.visible_count == 0 and st.tile_entries == 0
    assert np.all(img.astype(np.float32) == 0.0)


def test_single_gaussian_and_giant_splats_overflow_path():
    # 300 Gaussians just in front of the camera cover every tile of a 1080p
    # frame: 300 x 8160 entries exceed the initial entry capacity (1 Mi), so
    # the frame must grow the buffers and re-render.
    raw = scene.small_scene(11, 300)
    raw[:, 0:3] *= 0.05
    raw[:, 52:55] = 0.0   # scale e^0 = 1 m
    rows = RR.pack_raw(raw)
    cam = RR.camera_uniforms((0.0, 0.0, 1.2), float(np.pi), 0.0, 1920, 1080)
    ref_img, ref = oracle_alpha(rows, cam, 1920, 1080)
    with make_renderer(rows) as r:
        img = r.draw_frame(cam)
        st = r.stats()
    assert st.tile_overflow == 0 and st.tile_entries > (1 << 20)
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate
    one = rows[:1]
    ref1, _ = oracle_alpha(one, cam, 1920, 1080)
    with make_renderer(one) as r:
        img1 = r.draw_frame(cam)
    assert image_gate(img1, ref1)["ok"]


def test_overflowing_frame_through_stream_ordered_render():
    """gs_render (device output, the drop-in renderer_draw_frame path) on the
    giant-splat scene: the first frame's tile entries overflow the initial
    buffers, and gs_render must grow them and re-render before it returns
    GS_OK, so the image in device memory is the whole frame, not a truncated
    one."""
    import torch

    raw = scene.small_scene(11, 300)
    raw[:, 0:3] *= 0.05
    raw[:, 52:55] = 0.0
    rows = RR.pack_raw(raw)
    W, H = 1920, 1080
    cam = RR.camera_uniforms((0.0, 0.0, 1.2), float(np.pi), 0.0, W, H)
    ref_img, _ = oracle_alpha(rows, cam, W, H)
    out = torch.empty(W * H * 4, dtype=torch.float16, device="cuda")
    with make_renderer(rows) as r:
        for _ in range(2):   # the first call overflows and re-renders; the second fits
            out.fill_(float("nan"))
            r.draw_frame(cam, out_ptr=out.data_ptr())
            st = r.stats()
            assert st.tile_overflow == 0 and st.tile_entries > (1 << 20)
            img = out.view(H, W, 4).cpu().numpy()
            gate = image_gate(img, ref_img)
            assert gate["ok"], gate


def test_errors_are_status_codes():
    r = Renderer(0)
    cam = small_cam(64, 64)
    with pytest.raises(L.GsError) as e:
        r.draw_frame(cam)
    assert e.value.status == L.GS_ERR_NO_SCENE
    with pytest.raises(L.GsError) as e:
        r.upload_gaussians(np.zeros((0, 64), np.float32))
    assert e.value.status == L.GS_ERR_BAD_ARG
    r.upload_gaussians(small_rows(1000))
    bad = cam.copy()
    bad[32] = 0.0
    with pytest.raises(L.GsError) as e:
        r.draw_frame(bad)
    assert e.value.status == L.GS_ERR_BAD_ARG
    # viewports that are not finite or beyond 32767 pixels are refused before
    # any target is sized (the output buffer is never touched)
    buf = np.zeros(4, np.float16)
    for v, status in ((float("nan"), L.GS_ERR_BAD_ARG), (-5.0, L.GS_ERR_BAD_ARG), (0.49, L.GS_ERR_BAD_ARG),
                      (float("inf"), L.GS_ERR_TOO_LARGE), (1e10, L.GS_ERR_TOO_LARGE), (32767.6, L.GS_ERR_TOO_LARGE)):
        for axis in (32, 33):
            bad = cam.copy()
            bad[axis] = v
            cc = RR.camera_from_array(bad)
            assert L.lib().gs_render_host(r._ctx, C.byref(cc), buf.ctypes.data) == status, (axis, v)
    assert r.draw_frame(cam).shape == (64, 64, 4)
    assert r.set_gps_work_budget(0) is False
    assert r.set_gps_work_budget(1 << 16) is True
    r.destroy()


@pytest.mark.parametrize("frame", [0, 37])
def test_alpha_room3m_1080p_full_size(frame):
    """The benchmark workload itself (3M SH3 Gaussians, 1920x1080 orbit)."""
    raw = scene.room_scene(1)
    rows = RR.pack_raw(raw)
    del raw
    pos, yaw, pitch = scene.orbit_pose(frame)
    cam = RR.camera_uniforms(pos, yaw, pitch, 1920, 1080)
    ref_img, ref = oracle_alpha(rows, cam, 1920, 1080)
    with make_renderer(rows) as r:
        img = r.draw_frame(cam)
        st = r.stats()
        n = rows.shape[0]
        si = r.debug_read(L.GS_DEBUG_SORTED_IDS, n)
    assert st.visible_count == ref["vc"]
    assert np.array_equal(si, ref["sorted_ids"])
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate
