"""gs_render_host readback paths give the same image as gs_render: a
page-locked destination (alpha mode: the rasterizer writes the pixels into
it through its mapped device address; other modes: one copy into it) and a
pageable destination (chunked copy through pinned staging, overlapped with
the host copy), at sizes that are not multiples of the tile size; and the
streamed readback (gs_render_host_submit / gs_render_host_wait), frame by
frame."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from gamesplat_b200 import Renderer, _lib as L
from gamesplat_b200.renderer import camera_from_array, camera_uniforms

from helpers import small_cam, small_rows

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h,mode", [(320, 180, "alpha"), (333, 211, "alpha"), (64, 17, "alpha"),
                                      (200, 120, "stochastic"), (200, 120, "gps")])
def test_readback_paths_agree(w, h, mode):
    rows = small_rows(20_000, seed=13)
    cam = small_cam(w, h)
    camc = camera_from_array(cam)
    with Renderer(0) as r:
        r.set(splat_render_mode=mode, black_background=1, stochastic_taa_enabled=0,
              stochastic_accumulation_enabled=0)
        r.upload_gaussians(rows)
        dev = torch.empty((h, w, 4), dtype=torch.float16, device="cuda")
        r.draw_frame(cam, out_ptr=dev.data_ptr())
        torch.cuda.synchronize()
        ref = dev.cpu().numpy()
        pinned = torch.empty((h, w, 4), dtype=torch.float16, pin_memory=True)
        pageable = np.empty((h, w, 4), np.float16)
        for _ in range(2):   # twice: the second call reuses the staging buffer and events
            L.check(L.lib().gs_render_host(r._ctx, C.byref(camc), pinned.data_ptr()), "gs_render_host")
            L.check(L.lib().gs_render_host(r._ctx, C.byref(camc), pageable.ctypes.data), "gs_render_host")
            if mode == "alpha":
                assert np.array_equal(pinned.numpy().view(np.uint16), ref.view(np.uint16))
                assert np.array_equal(pageable.view(np.uint16), ref.view(np.uint16))
            else:
                # stochastic and GPS frames change with the frame seed: check
                # both destinations hold complete frames
                for img in (pinned.numpy().astype(np.float32), pageable.astype(np.float32)):
                    assert np.isfinite(img).all()
                    assert img[..., 3].min() >= 0.0 and img[..., 3].max() <= 1.0
                    assert (img[..., 3] > 0).mean() > 0.05


def _cams(sizes):
    """A camera per frame, each from another position near (0, 0, 3)."""
    return [camera_uniforms((0.05 * i, 0.02 * i, 3.0), np.pi, 0.0, w, h) for i, (w, h) in enumerate(sizes)]


def test_streamed_readback_matches_gs_render():
    """gs_render_host_submit / gs_render_host_wait: every frame's image lands in
    its own page-locked buffer bit-identical to gs_render's, with two frames
    in flight, a viewport change mid-stream and a buffer reused at once."""
    rows = small_rows(20_000, seed=14)
    sizes = [(320, 180)] * 4 + [(333, 211)] * 3
    cams = _cams(sizes)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        refs = []
        for cam, (w, h) in zip(cams, sizes):
            dev = torch.empty((h, w, 4), dtype=torch.float16, device="cuda")
            r.draw_frame(cam, out_ptr=dev.data_ptr())
            torch.cuda.synchronize()
            refs.append(dev.cpu().numpy())
        bufs = [torch.full((h, w, 4), float("nan"), dtype=torch.float16, pin_memory=True) for w, h in sizes]
        for cam, buf in zip(cams, bufs):
            r.submit_frame(cam, buf)
        r.wait_frames()
        for k, (buf, ref) in enumerate(zip(bufs, refs)):
            assert np.array_equal(buf.numpy().view(np.uint16), ref.view(np.uint16)), k
        # the same buffer twice in a row: the second frame is what it holds
        one = torch.empty((180, 320, 4), dtype=torch.float16, pin_memory=True)
        r.submit_frame(cams[0], one)
        r.submit_frame(cams[3], one)
        r.wait_frames(one)
        assert np.array_equal(one.numpy().view(np.uint16), refs[3].view(np.uint16))
        r.wait_frames(one)   # nothing in flight for it: returns at once


def test_streamed_readback_refuses_pageable_memory():
    rows = small_rows(5_000, seed=15)
    cam = small_cam(64, 48)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        pageable = np.empty((48, 64, 4), np.float16)
        assert L.lib().gs_render_host_submit(r._ctx, C.byref(camera_from_array(cam)),
                                             pageable.ctypes.data) == L.GS_ERR_BAD_ARG
        assert L.lib().gs_render_host_wait(r._ctx, None) == L.GS_OK


def test_streamed_readback_of_an_overflowing_frame():
    """The giant-splat scene overflows the initial tile-entry buffers on its
    first frame: the streamed frame's image must be the re-rendered whole
    frame (within the parity gate of the oracle's), and so must the next one,
    which fits."""
    from gamesplat_b200 import renderer as RR
    from gamesplat_b200 import scene

    from helpers import image_gate, oracle_alpha

    raw = scene.small_scene(11, 300)
    raw[:, 0:3] *= 0.05
    raw[:, 52:55] = 0.0   # scale e^0 = 1 m: every splat covers the whole frame
    rows = RR.pack_raw(raw)
    W, H = 1920, 1080
    cam = RR.camera_uniforms((0.0, 0.0, 1.2), float(np.pi), 0.0, W, H)
    ref_img, _ = oracle_alpha(rows, cam, W, H)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        bufs = [torch.full((H, W, 4), float("nan"), dtype=torch.float16, pin_memory=True) for _ in range(2)]
        for b in bufs:
            r.submit_frame(cam, b)
        r.wait_frames()
        st = r.stats()
        assert st.tile_overflow == 0 and st.tile_entries > (1 << 20)
        for b in bufs:
            gate = image_gate(b.numpy(), ref_img)
            assert gate["ok"], gate


@pytest.mark.parametrize("mode", ["stochastic", "gps"])
def test_streamed_frames_keep_the_render_state(mode):
    """Stochastic and GPS frames carry state from frame to frame (sample
    seeds, running accumulation, TAA history): six streamed frames equal, bit
    for bit, the frames of a second context that draws the same cameras one
    gs_render_host call at a time."""
    rows = small_rows(20_000, seed=16)
    W, H = 200, 120
    cams = [camera_uniforms((0.03 * (i % 3), 0.0, 3.0), np.pi, 0.0, W, H) for i in range(6)]
    knobs = dict(splat_render_mode=mode, black_background=1)
    with Renderer(0) as a, Renderer(0) as b:
        for r in (a, b):
            r.set(**knobs)
            r.upload_gaussians(rows)
        ref = [a.draw_frame(cam) for cam in cams]
        bufs = [torch.empty((H, W, 4), dtype=torch.float16, pin_memory=True) for _ in cams]
        for cam, buf in zip(cams, bufs):
            b.submit_frame(cam, buf)
        b.wait_frames()
        for k, (buf, img) in enumerate(zip(bufs, ref)):
            assert np.array_equal(buf.numpy().view(np.uint16), img.view(np.uint16)), k
