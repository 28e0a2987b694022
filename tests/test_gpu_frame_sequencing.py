"""GPU tests of the frame sequencing on one context: consecutive gs_render
frames alternate between two control blocks whose counters are read back and
zeroed on a stream of their own while the next frame runs.  Frames that
alternate cameras, viewports and modes must each report their own counters
(gs_read_stats, gs_debug_read) and produce the image a fresh context produces
for that frame alone, through the stream-ordered, synchronous and streamed
entry points."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gamesplat_b200 import Renderer, _lib as L
from gamesplat_b200 import renderer as RR
from gamesplat_b200 import scene
from oracle import oracle as O

from helpers import small_rows

pytestmark = pytest.mark.gpu

N = 30_000


@pytest.fixture(scope="module")
def setup():
    rows = small_rows(N, seed=9)
    pose = scene.small_camera_pose()
    cams = [RR.camera_uniforms(*pose, 320, 180),
            RR.camera_uniforms((0.0, 0.0, 0.4), 3.0, -0.1, 320, 180, fov_y=1.9),
            RR.camera_uniforms((0.3, 0.2, 2.2), 3.4, 0.1, 256, 144, ortho_blend=0.5)]
    refs = []
    for cam in cams:
        ids, keys, proj, vc, _ = O.cull(rows, cam)
        _, si = O.sort_pairs(keys, ids)
        refs.append((vc, si[:vc]))
    fresh = []
    for cam in cams:
        with Renderer(0) as r:
            r.set(splat_render_mode="alpha", black_background=1)
            r.upload_gaussians(rows)
            fresh.append(r.draw_frame(cam))
    return rows, cams, refs, fresh


def test_alternating_frames_report_their_own_counters(setup):
    rows, cams, refs, fresh = setup
    order = [0, 1, 0, 2, 2, 1, 0, 1]
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        for k in order:
            cam = cams[k]
            w, h = int(cam[32]), int(cam[33])
            out = torch.empty(h * w * 4, dtype=torch.float16, device="cuda")
            r.draw_frame(cam, out_ptr=out.data_ptr())     # stream-ordered
            st = r.stats()
            vc, si = refs[k]
            assert st.visible_count == vc, k
            got = r.debug_read(L.GS_DEBUG_SORTED_IDS, N)
            assert np.array_equal(got[:vc], si), k
            torch.cuda.synchronize()
            img = out.cpu().numpy().reshape(h, w, 4)
            assert np.array_equal(img.view(np.uint16), fresh[k].view(np.uint16)), k


def test_back_to_back_frames_without_host_reads(setup):
    """Eight frames queued back to back (no stats in between), then each
    image compared: the blocks' zeroing on the counter stream keeps up."""
    rows, cams, _, fresh = setup
    order = [1, 0, 1, 0, 2, 1, 0, 2]
    outs = []
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        for k in order:
            w, h = int(cams[k][32]), int(cams[k][33])
            o = torch.empty(h * w * 4, dtype=torch.float16, device="cuda")
            r.draw_frame(cams[k], out_ptr=o.data_ptr())
            outs.append(o)
        torch.cuda.synchronize()
        st = r.stats()
    assert st.visible_count == setup[2][order[-1]][0]
    for k, o in zip(order, outs):
        w, h = int(cams[k][32]), int(cams[k][33])
        assert np.array_equal(o.cpu().numpy().reshape(h, w, 4).view(np.uint16), fresh[k].view(np.uint16)), k


def test_mode_switches_and_streamed_frames(setup):
    """Alpha, stochastic and GPS frames in turn on one context, then streamed
    frames: the alpha frames stay identical to a fresh context's, and each
    frame's statistics belong to it."""
    rows, cams, refs, fresh = setup
    with Renderer(0) as r:
        r.set(black_background=1)
        r.upload_gaussians(rows)
        for mode in ("alpha", "stochastic", "alpha", "gps", "alpha"):
            r.set(splat_render_mode=mode)
            img = r.draw_frame(cams[0])                   # synchronous
            st = r.stats()
            assert st.visible_count == refs[0][0], mode
            if mode == "alpha":
                assert np.array_equal(img.view(np.uint16), fresh[0].view(np.uint16))
            if mode == "gps":
                assert st.gps_requested_work_items > 0
        r.set(splat_render_mode="alpha")
        w, h = int(cams[1][32]), int(cams[1][33])
        hb = [torch.empty((h, w, 4), dtype=torch.float16).pin_memory() for _ in range(2)]
        for i in range(6):
            r.submit_frame(cams[1], hb[i & 1].numpy())
        r.wait_frames()
        for b in hb:
            assert np.array_equal(b.numpy().view(np.uint16), fresh[1].view(np.uint16))
        assert r.stats().visible_count == refs[1][0]
