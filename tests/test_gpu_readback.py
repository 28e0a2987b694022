"""gs_render_host readback paths give the same image as gs_render: a
page-locked destination (alpha mode: the rasterizer writes the pixels into
it through its mapped device address; other modes: one copy into it) and a
pageable destination (chunked copy through pinned staging, overlapped with
the host copy), at sizes that are not multiples of the tile size."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from gamesplat_b200 import Renderer, _lib as L
from gamesplat_b200.renderer import camera_from_array

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
