"""Failure injection on the host (no GPU fault): every device allocation of
an upload and of a frame is made to fail in turn (gs_debug_fail_alloc), as a
full GPU would make it fail.  Each failing call must return GS_ERR_OOM, and
the same context must then upload and render normally: alpha frames bit
for bit equal to an uninjected context's, stochastic and GPS frames finite.
The renderer refuses oversized scenes before allocating
(src/renderer.cpp:717-763); this checks the library's equivalent paths."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L

from helpers import small_cam, small_rows

pytestmark = pytest.mark.gpu

N = 20_000
W, H = 256, 144


@pytest.fixture(autouse=True)
def injection_off():
    yield
    L.lib().gs_debug_fail_alloc(-1)


@pytest.mark.parametrize("mode", ["alpha", "stochastic", "gps"])
def test_every_allocation_failure_leaves_a_usable_context(mode):
    rows = small_rows(N, seed=12)
    cam = small_cam(W, H)
    with Renderer(0) as r:
        r.set(splat_render_mode=mode, black_background=1)
        r.upload_gaussians(rows)
        clean = r.draw_frame(cam)
    lib = L.lib()
    failures = 0
    for k in range(200):
        with Renderer(0) as r:
            r.set(splat_render_mode=mode, black_background=1)
            lib.gs_debug_fail_alloc(k)
            try:
                r.upload_gaussians(rows)
                r.draw_frame(cam)
                failed = False
            except L.GsError as e:
                assert e.status == L.GS_ERR_OOM, e
                failed = True
            lib.gs_debug_fail_alloc(-1)
            if not failed:
                break
            failures += 1
            r.upload_gaussians(rows)
            img = r.draw_frame(cam)
            if mode == "alpha":
                assert np.array_equal(img.view(np.uint16), clean.view(np.uint16)), k
            else:
                assert np.isfinite(img.astype(np.float32)).all(), k
    assert failures > 5          # the upload and the frame allocate more than that
    assert not failed            # the loop ended with a run that allocated everything
