"""The device-side wait limits, exercised without a GPU fault: the probe runs
the library's bounded look-back and mbarrier waits against a word nothing
publishes, the wait runs out, the call reports GS_ERR_DEVICE_TIMEOUT, and the
same context then renders a correct frame."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L
from oracle import oracle as O

from helpers import image_gate, small_cam, small_rows

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, 1])
def test_wait_runs_out_and_context_stays_usable(which):
    w, h = 256, 144
    rows = small_rows(8_000, seed=11)
    cam = small_cam(w, h)
    ids, keys, proj, vc, _ = O.cull(rows, cam)
    _, si = O.sort_pairs(keys, ids)
    ref, _ = O.composite_alpha(si, proj, w, h, cam, bg=0.0)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        st = L.lib().gs_debug_wait_probe(r._ctx, which, 2000)
        assert st == L.GS_ERR_DEVICE_TIMEOUT, L.lib().gs_status_str(st)
        assert b"ran out" in L.lib().gs_last_error(r._ctx)
        img = r.draw_frame(cam)              # the context is still usable
        assert r.stats().error_flags == 0
    gate = image_gate(img, ref.astype(np.float16))
    assert gate["ok"], gate


def test_probe_argument_checks():
    with Renderer(0) as r:
        assert L.lib().gs_debug_wait_probe(r._ctx, 2, 100) == L.GS_ERR_BAD_ARG
        assert L.lib().gs_debug_wait_probe(r._ctx, 0, 0) == L.GS_ERR_BAD_ARG
