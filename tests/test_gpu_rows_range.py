"""GPU: gs_upload_rows_range replaces a range of the resident scene's rows
(and the heads copy the cull's visibility pass reads): the next frame's cull
records, keys and mask are bit-exact with the CPU oracle on the edited rows,
and its image within the alpha-path gate.  Ranges beyond the scene are
refused."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L

from helpers import image_gate, oracle_alpha, small_cam, small_rows

pytestmark = pytest.mark.gpu

W, H = 320, 180
N = 50_000


def test_range_edit_matches_oracle():
    rows = small_rows(N, seed=2)
    edited = rows.copy()
    edited[10_000:30_000] = small_rows(20_000, seed=7)
    edited[N - 1] = small_rows(1, seed=8)[0]
    cam = small_cam(W, H)
    ref_img, ref = oracle_alpha(edited, cam, W, H)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1, write_invisible_records=1)
        r.upload_gaussians(rows)
        r.draw_frame(cam)
        r.upload_rows_range(edited[10_000:30_000], 10_000)
        r.upload_rows_range(edited[N - 1:], N - 1)
        r.upload_rows_range(edited[:0], N)          # empty range at the end
        img = r.draw_frame(cam)
        ids = r.debug_read(L.GS_DEBUG_IDS, N)
        keys = r.debug_read(L.GS_DEBUG_KEYS, N)
        proj = r.debug_read(L.GS_DEBUG_PROJECTED, N * 16, np.float32, (N, 16))
    assert np.array_equal(ids, ref["ids"])
    assert np.array_equal(keys, ref["keys"])
    assert np.array_equal(proj.view(np.uint32), ref["proj"].view(np.uint32))
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate


def test_range_checks():
    rows = small_rows(1000, seed=4)
    with Renderer(0) as r:
        with pytest.raises(L.GsError) as e:
            r.upload_rows_range(rows[:10], 0)
        assert e.value.status == L.GS_ERR_NO_SCENE
        r.upload_gaussians(rows)
        for first, count in ((991, 10), (1000, 1), (1001, 0), (2**63, 1)):
            st = L.lib().gs_upload_rows_range(r._ctx, rows.ctypes.data, first, count)
            assert st == L.GS_ERR_BAD_ARG, (first, count)
        assert L.lib().gs_upload_rows_range(r._ctx, None, 5, 0) == L.GS_OK
        assert L.lib().gs_upload_rows_range(r._ctx, None, 5, 1) == L.GS_ERR_BAD_ARG
