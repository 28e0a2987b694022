"""GPU parity of the gsanim int8 appearance-delta decode inside the cull
kernel (shaders/cull.glsl:125-164): projected records bit-exact against the
oracle for a single state and for a blend of two states; image within the
RGBA16F gate."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L
from oracle import oracle as O

from helpers import image_gate, small_cam, small_rows

pytestmark = pytest.mark.gpu

N = 40_000
W, H = 480, 270


@pytest.fixture(scope="module")
def anim():
    rows = small_rows(N, seed=4)
    rng = np.random.default_rng(4)
    deltas = np.clip(np.round(rng.normal(0.0, 20.0, size=(3, N, 48))), -127, 127).astype(np.int8)
    scales = np.full(48, 1.0 / 256.0, np.float32)
    return rows, deltas, scales


# (0, 0, 0.3): between two linear keys of the base state the shader still
# blends the row with itself, (1 - w) x + w x, which need not round to x
@pytest.mark.parametrize("state", [(0, 0, 0.0), (2, 0, 0.0), (1, 3, 0.375), (0, 0, 0.3), (2, 2, 0.7)])
def test_anim_records_and_image(anim, state):
    rows, deltas, scales = anim
    cam = small_cam(W, H)
    a, b, w = state
    ids, keys, proj, vc, _ = O.cull_anim(rows, cam, deltas, scales, a, b, w)
    _, si = O.sort_pairs(keys, ids)
    ref, _ = O.composite_alpha(si, proj, W, H, cam, bg=0.0)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        r.upload_animation(deltas, scales)
        r.set_animation_state(a, b, w)
        img = r.draw_frame(cam)
        got = r.debug_read(L.GS_DEBUG_PROJECTED, N * 16, np.float32, (N, 16))
    vis = ids != O.SENTINEL
    assert np.array_equal(got[vis].view(np.uint32), proj[vis].view(np.uint32))
    gate = image_gate(img, ref.astype(np.float16))
    assert gate["ok"], gate


def test_anim_state_range_checked(anim):
    rows, deltas, scales = anim
    with Renderer(0) as r:
        r.upload_gaussians(rows)
        r.upload_animation(deltas, scales)
        with pytest.raises(L.GsError):
            r.set_animation_state(4)
        with pytest.raises(L.GsError):
            r.set_animation_state(1, 2, 1.5)
