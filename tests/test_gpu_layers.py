"""GPU parity of the gsanim 0.3 appearance layers (shaders/cull.glsl:141-148,
354-416): each splat's colour is the sum over the layers of max(SH colour of
the layer's half coefficients, 0) * the layer's RGB weight.  Projected
records bit-exact against the oracle, image within the RGBA16F gate; the
layer path off again after an empty weight list; weight counts checked."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L
from oracle import oracle as O

from helpers import image_gate, small_cam, small_rows

pytestmark = pytest.mark.gpu

N = 30_000
W, H = 480, 270


@pytest.fixture(scope="module")
def layered():
    rows = small_rows(N, seed=8)
    rows[:, 12:15] = 0.0          # a version 0.3 base carries no appearance
    rows[:, 16:61] = 0.0
    rng = np.random.default_rng(8)
    halves = rng.normal(0.0, 0.6, size=(3, N, 48)).astype(np.float16).view(np.uint16)
    weights = rng.uniform(0.0, 2.0, size=(3, 3)).astype(np.float32)
    return rows, halves, weights


@pytest.mark.parametrize("count,sh_degree", [(1, 3), (3, 3), (3, 1)])
def test_layer_records_and_image(layered, count, sh_degree):
    rows, halves, weights = layered
    cam = small_cam(W, H)
    ids, keys, proj, vc, _ = O.cull_layers(rows, cam, halves[:count], weights[:count], sh_degree=sh_degree)
    _, si = O.sort_pairs(keys, ids)
    ref, _ = O.composite_alpha(si, proj, W, H, cam, bg=0.0)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1, sh_degree=sh_degree)
        r.upload_gaussians(rows)
        r.upload_layers(halves)
        r.set_layer_weights(weights[:count])
        img = r.draw_frame(cam)
        got = r.debug_read(L.GS_DEBUG_PROJECTED, N * 16, np.float32, (N, 16))
        assert r.stats().visible_count == vc
    vis = ids != O.SENTINEL
    assert np.array_equal(got[vis].view(np.uint32), proj[vis].view(np.uint32))
    gate = image_gate(img, ref.astype(np.float16))
    assert gate["ok"], gate


def test_layers_off_and_checked(layered):
    rows, halves, weights = layered
    cam = small_cam(W, H)
    ids, _, proj, _, _ = O.cull(rows, cam)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        r.upload_layers(halves[:2])
        with pytest.raises(L.GsError):
            r.set_layer_weights(weights)               # 3 weights, 2 layers
        r.set_layer_weights(weights[:2])
        r.draw_frame(cam)
        r.set_layer_weights(np.zeros((0, 3), np.float32))
        r.draw_frame(cam)
        got = r.debug_read(L.GS_DEBUG_PROJECTED, N * 16, np.float32, (N, 16))
    vis = ids != O.SENTINEL
    assert np.array_equal(got[vis].view(np.uint32), proj[vis].view(np.uint32))
