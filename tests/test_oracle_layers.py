"""The oracle's gsanim 0.3 layer colour (shaders/cull.glsl:141-148, 354-416)
against identities of the formula: a layer of DC coefficients alone gives
max(SH_C0 * dc, 0) * weight exactly; the geometry fields are those of the
layer-free cull; two identical layers of weight 1 give twice one layer; a
single SH coefficient reaches only its own channel.  CPU only."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

from helpers import small_cam, small_rows

SH_C0 = np.float32(0.28209479177387814)


def scene():
    rows = small_rows(3000, seed=21)
    rows[:, 12:15] = 0.0
    rows[:, 16:61] = 0.0
    return rows, small_cam(320, 180)


def test_dc_layer_and_geometry():
    rows, cam = scene()
    ids, keys, base, _, _ = O.cull(rows, cam)
    rng = np.random.default_rng(1)
    halves = np.zeros((2, rows.shape[0], 48), np.uint16)
    dc = rng.normal(0, 1, (rows.shape[0], 3)).astype(np.float16)
    halves[0, :, 0:3] = dc.view(np.uint16)
    w = np.array([[0.5, 1.0, 2.0], [3.0, 3.0, 3.0]], np.float32)    # layer 1 is all zero: adds 0
    i1, k1, proj, _, _ = O.cull_layers(rows, cam, halves, w)
    vis = ids != O.SENTINEL
    assert np.array_equal(i1, ids) and np.array_equal(k1, keys)
    expect = np.maximum(SH_C0 * dc.astype(np.float32), np.float32(0)) * w[0]
    assert np.array_equal(proj[vis, :3], expect[vis])
    assert np.array_equal(proj[vis, 3:].view(np.uint32), base[vis, 3:].view(np.uint32))


def test_layer_sums_and_channels():
    rows, cam = scene()
    n = rows.shape[0]
    rng = np.random.default_rng(2)
    one = rng.normal(0, 0.5, (1, n, 48)).astype(np.float16).view(np.uint16)
    ones = np.ones((2, 3), np.float32)
    ids, _, p1, _, _ = O.cull_layers(rows, cam, one, ones[:1])
    _, _, p2, _, _ = O.cull_layers(rows, cam, np.concatenate([one, one]), ones)
    vis = ids != O.SENTINEL
    assert np.array_equal(p2[vis, :3], 2 * p1[vis, :3])
    # one SH coefficient (k = 0, channel c) with a large DC on the same channel: other channels stay at 0
    for c in range(3):
        h = np.zeros((1, n, 48), np.float16)
        h[0, :, c] = 4.0                       # DC of channel c
        h[0, :, 3 + c * 15 + 0] = 1.0          # SH(0) of channel c
        _, _, p, _, _ = O.cull_layers(rows, cam, h.view(np.uint16), ones[:1])
        others = [k for k in range(3) if k != c]
        assert np.all(p[vis][:, others] == 0)
        assert np.all(p[vis][:, c] > 0)
