"""An animated gsanim asset against the same asset decoded into a static
scene, the property the reference's rendered integration test checks
(tests/test_gsanim_render.py: animated vs codec-decoded static PLY), here on
the projected records and without a GL display: a .gsanim archive is loaded
(gs_gsanim_load), sampled at playback times (gs_gsanim_sample), its appearance
deltas are baked into static rows in the shader's operation order
(shaders/cull.glsl:125-164), and the cull with deltas must give the same
records as the cull of the baked rows, bit for bit.  The CUDA cull is
bit-exact with the oracle cull in both forms (the GPU parity tests).  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import load_gsanim
from oracle import oracle as O
from tests import gsanim_fixture as F

from helpers import small_cam

# row slot of coefficient j: DC j = 0..2 at slots 12..14; j = 3 + 15 c + k at slot 16 + 3 k + c
SLOT = np.array([12, 13, 14] + [16 + 3 * ((j - 3) % 15) + (j - 3) // 15 for j in range(3, 48)])


def bake(rows, deltas, scales, a, b, w):
    base = rows[:, SLOT].astype(np.float32)

    def state(s):
        return base if s == 0 else base + deltas[s - 1].astype(np.float32) * scales

    v = state(a)
    if w > 0:
        v = np.float32(1.0 - w) * v + np.float32(w) * state(b)
    out = rows.copy()
    out[:, SLOT] = v
    return out


@pytest.mark.parametrize("version,interp", [("0.1", "step"), ("0.1", "linear"), ("0.2", "step")])
def test_animated_equals_baked(tmp_path, version, interp):
    n = 400
    m, b, s, d = F.v01_asset(n=n, states=4, seed=40, version=version, interpolation=interp)
    # put the Gaussians in front of the test camera
    b[:, 0:3] = np.random.default_rng(41).uniform(-1.5, 1.5, (n, 3)).astype(np.float32)
    b[:, 55:58] = -4.0
    a = load_gsanim(F.pack(tmp_path / "a.gsanim", F.entries_v01(m, b, s, d)))
    cam = small_cam(320, 180)
    seen = set()
    for t in (0.0, 0.5, 1.25, 2.0, 2.75, 5.5, 7.9):
        sa, sb, w = a.sample(t)
        seen.add((sa, sb, w > 0))
        ids, _, anim_proj, _, _ = O.cull_anim(a.rows, cam, a.deltas, a.scales, sa, sb, w)
        baked = bake(a.rows, a.deltas, a.scales, sa, sb, w)
        ids2, _, static_proj, _, _ = O.cull(baked, cam)
        assert np.array_equal(ids, ids2)
        vis = ids != O.SENTINEL
        assert vis.sum() > n // 4
        assert np.array_equal(anim_proj[vis].view(np.uint32), static_proj[vis].view(np.uint32)), t
    assert len(seen) >= 2
    a.close()
