"""CPU checks of the host-side pieces of the denoised, precision and batched
variants (no GPU): the denoiser's parameter layout, the batched workload's
cameras, and the ABI structs the variants added."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from gamesplat_b200 import _lib as L
from gamesplat_b200 import denoiser as DN
from gamesplat_b200 import scene


def test_denoiser_parameter_layout():
    n = int(L.lib().gs_denoiser_param_count())
    assert n == sum(9 * cin * cout + cout for cin, cout in DN.LAYERS) == 37008
    flat = np.arange(n, dtype=np.float32)
    parts = DN.split_params(flat)
    assert [w.shape for w, _ in parts] == [(3, 3, cin, cout) for cin, cout in DN.LAYERS]
    assert np.array_equal(np.concatenate([np.concatenate([w.ravel(), b]) for w, b in parts]), flat)


def test_batch_cameras():
    cams = scene.batch_cameras(3, 64)
    assert len(cams) == 64
    assert [(w, h) for _, _, _, w, h in cams[:3]] == list(scene.BATCH_VIEWPORTS)
    rng = np.random.default_rng(3)
    for pos, yaw, pitch, w, h in cams:
        r = float(np.linalg.norm(pos))
        assert 4.0 - 1e-5 <= r <= 8.0 + 1e-5
        fwd = np.array([math.cos(pitch) * math.sin(yaw), math.sin(pitch), math.cos(pitch) * math.cos(yaw)])
        # the camera looks at a point within 1 m of the origin
        p = np.asarray(pos, np.float64)
        t = -p @ fwd
        closest = p + t * fwd
        assert t > 0 and np.linalg.norm(closest) <= 1.0 + 1e-4
    assert scene.batch_cameras(3, 64) == cams


def test_look_at_pose_inverts_forward():
    yaw, pitch = scene.look_at_pose((1.0, 2.0, 3.0), (0.0, 0.0, 0.0))
    fwd = np.array([math.cos(pitch) * math.sin(yaw), math.sin(pitch), math.cos(pitch) * math.cos(yaw)])
    d = -np.array([1.0, 2.0, 3.0]) / math.sqrt(14.0)
    assert np.allclose(fwd, d, atol=1e-12)


def test_variant_structs():
    assert C.sizeof(L.GsStats) == 96
    assert C.sizeof(L.GsKnobs) == 64
    assert C.sizeof(L.GsTuneResult) == 20 + 4 * 32 * 4
    assert L.GS_MODE_DENOISED == 3
