"""Device-side decode of raw 3DGS attributes (gs_pack_raw_device) against the
host packer gs_pack_raw, which is pinned to the reference PLY loader: every
field bit-identical except scale (one ulp) and opacity (two ulps at most)
where glibc's expf is not correctly rounded; then a frame rendered from the
device-packed rows matches the oracle on those rows."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gamesplat_b200 import Renderer, _lib as L, pack_raw
from oracle import oracle as O

from helpers import image_gate, small_cam

pytestmark = pytest.mark.gpu


def _raw(n, seed):
    rng = np.random.default_rng(seed)
    raw = np.empty((n, 59), np.float32)
    raw[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    raw[:, 3:6] = rng.normal(0, 0.5, (n, 3))
    raw[:, 6:51] = rng.normal(0, 0.05, (n, 45))
    raw[:, 51] = rng.normal(0, 1.5, n)
    raw[:, 52:55] = rng.normal(-4, 0.5, (n, 3))
    raw[:, 55:59] = rng.normal(0, 1, (n, 4))
    raw[:8, 55:59] = 0.0                       # degenerate quaternion: left unnormalised
    raw[8:16, 51] = [-100, -40, -1e-8, 0, 1e-8, 20, 40, 100]
    return raw


def _ulps(a, b):
    ai = a.view(np.int32).astype(np.int64)
    bi = b.view(np.int32).astype(np.int64)
    return np.abs(ai - bi)


def test_device_pack_matches_host_pack():
    n = 200_000
    raw = _raw(n, 21)
    ref = pack_raw(raw)
    raw_d = torch.from_numpy(raw).cuda()
    rows_d = torch.empty((n, 64), dtype=torch.float32, device="cuda")
    st = L.lib().gs_pack_raw_device(raw_d.data_ptr(), n, rows_d.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    got = rows_d.cpu().numpy()
    exact = np.ones(64, bool)
    exact[[3, 4, 5, 6]] = False
    assert np.array_equal(got[:, exact].view(np.uint32), ref[:, exact].view(np.uint32))
    ds = _ulps(got[:, [4, 5, 6]], ref[:, [4, 5, 6]])   # exp of the log-scale
    do = _ulps(got[:, 3], ref[:, 3])                   # 1 / (1 + exp(-x)): a denominator ulp can be two
    assert ds.max() <= 1 and do.max() <= 2
    assert (ds > 0).mean() < 1e-3 and (do > 0).mean() < 1e-3


def test_frame_from_device_packed_rows():
    n, w, h = 30_000, 320, 180
    raw = _raw(n, 22)
    raw_d = torch.from_numpy(raw).cuda()
    rows_d = torch.empty((n, 64), dtype=torch.float32, device="cuda")
    assert L.lib().gs_pack_raw_device(raw_d.data_ptr(), n, rows_d.data_ptr(), None) == 0
    torch.cuda.synchronize()
    rows = rows_d.cpu().numpy()
    cam = small_cam(w, h)
    ids, keys, proj, vc, _ = O.cull(rows, cam)
    _, si = O.sort_pairs(keys, ids)
    ref, _ = O.composite_alpha(si, proj, w, h, cam, bg=0.0)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians_device(rows_d.data_ptr(), n)
        img = r.draw_frame(cam)
    gate = image_gate(img, ref.astype(np.float16))
    assert gate["ok"], gate


def test_device_pack_argument_checks():
    raw_d = torch.zeros((4, 59), dtype=torch.float32, device="cuda")
    rows_d = torch.zeros((4 * 64 + 1,), dtype=torch.float32, device="cuda")
    assert L.lib().gs_pack_raw_device(raw_d.data_ptr(), 4, rows_d.data_ptr() + 4, None) == L.GS_ERR_BAD_ARG
    assert L.lib().gs_pack_raw_device(raw_d.data_ptr(), 0, rows_d.data_ptr(), None) == 0
