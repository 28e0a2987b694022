"""Error of FP16 storage in the sorted-alpha frame, stated per image
against the float64 restatement of the splatting equations (oracle64), beside
the FP32 path's own error.  Two storage choices are measured, each with FP32
arithmetic around it: SH coefficients stored in FP16 (rows rounded before
the cull) and, on top of that, the conic stored in FP16 between the cull and
the compositor.  FP16 SH storage stays inside the RGBA16F gate of the FP32
path (max-abs 2^-9 per channel, PSNR >= 55 dB): it moves pixels by ~1e-4.
FP16 conics do not: their rounding moves fragments across the alpha >= 1/255
cut-off, and each such fragment changes its pixel by up to ~1/255 (~3.9e-3,
measured 3.6e-3 to 4.2e-3 over four scenes and two cameras), so a
reduced-precision record keeps its conic in FP32.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import renderer as RR
from oracle import oracle as O
from oracle import oracle64 as O64

from helpers import MAX_ABS, image_gate, psnr, small_rows

W, H = 320, 180
POSES = [((0.0, 0.0, 3.0), np.pi, 0.0), ((1.5, 0.5, 2.5), np.pi - 0.5, -0.2)]


def frame32(rows, cam, conic16=False):
    ids, keys, proj, _, _ = O.cull(rows, cam)
    _, si = O.sort_pairs(keys, ids)
    if conic16:
        proj = O.conic_to_fp16(proj)
    img, _ = O.composite_alpha(si, proj, W, H, cam, bg=0.0)
    return img


@pytest.mark.parametrize("seed", [0, 5])
@pytest.mark.parametrize("pose", range(len(POSES)))
def test_fp16_storage_error_against_fp64(seed, pose):
    rows = small_rows(20_000, seed=seed)
    p = POSES[pose]
    cam = RR.camera_uniforms(p[0], p[1], p[2], W, H)
    exact = O64.frame64(rows, cam, W, H)
    img32 = frame32(rows, cam)
    img_sh = frame32(O.sh_to_fp16(rows), cam)
    img_cn = frame32(O.sh_to_fp16(rows), cam, conic16=True)
    err = {k: float(np.abs(v.astype(np.float64) - exact).max()) for k, v in
           (("fp32", img32), ("sh16", img_sh), ("sh16_conic16", img_cn))}
    db = {k: psnr(v.astype(np.float64), exact) for k, v in
          (("fp32", img32), ("sh16", img_sh), ("sh16_conic16", img_cn))}
    # against the exact image: the FP32 path (isolated cut-off fragments
    # aside, as in test_oracle_fp64), FP16 SH, FP16 SH + conic
    assert db["fp32"] > 100 and err["fp32"] <= 2.0 ** -8, (err, db)
    assert db["sh16"] > 95, (err, db)
    assert db["sh16_conic16"] > 85, (err, db)
    # against the FP32 path, the parity reference of the kernels
    assert float(np.abs(img_sh - img32).max()) < 2.0 ** -11
    ref16 = img32.astype(np.float16)
    assert image_gate(img_sh.astype(np.float16), ref16)["ok"]
    assert float(np.abs(img_cn - img32).max()) > MAX_ABS
    assert not image_gate(img_cn.astype(np.float16), ref16)["ok"]


def test_sh_rounding_touches_only_sh():
    rows = small_rows(1000, seed=1)
    q = O.sh_to_fp16(rows)
    keep = np.r_[0:12, 15, 61:64]
    assert np.array_equal(q[:, keep].view(np.uint32), rows[:, keep].view(np.uint32))
    sh = np.r_[12:15, 16:61]
    assert np.array_equal(q[:, sh], rows[:, sh].astype(np.float16).astype(np.float32))
