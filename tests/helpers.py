"""Shared helpers for the parity tests: oracle reference frames and image
metrics.  The oracle is only ever the checker here."""
from __future__ import annotations

import numpy as np

from gamesplat_b200 import renderer as R
from gamesplat_b200 import scene
from oracle import oracle as O

# RGBA16F parity gate: max-abs <= 2^-9 per channel (plus one fp16 ulp where
# the value itself is >= 2, where one ulp already exceeds 2^-9) and PSNR >= 55.
MAX_ABS = 2.0 ** -9
MIN_PSNR = 55.0


def small_rows(n=100_000, seed=0):
    return R.pack_raw(scene.small_scene(seed, n))


def small_cam(width=1280, height=720):
    return R.camera_uniforms(*scene.small_camera_pose(), width, height)


def oracle_alpha(rows, cam, width, height, black=True, sh_degree=3):
    ids, keys, proj, vc, diag = O.cull(rows, cam, sh_degree=sh_degree)
    _, si = O.sort_pairs(keys, ids)
    img, frags = O.composite_alpha(si, proj, width, height, cam, bg=0.0 if black else 0.1)
    return img.astype(np.float16), dict(ids=ids, keys=keys, proj=proj, vc=vc, diag=diag, sorted_ids=si,
                                        frags=frags)


def psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(1.0 / mse)


def image_gate(gpu16, ref16):
    g = gpu16.astype(np.float32)
    r = ref16.astype(np.float32)
    err = np.abs(g - r)
    ulp = np.spacing(np.abs(r).astype(np.float16)).astype(np.float32)
    allowed = np.maximum(MAX_ABS, ulp)
    return dict(max_abs=float(err.max()), over=int((err > allowed).sum()), psnr=psnr(g, r),
                ok=bool((err <= allowed).all()) and psnr(g, r) >= MIN_PSNR)
