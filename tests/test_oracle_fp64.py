"""The single-precision path against the same equations in double precision
(oracle/oracle64.py): the error of the FP32 arithmetic, stated per image.
The FP32 oracle is bit-exact with the CUDA kernels' records, and the CUDA
frame is within max-abs 2^-9 / PSNR 55 dB of the oracle frame (the image
gate), so these bounds carry over to the library's frames.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from oracle import oracle64 as O64

from helpers import small_cam, small_rows


def psnr(a, b):
    mse = float(np.mean((a[..., :3] - b[..., :3]) ** 2))
    return float("inf") if mse == 0 else 10 * np.log10(1.0 / mse)


@pytest.mark.parametrize("n,w,h,seed,sh", [(3000, 160, 90, 1, 3), (20000, 320, 180, 2, 3), (8000, 211, 133, 3, 1),
                                            (8000, 211, 133, 4, 0)])
def test_fp32_frame_against_fp64(n, w, h, seed, sh):
    rows = small_rows(n, seed=seed)
    cam = small_cam(w, h)
    ids, keys, proj, _, _ = O.cull(rows, cam, sh_degree=sh)
    _, si = O.sort_pairs(keys, ids)
    img32, _ = O.composite_alpha(si, proj, w, h, cam, bg=0.0)
    vis64, _, _ = O64.project64(rows, cam, sh_degree=sh)
    img64 = O64.frame64(rows, cam, w, h, sh_degree=sh)
    assert np.array_equal(ids != O.SENTINEL, vis64)
    err32 = np.abs(img32.astype(np.float64) - img64)
    out16 = img32.astype(np.float16).astype(np.float64)        # what an RGBA16F target holds
    err16 = np.abs(out16 - img64)
    # float32 depth keys tie or cross where float64 depths differ slightly: those
    # splats composite in another order, which moves the few pixels they share
    _, depth64, _ = O64.project64(rows, cam, sh_degree=sh)
    vis = np.nonzero(vis64)[0]
    reordered = int(np.sum(si[:vis.size] != vis[np.lexsort((vis, -depth64[vis]))]))
    stats = dict(fp32_max_abs=float(err32.max()), fp32_psnr=psnr(img32.astype(np.float64), img64),
                 fp32_pixels_over_2em12=int(np.sum(err32.max(axis=2) > 2.0 ** -12)),
                 fp16_max_abs=float(err16.max()), fp16_psnr=psnr(out16, img64), reordered_splats=reordered)
    print(f"\n{n} splats {w}x{h} SH{sh}: {stats}")
    assert stats["fp32_psnr"] >= 100.0 and stats["fp32_max_abs"] <= 2.0 ** -8, stats
    assert stats["fp32_pixels_over_2em12"] <= max(2, w * h // 1000), stats
    assert stats["fp16_psnr"] >= 60.0 and stats["fp16_max_abs"] <= 2.0 ** -8, stats
