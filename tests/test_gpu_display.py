"""GPU parity of the display transform (renderer_display_appearance,
src/renderer.cpp:2120-2137; shaders/accum.glsl:201-240 with a gsanim 0.3
LUT, the blit of :181-192 without): bit-exact against the oracle, plus the
argument checks of the LUT upload (src/gaussian_loader_gsanim.cpp:237,244)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from gamesplat_b200 import Renderer, _lib as L
from oracle import oracle as O

from helpers import small_cam, small_rows

pytestmark = pytest.mark.gpu


def _frame(h, w, seed):
    rng = np.random.default_rng(seed)
    img = (rng.random((h, w, 4)) * 3.0).astype(np.float16)
    img[0, :5, :3] = 0.0                       # black pixels: clamp at exp2(log2_min)
    img[1, :5, :3] = np.float16(60000.0)       # above the range: clamp at 1
    img[2, :5, :3] = np.float16(6e-8)          # subnormal halves
    return img


def _run(r, img, exposure):
    h, w = img.shape[:2]
    src = torch.from_numpy(img.view(np.uint16).copy()).cuda()
    dst = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    r.display(src.data_ptr(), dst.data_ptr(), w, h, exposure)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


@pytest.mark.parametrize("n,lo,hi,exposure", [(2, -10.0, 2.0, 0.0), (17, -12.0, 4.0, 1.5), (33, -6.0, 3.0, -2.25)])
def test_display_lut_bit_exact(n, lo, hi, exposure):
    rng = np.random.default_rng(n)
    lut = rng.integers(0, 65536, (n, n, n, 3), dtype=np.uint16)
    img = _frame(67, 129, n)
    ref = O.display(img, lut, lo, hi, exposure)
    with Renderer(0) as r:
        r.set_display_lut(lut, lo, hi)
        got = _run(r, img, exposure)
        got2 = _run(r, img, exposure)           # a second call on the same context
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(got2.view(np.uint32), ref.view(np.uint32))


def test_display_blit_without_lut():
    img = _frame(31, 45, 7)
    ref = O.display(img, None, 0.0, 1.0, 0.0)
    with Renderer(0) as r:
        lut = np.zeros((2, 2, 2, 3), np.uint16)
        r.set_display_lut(lut, 0.0, 1.0)
        r.set_display_lut(None)                  # removed again: plain blit
        got = _run(r, img, 3.0)                  # exposure only applies with a LUT
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_display_of_a_rendered_frame():
    """The display pass applied to a gs_render frame, against the oracle on that frame."""
    w, h = 320, 180
    rows = small_rows(20_000, seed=5)
    cam = small_cam(w, h)
    n = 9
    ii = np.arange(n, dtype=np.float64) / (n - 1)
    # an s -> sqrt(s) tone curve per channel
    lut = np.empty((n, n, n, 3), np.uint16)
    lut[..., 0] = np.round(np.sqrt(ii)[None, None, :] * 65535)
    lut[..., 1] = np.round(np.sqrt(ii)[None, :, None] * 65535)
    lut[..., 2] = np.round(np.sqrt(ii)[:, None, None] * 65535)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        out16 = torch.empty((h, w, 4), dtype=torch.float16, device="cuda")
        r.draw_frame(cam, out_ptr=out16.data_ptr())
        r.set_display_lut(lut, -9.0, 1.0)
        disp = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        r.display(out16.data_ptr(), disp.data_ptr(), w, h, 0.5)
        torch.cuda.synchronize()
        frame = out16.cpu().numpy()
        got = disp.cpu().numpy()
    ref = O.display(frame, lut, -9.0, 1.0, 0.5)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert got[..., 3].min() == 1.0


def test_display_argument_checks():
    with Renderer(0) as r:
        with pytest.raises(L.GsError):
            r.set_display_lut(np.zeros((1, 1, 1, 3), np.uint16), 0.0, 1.0)     # size < 2
        with pytest.raises(L.GsError):
            r.set_display_lut(np.zeros((2, 2, 2, 3), np.uint16), 1.0, 1.0)     # log2_min >= log2_max
        src = torch.zeros(64, dtype=torch.int16, device="cuda")
        dst = torch.zeros(64 + 4, dtype=torch.float32, device="cuda")
        with pytest.raises(L.GsError):
            r.display(src.data_ptr(), dst.data_ptr() + 4, 4, 4, 0.0)           # misaligned output
        with pytest.raises(L.GsError):
            r.display(src.data_ptr(), dst.data_ptr(), 0, 4, 0.0)
