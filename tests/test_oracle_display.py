"""CPU checks of the oracle's display transform (shaders/accum.glsl:201-240):
known answers (constant LUT, linear LUT, blit) and agreement with a float64
restatement of the shader to within float rounding."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def _img(seed, h=11, w=17):
    rng = np.random.default_rng(seed)
    return (rng.random((h, w, 4)) * 4.0 + 1e-3).astype(np.float16)


def _shader_f64(img, lut, lo, hi, ev):
    n = lut.shape[0]
    rad = img[..., :3].astype(np.float64) * 2.0 ** ev
    s = np.clip((np.log2(np.maximum(rad, 2.0 ** lo)) - lo) / (hi - lo), 0.0, 1.0)
    p = s * (n - 1)
    i0 = np.floor(p).astype(int)
    i1 = np.minimum(i0 + 1, n - 1)
    f = p - i0
    L = lut.astype(np.float64) / 65535.0
    out = np.zeros(img.shape[:2] + (3,))
    for c in range(3):
        def e(x, y, z):
            return L[z, y, x, c]
        a = (e(i0[..., 0], i0[..., 1], i0[..., 2]) * (1 - f[..., 0]) + e(i1[..., 0], i0[..., 1], i0[..., 2]) * f[..., 0]) * (1 - f[..., 1]) \
            + (e(i0[..., 0], i1[..., 1], i0[..., 2]) * (1 - f[..., 0]) + e(i1[..., 0], i1[..., 1], i0[..., 2]) * f[..., 0]) * f[..., 1]
        b = (e(i0[..., 0], i0[..., 1], i1[..., 2]) * (1 - f[..., 0]) + e(i1[..., 0], i0[..., 1], i1[..., 2]) * f[..., 0]) * (1 - f[..., 1]) \
            + (e(i0[..., 0], i1[..., 1], i1[..., 2]) * (1 - f[..., 0]) + e(i1[..., 0], i1[..., 1], i1[..., 2]) * f[..., 0]) * f[..., 1]
        out[..., c] = a * (1 - f[..., 2]) + b * f[..., 2]
    return out, s


def test_constant_lut():
    lut = np.full((4, 4, 4, 3), 32768, np.uint16)
    out = O.display(_img(1), lut, -8.0, 3.0, 0.0)
    assert np.allclose(out[..., :3], 32768 / 65535, rtol=0, atol=1e-7)
    assert (out[..., 3] == 1.0).all()


def test_linear_lut_returns_the_log_coordinate():
    n = 2
    lut = np.zeros((n, n, n, 3), np.uint16)
    lut[:, :, 1, 0] = 65535
    lut[:, 1, :, 1] = 65535
    lut[1, :, :, 2] = 65535
    img = _img(2)
    out = O.display(img, lut, -6.0, 3.0, 0.75)
    _, s = _shader_f64(img, lut, -6.0, 3.0, 0.75)
    assert np.abs(out[..., :3] - s).max() < 2e-6


def test_random_lut_matches_float64_shader():
    rng = np.random.default_rng(3)
    lut = rng.integers(0, 65536, (9, 9, 9, 3), dtype=np.uint16)
    img = _img(3, 23, 31)
    out = O.display(img, lut, -10.0, 4.0, -1.0)
    ref, _ = _shader_f64(img, lut, -10.0, 4.0, -1.0)
    assert np.abs(out[..., :3] - ref).max() < 1e-4


def test_blit_is_the_input():
    img = _img(4)
    out = O.display(img, None, 0.0, 1.0, 2.0)
    assert np.array_equal(out, img.astype(np.float32))
