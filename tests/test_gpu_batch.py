"""GPU tests of the batched rendering entry points through the C ABI:

- gs_render_batch: frames of cameras with different positions and viewports
  in one persistent raster launch, each image bit-identical to the same
  camera's gs_render image, and one of them within the parity gate of the
  CPU oracle; a batch whose frames overflow the initial tile entries is
  re-binned and still identical;
- gs_render_anim_batch: gsanim appearance states (and blends) of one camera,
  each image bit-identical to gs_render after gs_set_anim_state.
"""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer
from gamesplat_b200 import renderer as RR
from gamesplat_b200 import scene

from helpers import image_gate, oracle_alpha

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _cams():
    views = [(320, 180), (64, 48), (256, 256), (333, 211), (128, 72), (320, 180)]
    out = []
    for k, (w, h) in enumerate(views):
        a = np.pi + 0.25 * (k - 2.5)
        pos = (float(3.0 * np.sin(a + np.pi) * 0.4), 0.1 * (k % 3) - 0.1, float(3.0 - 0.2 * k))
        out.append(RR.camera_uniforms(pos, float(a), 0.05 * (k % 2), w, h))
    return out


def _render_single(r, cam):
    w, h = int(cam[32]), int(cam[33])
    o = torch.zeros(h * w * 4, dtype=torch.float16, device="cuda")
    r.draw_frame(cam, out_ptr=o.data_ptr())
    torch.cuda.synchronize()
    return o.view(h, w, 4).cpu().numpy()


def _render_batch(r, cams):
    outs = [torch.full((int(c[33]) * int(c[32]) * 4,), float("nan"), dtype=torch.float16, device="cuda")
            for c in cams]
    r.render_batch(cams, [o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    return [o.view(int(c[33]), int(c[32]), 4).cpu().numpy() for o, c in zip(outs, cams)]


def test_camera_batch_equals_single_frames():
    rows = RR.pack_raw(scene.small_scene(7, 40_000))
    cams = _cams()
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        singles = [_render_single(r, c) for c in cams]
        for _ in range(2):   # twice: the slots are reused
            batch = _render_batch(r, cams)
            for k, (a, b) in enumerate(zip(batch, singles)):
                assert np.array_equal(a.view(np.uint16), b.view(np.uint16)), k
    ref, _ = oracle_alpha(rows, cams[0], 320, 180)
    assert image_gate(batch[0], ref)["ok"]


def test_camera_batch_with_overflowing_frames():
    raw = scene.small_scene(11, 300)
    raw[:, 0:3] *= 0.05
    raw[:, 52:55] = 0.0
    rows = RR.pack_raw(raw)
    cams = [RR.camera_uniforms((0.0, 0.0, 1.2), float(np.pi), 0.0, 1920, 1080),
            RR.camera_uniforms((0.0, 0.0, 1.5), float(np.pi), 0.0, 640, 360)]
    ref, _ = oracle_alpha(rows, cams[0], 1920, 1080)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        batch = _render_batch(r, cams)
        single = _render_single(r, cams[1])
    assert image_gate(batch[0], ref)["ok"]
    assert np.array_equal(batch[1].view(np.uint16), single.view(np.uint16))


def test_anim_state_batch_equals_single_frames():
    n, states = 30_000, 5
    rows = RR.pack_raw(scene.small_scene(9, n))
    rng = np.random.default_rng(3)
    deltas = np.clip(np.round(rng.normal(0, 20, size=(states, n, 48))), -127, 127).astype(np.int8)
    scales = np.full(48, 1.0 / 256.0, np.float32)
    cam = RR.camera_uniforms(*scene.small_camera_pose(), 320, 180)
    sa = [0, 1, 2, 5, 3, 1]
    sb = [0, 0, 0, 0, 4, 5]
    wt = [0.0, 0.0, 0.0, 0.0, 0.25, 0.6]
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        r.upload_animation(deltas, scales)
        singles = []
        for a, b, w in zip(sa, sb, wt):
            r.set_animation_state(a, b, w)
            singles.append(_render_single(r, cam))
        outs = [torch.full((180 * 320 * 4,), float("nan"), dtype=torch.float16, device="cuda") for _ in sa]
        r.render_anim_batch(cam, sa, [o.data_ptr() for o in outs], sb, wt)
        torch.cuda.synchronize()
    for k, (o, s) in enumerate(zip(outs, singles)):
        img = o.view(180, 320, 4).cpu().numpy()
        assert np.array_equal(img.view(np.uint16), s.view(np.uint16)), k
    assert not np.array_equal(singles[0].view(np.uint16), singles[1].view(np.uint16))


@pytest.mark.parametrize("shape", [(16, 16), (32, 8), (8, 32)])
def test_tile_shapes_in_the_parity_gate(shape):
    """Every tile shape draws the frame within the alpha parity gate of the
    oracle, single frames and batches alike."""
    rows = RR.pack_raw(scene.small_scene(7, 40_000))
    cams = _cams()[:3]
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        import ctypes as C

        from gamesplat_b200 import _lib as L
        L.check(L.lib().gs_set_tile_shape(r._ctx, shape[0], shape[1]), "gs_set_tile_shape")
        single = _render_single(r, cams[0])
        batch = _render_batch(r, cams)
    for cam, img in [(cams[0], single)] + list(zip(cams, batch)):
        w, h = int(cam[32]), int(cam[33])
        ref, _ = oracle_alpha(rows, cam, w, h)
        gate = image_gate(img, ref)
        assert gate["ok"], (shape, gate)


def test_autotuner_picks_a_measured_configuration():
    import ctypes as C

    from gamesplat_b200 import _lib as L

    rows = RR.pack_raw(scene.small_scene(7, 40_000))
    cams = _cams()
    outs = [torch.zeros(int(c[33]) * int(c[32]) * 4, dtype=torch.float16, device="cuda") for c in cams]
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        n = len(cams)
        arr = (L.GsCamera * n)(*[RR.camera_from_array(c) for c in cams])
        ptrs = (C.c_void_p * n)(*[C.c_void_p(o.data_ptr()) for o in outs])
        res = L.GsTuneResult()
        L.check(L.lib().gs_autotune_batch(r._ctx, arr, n, ptrs, C.byref(res)), "gs_autotune_batch")
        torch.cuda.synchronize()
        tried = [(res.tried_tile_w[i], res.tried_tile_h[i], res.tried_depth[i], res.tried_ms[i])
                 for i in range(res.tried)]
        assert res.tried >= 3 and {(t[0], t[1]) for t in tried} == {(16, 16), (32, 8), (8, 32)}
        assert (res.tile_w, res.tile_h, res.batch_depth) in [(t[0], t[1], t[2]) for t in tried]
        assert res.best_ms == min(t[3] for t in tried) and res.best_ms > 0
        batch = _render_batch(r, cams)   # with the chosen configuration
    for cam, img in zip(cams, batch):
        ref, _ = oracle_alpha(rows, cam, int(cam[32]), int(cam[33]))
        assert image_gate(img, ref)["ok"]
