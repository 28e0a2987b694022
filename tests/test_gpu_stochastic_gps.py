"""GPU parity of the stochastic and Gaussian Point Splatting paths and of the
accumulation passes, through the C ABI.  The stochastic sample (kept
fragment per pixel, colour and D24 depth) and the GPS resolve are
deterministic and compared bit for bit with the CPU oracle."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L
from gamesplat_b200 import renderer as RR
from oracle import oracle as O

from helpers import small_cam, small_rows

pytestmark = pytest.mark.gpu

W, H = 640, 360


@pytest.fixture(scope="module")
def scene_small():
    rows = small_rows(60_000, seed=2)
    cam = small_cam(W, H)
    ids, keys, proj, vc, _ = O.cull(rows, cam)
    return rows, cam, ids, proj


def stochastic_renderer(rows, **kw):
    r = Renderer(0)
    knobs = dict(splat_render_mode="stochastic", black_background=1, stochastic_taa_enabled=0,
                 stochastic_accumulation_enabled=0, stochastic_samples_per_frame=1)
    knobs.update(kw)
    r.set(**knobs)
    r.upload_gaussians(rows)
    return r


def test_stochastic_sample_bit_exact(scene_small):
    rows, cam, ids, proj = scene_small
    with stochastic_renderer(rows) as r:
        img = r.draw_frame(cam)
        sample = r.debug_read(L.GS_DEBUG_SAMPLE, W * H * 4, np.float32, (H, W, 4))
        depth = r.debug_read(L.GS_DEBUG_DEPTH, W * H, np.float32, (H, W))
    ref, ref_depth, kept = O.stochastic_sample(ids, proj, W, H, 1.0, cam, bg=0.0, rgba8=True)
    assert kept > 0
    assert np.array_equal(sample.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(depth.view(np.uint32), ref_depth.view(np.uint32))
    assert np.array_equal(img, ref.astype(np.float16))


def test_stochastic_linear_target_bit_exact(scene_small):
    rows, cam, ids, proj = scene_small
    with stochastic_renderer(rows, linear_color=1) as r:
        r.draw_frame(cam)
        sample = r.debug_read(L.GS_DEBUG_SAMPLE, W * H * 4, np.float32, (H, W, 4))
    ref, _, _ = O.stochastic_sample(ids, proj, W, H, 1.0, cam, bg=0.0, rgba8=False)
    assert np.array_equal(sample.view(np.uint32), ref.view(np.uint32))


def test_stochastic_running_accumulation_bit_exact(scene_small):
    rows, cam, ids, proj = scene_small
    with stochastic_renderer(rows, stochastic_accumulation_enabled=1) as r:
        for _ in range(3):
            r.draw_frame(cam)
        acc = r.debug_read(L.GS_DEBUG_ACCUM, W * H * 4, np.float32, (H, W, 4))
        st = r.stats()
    assert st.sample_count == 3 and st.frame_seed == 3
    a = None
    for k in (1, 2, 3):
        s, _, _ = O.stochastic_sample(ids, proj, W, H, float(k), cam, bg=0.0, rgba8=True)
        a = O.accum(s, s if a is None else a, float(k))
    assert np.array_equal(acc.view(np.uint32), a.view(np.uint32))


def test_stochastic_taa_frames_bit_exact(scene_small):
    """Default stochastic mode (TAA on, 4 jittered samples per frame) over two
    frames with a moved camera, bit for bit against the oracle's samples,
    running mean and TAA pass."""
    rows, cam, _, _ = scene_small
    cam2 = RR.camera_uniforms((0.05, 0.0, 3.0), float(np.pi) + 0.01, 0.0, W, H)
    with stochastic_renderer(rows, stochastic_taa_enabled=1, stochastic_taa_current_samples=4) as r:
        r.draw_frame(cam)
        r.draw_frame(cam2)
        acc = r.debug_read(L.GS_DEBUG_ACCUM, W * H * 4, np.float32, (H, W, 4))
    seed = 0
    hist_c = np.zeros((H, W, 4), np.float32)
    hist_x = np.zeros((H, W, 4), np.float32)
    prev = None
    for k, c in enumerate((cam, cam2)):
        ids, keys, proj, vc, _ = O.cull(rows, c)
        avg = None
        depth = None
        for i in range(4):
            seed += 1
            j = (seed % 1024) + 1
            jit = (O.lib().oc_halton(j, 2) - 0.5, O.lib().oc_halton(j, 3) - 0.5)
            s, depth, _ = O.stochastic_sample(ids, proj, W, H, float(seed), c, bg=0.0, jitter=jit, rgba8=True)
            avg = O.accum(s, s if avg is None else avg, float(i + 1))
        ok, inv = O.mat4_inverse(c[:16])
        assert ok
        has_hist = prev is not None
        pv = prev if has_hist else c
        vo = np.array([c[32], c[33], c[34], pv[34]], np.float32)
        fc = np.array([c[35], c[36], c[37], c[38]], np.float32)
        pfc = np.array([pv[35], pv[36], pv[37], 0.0], np.float32)
        pz = np.array([c[26], c[30], 0.0, 0.0], np.float32)
        changed = 1.0 if (has_hist and not np.array_equal(prev, c)) else 0.0
        hist_c, hist_x = O.taa(avg, depth, hist_c, hist_x, inv, pv[:16], vo, fc, pfc, pz,
                               1.0 if has_hist else 0.0, changed)
        prev = c
    # the inverse view is the reference's cofactor inverse on both sides
    # (src/renderer.cpp:86-206), so the TAA history matches bit for bit
    assert np.array_equal(acc.view(np.uint32), hist_c.view(np.uint32)), np.abs(acc - hist_c).max()


def gps_renderer(rows, **kw):
    r = Renderer(0)
    knobs = dict(splat_render_mode="gps", black_background=1, stochastic_accumulation_enabled=0,
                 gps_supersample_factor=2)
    knobs.update(kw)
    r.set(**knobs)
    r.upload_gaussians(rows)
    return r


@pytest.mark.parametrize("ss", [1, 2, 3])
def test_gps_frame_bit_exact(scene_small, ss):
    rows, cam, ids, proj = scene_small
    with gps_renderer(rows, gps_supersample_factor=ss) as r:
        img = r.draw_frame(cam)
        sample = r.debug_read(L.GS_DEBUG_SAMPLE, W * H * 4, np.float32, (H, W, 4))
        depth = r.debug_read(L.GS_DEBUG_DEPTH, W * H, np.float32, (H, W))
        st = r.stats()
    ref, ref_depth, requested, overflow = O.gps_frame(ids, proj, W, H, ss, 16 << 20, 1.0)
    assert overflow == 0 and st.gps_budget_exhausted == 0
    assert st.gps_requested_work_items == requested > 0
    assert np.array_equal(sample.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(depth.view(np.uint32), ref_depth.view(np.uint32))
    assert np.array_equal(img, ref.astype(np.float16))


def test_gps_budget_overflow_flag_and_resize(scene_small):
    rows, cam, ids, proj = scene_small
    with gps_renderer(rows) as r:
        assert r.set_gps_work_budget(1000)
        r.draw_frame(cam)
        st = r.stats()
        _, _, requested, overflow = O.gps_frame(ids, proj, W, H, 2, 1000, 1.0)
        assert overflow == 1 and st.gps_budget_exhausted == 1
        assert st.gps_requested_work_items == requested
        assert st.gps_max_work_items == 1000
        assert r.set_gps_work_budget(16 << 20)
        r.draw_frame(cam)
        assert r.stats().gps_budget_exhausted == 0


def test_gps_accumulation_bit_exact(scene_small):
    rows, cam, ids, proj = scene_small
    with gps_renderer(rows, stochastic_accumulation_enabled=1) as r:
        for _ in range(3):
            r.draw_frame(cam)
        acc = r.debug_read(L.GS_DEBUG_ACCUM, W * H * 4, np.float32, (H, W, 4))
    a = None
    for k in (1, 2, 3):
        s, _, _, _ = O.gps_frame(ids, proj, W, H, 2, 16 << 20, float(k))
        a = O.accum(s, s if a is None else a, float(k))
    assert np.array_equal(acc.view(np.uint32), a.view(np.uint32))
