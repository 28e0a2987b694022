"""CPU tests: pin the oracle against the reference's own shader stages
(shaders/cull.glsl, sort.glsl, splat.glsl, gps.glsl, accum.glsl with the
display transform), compiled from their
source for the CPU into oracle/_ref/libglslref.so (oracle/Makefile, with
oracle/glsl/extract.py and oracle/glsl/harness.cpp), through the committed
fixture tests/golden/shader_small.npz (tests/golden/make_shader_golden.py)
and, where the reference sources are present, live on seeded sweeps.

What the shader source fixes (each expression, its operand order, its float
types) is compared bit for bit.  What GLSL leaves to the implementation
(exp, log, sin/cos, the summation order of products, the fixed-function
rasterizer, blender and depth test) is the oracle's own definition on both
sides (oracle/glsl/glsl.h, oracle/glsl/harness.cpp), so these tests check the
oracle's restatement of every stage's arithmetic, not those choices.

The one difference allowed: GPS colours at pixels where two splats share a
depth key.  The reference's prototype keeps the first writer of the minimum
(`atomicMin` then a plain store, shaders/gps.glsl:277-283, racy on a GPU and
in invocation order here); the oracle and the CUDA path keep the smaller
(depth, colour) pair of one 64-bit minimum."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from gamesplat_b200 import renderer as R
from gamesplat_b200 import scene
from oracle import oracle as O

FIXTURE = Path(__file__).with_name("golden") / "shader_small.npz"
W, H = 128, 80

live = pytest.mark.skipif(not O.glsl_available(), reason="reference shader build (oracle/_ref) not present")


@pytest.fixture(scope="module")
def fx():
    return np.load(FIXTURE)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _same_cull(a, b):
    return (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(_bits(a[2]), _bits(b[2]))
            and a[3] == b[3] and np.array_equal(a[4], b[4]))


def _gps_colour_ties(a, b, limit):
    """Pixels whose RGBA8 colours differ; at most `limit` of them."""
    diff = int((np.rint(a * 255.0) != np.rint(b * 255.0)).any(-1).sum())
    assert diff <= limit, diff
    return diff


# ------------------------------------------------------------ committed fixture
@pytest.mark.parametrize("k", range(4))
def test_oracle_cull_matches_shader_fixture(fx, k):
    ids, keys, proj, vc, diag = O.cull(fx["rows"], fx["cams"][k])
    assert np.array_equal(ids, fx[f"ids_{k}"]) and np.array_equal(keys, fx[f"keys_{k}"])
    assert np.array_equal(_bits(proj), _bits(fx[f"proj_{k}"]))
    assert vc == int(fx[f"vc_{k}"]) and np.array_equal(diag, fx[f"diag_{k}"])


@pytest.mark.parametrize("k", range(4))
def test_oracle_frames_match_shader_fixture(fx, k):
    cam = fx["cams"][k]
    ids, keys, proj, _, _ = O.cull(fx["rows"], cam)
    _, si = O.sort_pairs(keys, ids)
    img, _ = O.composite_alpha(si, proj, W, H, cam, bg=0.0)
    assert np.array_equal(img.astype(np.float16).view(np.uint16), fx[f"alpha_{k}"].view(np.uint16))
    s, z, _ = O.stochastic_sample(ids, proj, W, H, 1.0, cam, bg=0.0, rgba8=True)
    assert np.array_equal(np.rint(s * 255.0).astype(np.uint8), fx[f"stoch_{k}"])
    assert np.array_equal(np.rint(z.astype(np.float64) * 16777215.0).astype(np.uint32), fx[f"zstoch_{k}"])
    g, gz, requested, overflow = O.gps_frame(ids, proj, W, H, 2, 16 << 20, 1.0)
    assert overflow == 0 and requested == int(fx[f"gpsw_{k}"])
    assert np.array_equal(_bits(gz), _bits(fx[f"zgps_{k}"]))
    _gps_colour_ties(g, fx[f"gps_{k}"].astype(np.float32) / 255.0, limit=W * H // 500)


@pytest.mark.parametrize("case", ["cull", "ties"])
def test_oracle_sort_matches_shader_fixture(fx, case):
    k, i = fx[f"sort_in_{case}"]
    ko, io = O.sort_pairs(k, i)
    assert np.array_equal(np.stack([ko, io]), fx[f"sort_out_{case}"])


def test_oracle_display_matches_shader_fixture(fx):
    lo, hi, ex = (float(v) for v in fx["disp_params"])
    got = O.display(fx["disp_in"], fx["disp_lut"], lo, hi, ex)
    assert np.array_equal(_bits(got), _bits(fx["disp_out"]))
    assert np.array_equal(_bits(O.display(fx["disp_in"], None, 0.0, 1.0, 0.0)), _bits(fx["blit_out"]))


def test_oracle_anim_matches_shader_fixture(fx):
    deltas = scene.anim_deltas(5, fx["rows"].shape[0], 3)
    for s, (a, b, w) in enumerate(fx["anim_states"]):
        ids, _, proj, _, _ = O.cull_anim(fx["rows"], fx["cams"][0], deltas, fx["anim_scales"], int(a), int(b),
                                         float(w))
        assert np.array_equal(ids, fx["anim_ids"])
        assert np.array_equal(_bits(proj), _bits(fx[f"anim_proj_{s}"])), (a, b, w)


# ------------------------------------------------------------------ live sweeps
def _fly_cameras(rng, count):
    """Seeded cameras: most look at a point near the scene from 0.5-4 units
    away, the rest in a random direction from anywhere around it."""
    for _ in range(count):
        if rng.random() < 0.75:
            d = rng.normal(size=3)
            pos = (d / np.linalg.norm(d) * rng.uniform(0.5, 4.0)).astype(np.float32)
            yaw, pitch = scene.look_at_pose(pos, rng.uniform(-0.4, 0.4, 3))
        else:
            pos = rng.uniform(-1.5, 1.5, 3).astype(np.float32)
            yaw, pitch = float(rng.uniform(-7, 7)), float(rng.uniform(-1.4, 1.4))
        w, h = int(rng.integers(16, 400)), int(rng.integers(16, 300))
        cam = R.camera_uniforms(pos, yaw, pitch, w, h, fov_y=float(rng.uniform(0.3, 2.4)),
                                ortho_blend=float(rng.choice([0.0, 1.0, rng.uniform(0, 1)])),
                                ortho_size=float(rng.uniform(0.5, 6.0)))
        cam = cam.copy()
        cam[37] = np.float32(rng.choice([1.0, -1.0]))
        cam[38] = np.float32(rng.choice([0.0, 1.0]))
        yield cam


@live
def test_cull_sweep_matches_shader():
    """Records, ids, keys, visible count and diagnostics of every row over
    seeded scenes and fly cameras: orthographic blends, both clip y signs and
    clip depth ranges, SH degrees 0-3, view-distance LOD on and off."""
    rng = np.random.default_rng(2024)
    visible = 0
    for seed in range(6):
        rows = R.pack_raw(scene.small_scene(100 + seed, 6000))
        for cam in _fly_cameras(rng, 30):
            deg = int(rng.integers(0, 4))
            lod = float(rng.choice([0.0, rng.uniform(0.5, 4.0)]))
            stats = bool(rng.integers(0, 2))
            a = O.cull(rows, cam, sh_degree=deg, sh_lod_distance=lod, collect_stats=stats)
            b = O.glsl_cull(rows, cam, sh_degree=deg, sh_lod_distance=lod, collect_stats=stats)
            assert _same_cull(a, b), (seed, deg, lod, cam[32:40])
            visible += a[3]
    assert visible > 100_000


@live
def test_sort_matches_shader():
    """The radix sort shaders (four 8-bit passes of hist / prefix / scatter,
    workgroups run with their barriers) against the oracle's sort: the same
    permutation, ties in index order, for partial, single and many
    workgroups, tie-heavy keys, random keys and a cull's output."""
    rng = np.random.default_rng(17)
    for n in (1, 2, 255, 256, 257, 4099, 70_001):
        k = rng.integers(0, 40, n).astype(np.uint32) * np.uint32(0x01010101)
        i = np.arange(n, dtype=np.uint32)
        a, b = O.sort_pairs(k, i), O.glsl_sort_pairs(k, i)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), n
    k = rng.integers(0, 2 ** 32, 30_000, dtype=np.uint64).astype(np.uint32)
    i = rng.permutation(30_000).astype(np.uint32)
    a, b = O.sort_pairs(k, i), O.glsl_sort_pairs(k, i)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    rows = R.pack_raw(scene.small_scene(4, 20_000))
    ids, keys, _, vc, _ = O.cull(rows, R.camera_uniforms((0.0, 0.0, 0.3), 3.0, -0.1, 320, 180, fov_y=1.9))
    assert 0 < vc < 20_000
    a, b = O.sort_pairs(keys, ids), O.glsl_sort_pairs(keys, ids)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@live
def test_anim_and_layers_match_shader():
    """int8 appearance deltas for single states and blends, states 0 and 0 at a
    positive weight included, and gsanim 0.3 half-float layers."""
    rng = np.random.default_rng(7)
    rows = R.pack_raw(scene.small_scene(3, 5000))
    cam = R.camera_uniforms(*scene.small_camera_pose(), 320, 180)
    n = rows.shape[0]
    deltas = scene.anim_deltas(9, n, 4)
    scales = rng.uniform(0.001, 0.02, 48).astype(np.float32)
    for a, b, w in [(0, 0, 0.0), (3, 0, 0.0), (1, 4, 0.25), (0, 0, 0.3), (0, 2, 0.9), (4, 4, 0.6), (2, 1, 1.0)]:
        ref = O.glsl_cull(rows, cam, deltas=deltas, scales=scales, state_a=a, state_b=b, weight=w)
        got = O.cull_anim(rows, cam, deltas, scales, a, b, w)
        assert _same_cull(got, ref), (a, b, w)
    for layers in (1, 3):
        halves = rng.normal(0.0, 0.4, (layers, n, 48)).astype(np.float16).view(np.uint16)
        weights = rng.uniform(0.0, 1.5, (layers, 3)).astype(np.float32)
        ref = O.glsl_cull(rows, cam, halves=halves, layer_weights=weights)
        got = O.cull_layers(rows, cam, halves, weights)
        assert _same_cull(got, ref), layers


@live
def test_alpha_and_stochastic_frames_match_shader():
    """splat_vs + splat_fs composite (FP32 blend) and splat_vs +
    splat_stochastic_fs samples, with sub-pixel jitter, odd frame sizes and
    both clip y signs; every pixel bit for bit."""
    rng = np.random.default_rng(11)
    rows = R.pack_raw(scene.small_scene(5, 8000))
    fragments = 0
    for cam in _fly_cameras(rng, 24):
        w, h = int(cam[32]), int(cam[33])
        ids, keys, proj, vc, _ = O.cull(rows, cam)
        _, si = O.sort_pairs(keys, ids)
        jit = tuple(float(v) for v in rng.uniform(-0.5, 0.5, 2))
        bg = float(rng.choice([0.0, 0.1]))
        a, fa = O.composite_alpha(si, proj, w, h, cam, bg=bg, jitter=jit)
        b, fb = O.glsl_composite_alpha(si, proj, w, h, cam, bg=bg, jitter=jit)
        assert fa == fb and np.array_equal(_bits(a), _bits(b)), (vc, fa, fb)
        fragments += fa
        for seed in (1.0, 37.0):
            rgba8 = bool(rng.integers(0, 2))
            s1, z1, k1 = O.stochastic_sample(ids, proj, w, h, seed, cam, bg=bg, jitter=jit, rgba8=rgba8)
            s2, z2, k2 = O.glsl_stochastic_sample(ids, proj, w, h, seed, cam, bg=bg, jitter=jit, rgba8=rgba8)
            assert k1 == k2 and np.array_equal(_bits(s1), _bits(s2)) and np.array_equal(_bits(z1), _bits(z2))
    assert fragments > 1_000_000


@live
@pytest.mark.parametrize("ss", [1, 2, 3])
def test_gps_frames_match_shader(ss):
    """gps_clear/expand/splat/resolve: requested work items, overflow flag and
    resolved depth exact; colours equal except where splats tie on a depth key."""
    rows = R.pack_raw(scene.small_scene(8, 8000))
    cam = R.camera_uniforms(*scene.small_camera_pose(), 200, 120)
    ids, keys, proj, _, _ = O.cull(rows, cam)
    for linear, budget, seed in ((False, 16 << 20, 1.0), (True, 16 << 20, 9.0), (False, 5000, 2.0)):
        a = O.gps_frame(ids, proj, 200, 120, ss, budget, seed, linear_color=linear)
        b = O.glsl_gps_frame(ids, proj, 200, 120, ss, budget, seed, linear_color=linear)
        assert a[2:] == b[2:]
        assert np.array_equal(_bits(a[1]), _bits(b[1]))
        _gps_colour_ties(a[0], b[0], limit=200 * 120 // 500)


@live
def test_mat4_inverse_matches_reference():
    """The TAA's inverse view: the oracle's cofactor inverse against the
    reference's own mat4_inverse (cut from src/renderer.cpp at build time) on
    view and projection matrices of fly cameras and on scaled general
    matrices: same refusals, same bits."""
    rng = np.random.default_rng(21)
    for k in range(1500):
        if k % 3 == 0:
            m = rng.normal(size=16).astype(np.float32) * np.float32(10.0 ** rng.uniform(-3, 3))
        else:
            cam = R.camera_uniforms(rng.uniform(-50, 50, 3), rng.uniform(-7, 7), rng.uniform(-1.5, 1.5), 64, 48,
                                    z_up=bool(k % 2), ortho_blend=float(rng.choice([0.0, 0.5, 1.0])))
            m = cam[:16] if k % 3 == 1 else cam[16:32]
        a, b = O.mat4_inverse(m), O.ref_mat4_inverse(m)
        assert a[0] == b[0] and (not a[0] or np.array_equal(_bits(a[1]), _bits(b[1]))), k
    for m in (np.zeros(16, np.float32), np.diag(np.float32([1e-3, 1e-3, 1e-3, 1e-3])).reshape(16)):
        assert O.mat4_inverse(m)[0] is False and O.ref_mat4_inverse(m)[0] is False


@live
def test_accum_and_taa_match_shader():
    """accum_fs on random frames; taa_accum_fs over a chain of frames whose
    camera moves, returns and holds, every output bit for bit."""
    rng = np.random.default_rng(5)
    w, h = 96, 64
    s, hist = rng.random((h, w, 4), dtype=np.float32), rng.random((h, w, 4), dtype=np.float32)
    for n in (0.0, 1.0, 2.0, 5.0, 64.0):
        assert np.array_equal(_bits(O.accum(s, hist, n)), _bits(O.glsl_accum(s, hist, n)))
    rows = R.pack_raw(scene.small_scene(2, 6000))
    cams = [R.camera_uniforms(*scene.small_camera_pose(), w, h),
            R.camera_uniforms((0.05, 0.0, 3.0), float(np.pi) + 0.01, 0.0, w, h),
            R.camera_uniforms((0.05, 0.0, 3.0), float(np.pi) + 0.01, 0.0, w, h, ortho_blend=0.5)]
    hc = hx = np.zeros((h, w, 4), np.float32)
    gc, gx = hc, hx
    prev = None
    for k, cam in enumerate([cams[0], cams[1], cams[1], cams[0], cams[2]]):
        ids, keys, proj, _, _ = O.cull(rows, cam)
        avg = depth = None
        for i in range(2):
            smp, depth, _ = O.stochastic_sample(ids, proj, w, h, float(10 * k + i + 1), cam, jitter=(0.2 * i, -0.1))
            avg = O.accum(smp, smp if avg is None else avg, float(i + 1))
        ok, inv = O.mat4_inverse(cam[:16])
        assert ok
        has = prev is not None
        pv = prev if has else cam
        vo = np.array([cam[32], cam[33], cam[34], pv[34]], np.float32)
        fc = np.array([cam[35], cam[36], cam[37], cam[38]], np.float32)
        pfc = np.array([pv[35], pv[36], pv[37], 0.0], np.float32)
        pz = np.array([cam[26], cam[30], 0.0, 0.0], np.float32)
        changed = 1.0 if (has and not np.array_equal(prev, cam)) else 0.0
        hc, hx = O.taa(avg, depth, hc, hx, inv, pv[:16], vo, fc, pfc, pz, float(has), changed)
        gc, gx = O.glsl_taa(avg, depth, gc, gx, inv, pv[:16], vo, fc, pfc, pz, float(has), changed)
        assert np.array_equal(_bits(hc), _bits(gc)) and np.array_equal(_bits(hx), _bits(gx)), k
        prev = cam


@live
def test_display_matches_shader():
    """layers_display_fs (LUT sizes 2 to 65, exposures, log2 ranges) and blit_fs
    on frames with zero, huge, subnormal and infinite channels: every output
    bit for bit.  NaN radiance is left out: GLSL does not define it, and the
    oracle defines it as the first lattice entry."""
    rng = np.random.default_rng(31)
    for n, lo, hi, ex in [(2, -10.0, 2.0, 0.0), (5, -3.0, 3.0, 0.5), (17, -12.0, 4.0, 1.5), (33, -6.0, 3.0, -2.25),
                          (65, -16.0, 8.0, 3.0)]:
        img = (rng.random((37, 53, 4)) * 4.0).astype(np.float16)
        img[0, :7, :3] = 0.0
        img[1, :7, :3] = np.float16(65504.0)
        img[2, :7, :3] = np.float16(6e-8)
        img[3, :7, :3] = np.float16(np.inf)
        lut = rng.integers(0, 65536, (n, n, n, 3), dtype=np.uint16)
        assert np.array_equal(_bits(O.display(img, lut, lo, hi, ex)), _bits(O.glsl_display(img, lut, lo, hi, ex))), n
        assert np.array_equal(_bits(O.display(img, None, lo, hi, ex)), _bits(O.glsl_display(img, None, lo, hi, ex)))
