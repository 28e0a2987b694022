"""CPU tests: pin the oracle (and the host helpers of libgs_cuda.so) against
the reference's own CPU code, through the committed golden fixture
tests/golden/ref_small.npz (made by tests/golden/make_golden.py from
src/gaussian.cpp, src/gaussian_loader_ply.cpp and src/camera.cpp) and, where
the reference sources are present, against oracle/_ref live."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from gamesplat_b200 import renderer as R
from gamesplat_b200 import scene
from oracle import oracle as O

GOLDEN = Path(__file__).with_name("golden") / "ref_small.npz"


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _cam_from_pose(meta):
    px, py, pz, yaw, pitch, fov, w, h, zup, ob = meta
    return R.camera_uniforms((px, py, pz), yaw, pitch, int(w), int(h), fov_y=fov, z_up=bool(zup),
                             ortho_blend=ob)


def test_pack_raw_matches_reference_loader(golden):
    rows = R.pack_raw(golden["raw"])
    assert np.array_equal(rows.view(np.uint32), golden["rows"].view(np.uint32))


def test_ply_loader_matches_reference_loader(golden, tmp_path):
    ply = tmp_path / "g.ply"
    scene.write_ply(str(ply), golden["raw"])
    rows = R.load_ply(str(ply))
    assert np.array_equal(rows.view(np.uint32), golden["rows"].view(np.uint32))


def test_camera_uniforms_match_reference_camera(golden):
    for k, meta in enumerate(golden["poses"]):
        cam = _cam_from_pose(meta)
        assert np.array_equal(cam[:16].view(np.uint32), golden["view"][k].view(np.uint32)), k
        assert np.array_equal(cam[16:32].view(np.uint32), golden["proj"][k].view(np.uint32)), k
        w, h = meta[6], meta[7]
        assert cam[32] == w and cam[33] == h
        # persp_focal = H/2/tan(fov/2) (src/main.cpp:1272)
        assert cam[35] == np.float32((np.float32(1.0) / np.tan(np.float32(meta[5]) * np.float32(0.5))) * np.float32(h) * np.float32(0.5))
        assert cam[37] == 1.0 and cam[38] == 0.0


def test_oracle_cull_matches_reference_cull(golden):
    """Visible set and depth keys of oracle cull == reference cull_gaussians."""
    for k, meta in enumerate(golden["poses"]):
        cam = _cam_from_pose(meta)
        ids, keys, proj, vc, diag = O.cull(golden["rows"], cam)
        vis = np.nonzero(ids != O.SENTINEL)[0].astype(np.uint32)
        assert vc == vis.size
        assert np.array_equal(vis, golden[f"visible_{k}"]), k
        ref_keys = (np.uint32(0xFFFFFFFF) - golden[f"depths_{k}"].view(np.uint32)).astype(np.uint32)
        assert np.array_equal(keys[vis], ref_keys), k
        # culled entries keep the cull_reset sentinels (shaders/cull.glsl:469-472)
        assert np.all(keys[ids == O.SENTINEL] == O.SENTINEL)


def test_oracle_sort_matches_reference_sort_modulo_ties(golden):
    """oracle sort == reference sort_gaussians reversed, except that the
    reference CPU sort orders equal keys by descending index while the GPU
    shader sort keeps ascending index (stable)."""
    for k, meta in enumerate(golden["poses"]):
        cam = _cam_from_pose(meta)
        ids, keys, proj, vc, diag = O.cull(golden["rows"], cam)
        ks, si = O.sort_pairs(keys, ids)
        si = si[:vc]
        ref_back_to_front = golden[f"sorted_{k}"]
        assert ref_back_to_front.size == vc
        # same multiset per key group, and keys ascending = depth descending
        assert np.all(np.diff(ks[:vc].astype(np.int64)) >= 0)
        ref_keys = keys[ref_back_to_front]
        assert np.array_equal(np.sort(ref_keys), ks[:vc])
        # identical ordering when ties are broken the same way
        order = np.lexsort((ref_back_to_front, ref_keys))
        assert np.array_equal(ref_back_to_front[order], si)


@pytest.mark.skipif(not O.ref_available(), reason="reference sources not present")
def test_oracle_cull_sort_live_reference_config0(tmp_path):
    raw = scene.small_scene(0, 100_000)
    ply = tmp_path / "s.ply"
    scene.write_ply(str(ply), raw)
    rows = R.load_ply(str(ply))
    pos, yaw, pitch = scene.small_camera_pose()
    cam = R.camera_uniforms(pos, yaw, pitch, 1280, 720)
    ids, keys, proj, vc, diag = O.cull(rows, cam)
    n = rows.shape[0]
    vis = np.empty(n, np.uint32)
    dep = np.empty(n, np.float32)
    srt = np.empty(n, np.uint32)
    rvc = O.ref().ref_cull_sort_ply(str(ply).encode(), cam[:16].copy(), cam[16:32].copy(), 0.0, vis, dep, srt)
    assert rvc == vc
    mask = ids != O.SENTINEL
    assert np.array_equal(np.nonzero(mask)[0].astype(np.uint32), vis[:rvc])
    assert np.array_equal(keys[mask], (np.uint32(0xFFFFFFFF) - dep[:rvc].view(np.uint32)).astype(np.uint32))


def test_oracle_sort_is_stable_radix():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 12, size=5000, dtype=np.uint32) * np.uint32(0x10001)
    ids = np.arange(5000, dtype=np.uint32)
    ks, si = O.sort_pairs(keys, ids)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(si, ids[order]) and np.array_equal(ks, keys[order])


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def test_deterministic_log_exp_sincos_error_bounds():
    L = O.lib()
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(1e-6, 50, 4000), np.exp(rng.uniform(-80, 80, 4000)), [1.0, 0.5, 2.0]])
    xs = xs.astype(np.float32)
    got = np.array([L.oc_logf(float(x)) for x in xs], np.float32)
    ref = np.log(xs.astype(np.float64)).astype(np.float32)
    assert _ulps(got, ref).max() <= 2
    ys = rng.uniform(-80, 80, 4000).astype(np.float32)
    got = np.array([L.oc_expf(float(y)) for y in ys], np.float32)
    ref = np.exp(ys.astype(np.float64)).astype(np.float32)
    assert _ulps(got, ref).max() <= 2
    zs = rng.uniform(0, 2 * math.pi, 4000).astype(np.float32)
    import ctypes as C

    s = C.c_float()
    c = C.c_float()
    gs_, gc = [], []
    for z in zs:
        L.oc_sincosf(float(z), C.byref(s), C.byref(c))
        gs_.append(s.value)
        gc.append(c.value)
    assert np.abs(np.array(gs_) - np.sin(zs.astype(np.float64))).max() < 2e-7
    assert np.abs(np.array(gc) - np.cos(zs.astype(np.float64))).max() < 2e-7
    assert L.oc_logf(0.0) == -math.inf and L.oc_expf(-200.0) == 0.0


def test_composite_fp16_rounding_gap_is_small():
    """Report-mode check: FP32 blending (round once) vs per-blend fp16
    rounding on the small workload differ by a bounded amount."""
    raw = scene.small_scene(0, 20_000)
    rows = R.pack_raw(raw)
    cam = R.camera_uniforms(*scene.small_camera_pose(), 320, 180)
    ids, keys, proj, vc, _ = O.cull(rows, cam)
    _, si = O.sort_pairs(keys, ids)
    a, fa = O.composite_alpha(si, proj, 320, 180, cam)
    b, fb = O.composite_alpha(si, proj, 320, 180, cam, fp16_per_blend=True)
    assert fa == fb > 0
    gap = np.abs(a.astype(np.float16).astype(np.float32) - b).max()
    assert gap < 0.05


def test_camera_uniforms_random_sweep_match_reference_camera():
    """gs_camera_uniforms against the reference's camera_get_view_matrix /
    camera_get_proj_matrix (src/camera.cpp:137-245) over seeded random fly
    cameras: positions, yaw and pitch over their whole range, field of view,
    near and far planes, z-up, orthographic size and blend, odd aspect ratios."""
    if not O.ref_available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    ref = O.ref()
    rng = np.random.default_rng(123)
    for k in range(500):
        pos = rng.uniform(-50, 50, 3).astype(np.float32)
        yaw, pitch = np.float32(rng.uniform(-7, 7)), np.float32(rng.uniform(-1.55, 1.55))
        fov = np.float32(rng.uniform(0.2, 2.5))
        near = np.float32(rng.uniform(0.01, 1.0))
        far = np.float32(near * rng.uniform(10, 10000))
        z_up = bool(rng.integers(0, 2))
        ortho_size = np.float32(rng.uniform(0.1, 20))
        blend = np.float32(rng.choice([0.0, 1.0, rng.uniform(0, 1)]))
        w, h = int(rng.integers(1, 4096)), int(rng.integers(1, 4096))
        cam = R.camera_uniforms(pos, yaw, pitch, w, h, fov_y=fov, near_plane=near, far_plane=far, z_up=z_up,
                                 ortho_size=ortho_size, ortho_blend=blend)
        view = np.zeros(16, np.float32)
        proj = np.zeros(16, np.float32)
        aspect = np.float32(np.float32(w) / np.float32(h))
        ref.ref_camera_matrices(pos, yaw, pitch, fov, near, far, int(z_up), ortho_size, blend, aspect, view, proj)
        assert np.array_equal(cam[:16].view(np.uint32), view.view(np.uint32)), k
        assert np.array_equal(cam[16:32].view(np.uint32), proj.view(np.uint32)), k


def test_oracle_cull_random_sweep_matches_reference_cull():
    """Visible set and depth keys of the oracle cull against the reference's
    cull_gaussians (src/gaussian.cpp:77-102) over seeded random scenes and
    cameras, orthographic blends included; positions cluster around the near
    plane and the frustum's 1.3 NDC margin so that the boundary cases occur."""
    if not O.ref_available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    ref = O.ref()
    rng = np.random.default_rng(321)
    for k in range(40):
        n = 4000
        w, h = int(rng.integers(64, 2000)), int(rng.integers(64, 2000))
        blend = float(rng.choice([0.0, 1.0, rng.uniform(0, 1)]))
        cam = R.camera_uniforms(rng.uniform(-3, 3, 3), rng.uniform(-3, 3), rng.uniform(-1.4, 1.4), w, h,
                                fov_y=float(rng.uniform(0.3, 2.0)), ortho_size=float(rng.uniform(0.5, 10)),
                                ortho_blend=blend)
        rows = np.zeros((n, 64), np.float32)
        # points along view rays through the NDC margin and depths around the near plane
        V = cam[:16].reshape(4, 4).T.astype(np.float64)         # column-major view matrix
        ndc = rng.uniform(-1.5, 1.5, (n, 2))
        depth = np.where(rng.random(n) < 0.3, rng.uniform(0.15, 0.25, n), rng.uniform(0.2, 40, n))
        p_view = np.stack([ndc[:, 0] * depth, ndc[:, 1] * depth, -depth, np.ones(n)], 1)
        world = (np.linalg.inv(V) @ p_view.T).T[:, :3]
        rows[:, 0:3] = world.astype(np.float32)
        rows[:, 3] = 0.5
        rows[:, 4:7] = 0.01
        rows[:, 8] = 1.0
        ids, keys, _, vc, _ = O.cull(rows, cam)
        vis = np.zeros(n, np.uint32)
        dep = np.zeros(n, np.float32)
        rc = ref.ref_cull_rows(rows.reshape(-1), n, np.ascontiguousarray(cam[:16]), np.ascontiguousarray(cam[16:32]),
                               blend, vis, dep)
        ours = np.nonzero(ids != O.SENTINEL)[0].astype(np.uint32)
        assert rc == vc == ours.size, k
        assert np.array_equal(vis[:rc], ours), k
        ref_keys = (np.uint32(0xFFFFFFFF) - dep[:rc].view(np.uint32)).astype(np.uint32)
        assert np.array_equal(keys[ours], ref_keys), k


def test_oracle_sort_random_sweep_matches_reference_sort_modulo_ties():
    """The oracle's depth order against the reference's sort_gaussians
    (src/gaussian.cpp:116-181) over seeded scenes in which most depths tie
    exactly (points on a few planes facing the camera): the same order once
    ties are broken the same way, the reference giving equal keys in
    descending index and the shader sort in ascending index."""
    if not O.ref_available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    ref = O.ref()
    rng = np.random.default_rng(654)
    for k in range(20):
        n = 3000
        cam = R.camera_uniforms([0.0, 0.0, 0.0], 0.0, 0.0, 640, 360)
        V = cam[:16].reshape(4, 4).T.astype(np.float64)
        levels = rng.uniform(1.0, 30.0, int(rng.integers(1, 12))).astype(np.float32)
        depth = rng.choice(levels, n).astype(np.float64)
        ndc = rng.uniform(-0.5, 0.5, (n, 2))
        p_view = np.stack([ndc[:, 0] * depth, ndc[:, 1] * depth, -depth, np.ones(n)], 1)
        rows = np.zeros((n, 64), np.float32)
        rows[:, 0:3] = (np.linalg.inv(V) @ p_view.T).T[:, :3].astype(np.float32)
        rows[:, 3], rows[:, 4:7], rows[:, 8] = 0.5, 0.01, 1.0
        ids, keys, _, vc, _ = O.cull(rows, cam)
        ks, si = O.sort_pairs(keys, ids)
        srt = np.zeros(n, np.uint32)
        rc = ref.ref_cull_sort_rows(rows.reshape(-1), n, np.ascontiguousarray(cam[:16]),
                                    np.ascontiguousarray(cam[16:32]), 0.0, srt)
        assert rc == vc, k
        back_to_front = srt[:rc]
        ref_keys = keys[back_to_front]
        assert np.array_equal(np.sort(ref_keys), ks[:vc]), k
        assert np.array_equal(back_to_front[np.lexsort((back_to_front, ref_keys))], si[:vc]), k
        assert np.unique(ks[:vc]).size < vc // 10        # ties everywhere
