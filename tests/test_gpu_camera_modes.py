"""GPU parity of the camera knobs of the cull (shaders/cull.glsl:209-351):
orthographic blends (the mix() branches of :256-291 with t = 0.5 and 1), the
SH level-of-detail distance (:348-351), and the refusal of the WGPU clip
convention, whose top-left fragment origin the rasteriser does not follow.
Records, keys and mask bit-exact against the CPU oracle; RGBA16F images
within the alpha-path gate."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Renderer, _lib as L
from gamesplat_b200 import renderer as RR
from gamesplat_b200 import scene
from oracle import oracle as O

from helpers import image_gate, oracle_alpha, small_rows

pytestmark = pytest.mark.gpu

W, H = 640, 360


@pytest.fixture(scope="module")
def rows():
    return small_rows()


def cam(**kw):
    pos, yaw, pitch = scene.small_camera_pose()
    return RR.camera_uniforms(pos, yaw, pitch, W, H, **kw)


def records(r, n):
    ids = r.debug_read(L.GS_DEBUG_IDS, n)
    keys = r.debug_read(L.GS_DEBUG_KEYS, n)
    proj = r.debug_read(L.GS_DEBUG_PROJECTED, n * 16, np.float32, (n, 16))
    return ids, keys, proj


@pytest.mark.parametrize("blend,size", [(1.0, 1.2), (0.5, 1.2), (0.25, 3.0)])
def test_orthographic_blend(rows, blend, size):
    c = cam(ortho_blend=blend, ortho_size=size)
    ref_img, ref = oracle_alpha(rows, c, W, H)
    assert ref["vc"] > 0
    n = rows.shape[0]
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1, write_invisible_records=1, splat_diagnostics_enabled=1)
        r.upload_gaussians(rows)
        img = r.draw_frame(c)
        ids, keys, proj = records(r, n)
        st = r.stats()
    assert st.visible_count == ref["vc"]
    assert np.array_equal(ids, ref["ids"])
    assert np.array_equal(keys, ref["keys"])
    assert np.array_equal(proj.view(np.uint32), ref["proj"].view(np.uint32))
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate


@pytest.mark.parametrize("lod", [2.5, 3.0])
def test_sh_lod_distance(rows, lod):
    """Splats beyond the distance take degree 0; the camera at z = 3 over a
    [-1, 1] cube puts both sides of each distance in view."""
    c = cam()
    ids, keys, proj, vc, _ = O.cull(rows, c, sh_degree=3, sh_lod_distance=lod)
    _, _, proj_full, _, _ = O.cull(rows, c, sh_degree=3)
    vis = ids != 0xFFFFFFFF
    changed = (proj[vis, :3] != proj_full[vis, :3]).any(axis=1)
    assert 0 < changed.sum() < vis.sum()
    n = rows.shape[0]
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1, write_invisible_records=1, sh_lod_distance=lod)
        r.upload_gaussians(rows)
        r.draw_frame(c)
        g_ids, g_keys, g_proj = records(r, n)
    assert np.array_equal(g_ids, ids)
    assert np.array_equal(g_keys, keys)
    assert np.array_equal(g_proj.view(np.uint32), proj.view(np.uint32))


def test_wgpu_clip_convention_is_refused(rows):
    wgpu = cam(webgpu=True)
    assert wgpu[37] == -1.0 and wgpu[38] == 1.0
    gl = cam()
    ref_img, _ = oracle_alpha(rows, gl, W, H)
    with Renderer(0) as r:
        r.set(splat_render_mode="alpha", black_background=1)
        r.upload_gaussians(rows)
        for bad in (wgpu, np.where(np.arange(40) == 38, 1.0, gl).astype(np.float32),
                    np.where(np.arange(40) == 37, -1.0, gl).astype(np.float32)):
            with pytest.raises(L.GsError) as e:
                r.draw_frame(bad)
            assert e.value.status == L.GS_ERR_BAD_ARG
        img = r.draw_frame(gl)
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate
