"""GPU tests of the denoised render mode through the C ABI:

- the two-sample stochastic raster (the denoiser's noisy input) against the
  CPU oracle's stochastic sample (shaders/splat.glsl:127-145, un-jittered)
  for both seeds: mean colour, alpha and mean depth bit-exact;
- a denoised frame whose every tile is over the error budget is the
  sorted-alpha frame (the fallback rasterizer), within the alpha parity gate;
- a denoised frame with the fallback off is the network's head: the
  denoiser's forward output on the same features plus the history, in
  RGBA16F.
"""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import Denoiser, Renderer, _lib as L
from gamesplat_b200 import renderer as RR
from gamesplat_b200 import scene
from oracle import oracle as O

from helpers import image_gate, oracle_alpha

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

W, H = 320, 180


@pytest.fixture(scope="module")
def small():
    rows = RR.pack_raw(scene.small_scene(3, 20_000))
    cam = RR.camera_uniforms(*scene.small_camera_pose(), W, H)
    return rows, cam


def _renderer(rows, mode):
    r = Renderer(0)
    r.set(splat_render_mode=mode, black_background=1)
    r.upload_gaussians(rows)
    return r


def test_two_sample_stochastic_input_bit_exact(small):
    rows, cam = small
    feats = torch.zeros(H, W, 16, dtype=torch.bfloat16, device="cuda")
    with _renderer(rows, "denoised") as r:
        r.render_features(cam, feats.data_ptr())
        sample = r.debug_read(L.GS_DEBUG_SAMPLE, W * H * 4, np.float32, (H, W, 4))
        depth = r.debug_read(L.GS_DEBUG_DEPTH, W * H, np.float32, (H, W))
    ids, keys, proj, vc, _ = O.cull(rows, cam)
    s = [O.stochastic_sample(ids, proj, W, H, float(seed), cam, bg=0.0, rgba8=False) for seed in (1, 2)]
    half = np.float32(0.5)
    ref_rgba = ((s[0][0] + s[1][0]) * half).astype(np.float32)
    ref_depth = ((s[0][1] + s[1][1]) * half).astype(np.float32)
    assert np.array_equal(sample.view(np.uint32), ref_rgba.view(np.uint32))
    assert np.array_equal(depth.view(np.uint32), ref_depth.view(np.uint32))
    f = feats.float().cpu().numpy()
    assert np.allclose(f[..., 0:4], ref_rgba, atol=4e-3)
    assert np.allclose(f[..., 4], ref_depth, atol=4e-3)
    assert np.all(f[..., 8:] == 0)


def test_all_tiles_over_budget_give_the_sorted_alpha_frame(small):
    """Budget 0: every tile is rendered again by the sorted-alpha rasterizer."""
    rows, cam = small
    ref_img, _ = oracle_alpha(rows, cam, W, H)
    with Denoiser(0) as d, _renderer(rows, "denoised") as r:
        r.set_denoiser(d)
        r.set_denoise_budget(0.0, True)
        img = r.draw_frame(cam)
        st = r.stats()
    assert st.denoise_fallback_tiles == ((W + 15) // 16) * ((H + 15) // 16)
    gate = image_gate(img, ref_img)
    assert gate["ok"], gate


def test_fallback_off_gives_the_network_head(small):
    rows, cam = small
    feats = torch.zeros(H, W, 16, dtype=torch.bfloat16, device="cuda")
    out = torch.zeros(H, W, 16, dtype=torch.float32, device="cuda")
    with Denoiser(0) as d, _renderer(rows, "denoised") as r, _renderer(rows, "denoised") as r2:
        r.set_denoiser(d)
        r.set_denoise_budget(1e-4, False)
        img = r.draw_frame(cam)
        st = r.stats()
        r2.render_features(cam, feats.data_ptr())   # the same first frame's features
        d.forward(feats.data_ptr(), 1, H, W, out.data_ptr())
        torch.cuda.synchronize()
    assert st.denoise_fallback_tiles == 0
    fv = feats.float()
    head = torch.cat([fv[..., 5:8] + out[..., 0:3], fv[..., 3:4] + out[..., 3:4]], dim=-1)
    ref = head.cpu().numpy().astype(np.float16)
    assert np.array_equal(img.view(np.uint16), ref.view(np.uint16))
