"""Generate tests/golden/shader_small.npz from the reference's own shader
stages (shaders/cull.glsl, sort.glsl, splat.glsl, gps.glsl, accum.glsl), compiled from their source
for the CPU by oracle/Makefile into oracle/_ref/libglslref.so.

Run in a checkout that has the reference sources:

    python tests/golden/make_shader_golden.py

The fixture holds, for a 1024-Gaussian seeded scene (`scene.small_scene(11,
1024)` packed by gs_pack_raw, whose rows ref_small.npz pins against the
reference loader) and four 128 x 80 cameras (perspective; orthographic
blend 0.4; clip y flipped with [0, 1] clip depth; a wide field of view from
inside the scene, which culls about half of it):
  rows                         : N x 64 float32 GpuGaussian rows
  cams                         : 4 x 40 CameraUniforms
  ids_k, keys_k, proj_k, vc_k, diag_k : cull_reset_cs + cull_cs (SH degree 3)
  alpha_k  : splat_vs + splat_fs in depth order with the premultiplied blend,
             background 0, rounded once to half (RGBA16F), top row first
  stoch_k, zstoch_k : splat_vs + splat_stochastic_fs with the D24 LESS test,
             draw order = the cull's index order, frame seed 1, no jitter;
             RGBA8 values (uint8) and D24 depths (uint32)
  gps_k, zgps_k, gpsw_k : gps_clear/expand/splat/resolve, supersample 2,
             frame seed 1, 16M work items; RGBA8 values (uint8), depth
             (float32), requested work items
  sort_in_t, sort_out_t : radix_hist_cs / radix_prefix_cs / radix_scatter_cs
             over the four 8-bit passes of the reference's driver; (key, id)
             pairs in and out (2 x n uint32) for t = cull (camera 3's keys and
             ids, invisible rows' sentinels included) and t = ties (5000 keys
             of 40 values with every byte varying, ids in index order)
  disp_in, disp_lut, disp_params, disp_out, blit_out : layers_display_fs
             (accum.glsl) on a seeded 40 x 64 RGBA16F frame (zero, huge,
             subnormal and infinite channels included) with a 17^3 LUT and
             (log2_min, log2_max, exposure_ev) = disp_params; blit_fs on it
  anim_ids, anim_proj_s : cull_cs with int8 deltas (`scene.anim_deltas(5, N,
             3)`, scales anim_scales) for camera 0 and the (state a, state b,
             weight) of anim_states[s]
Nothing here is read from the reference tree at test time.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gamesplat_b200 import renderer as R  # noqa: E402
from gamesplat_b200 import scene  # noqa: E402
from oracle import oracle as O  # noqa: E402

N = 1024
W, H = 128, 80
ANIM_STATES = np.array([(1, 3, 0.375), (0, 0, 0.3), (2, 2, 0.7)], np.float32)


def cameras():
    pose = scene.small_camera_pose()
    c0 = R.camera_uniforms(*pose, W, H)
    c1 = R.camera_uniforms(*pose, W, H, ortho_blend=0.4)
    c2 = R.camera_uniforms((0.15, -0.1, 2.6), 3.3, 0.08, W, H).copy()
    c2[37] = -1.0   # clip_y_sign
    c2[38] = 1.0    # clip_z_01
    c3 = R.camera_uniforms((0.0, 0.0, 0.3), 3.0, -0.1, W, H, fov_y=1.9)
    return np.stack([c0, c1, c2, c3]).astype(np.float32)


def main() -> None:
    O.build()
    if not O.glsl_available():
        raise SystemExit("oracle/_ref/libglslref.so is missing: the reference sources are needed")
    rows = R.pack_raw(scene.small_scene(11, N))
    cams = cameras()
    out = {"rows": rows, "cams": cams}
    for k, cam in enumerate(cams):
        ids, keys, proj, vc, diag = O.glsl_cull(rows, cam)
        out[f"ids_{k}"], out[f"keys_{k}"], out[f"proj_{k}"] = ids, keys, proj
        out[f"vc_{k}"], out[f"diag_{k}"] = np.uint32(vc), diag
        _, si = O.sort_pairs(keys, ids)
        img, _ = O.glsl_composite_alpha(si, proj, W, H, cam, bg=0.0)
        out[f"alpha_{k}"] = img.astype(np.float16)
        s, z, _ = O.glsl_stochastic_sample(ids, proj, W, H, 1.0, cam, bg=0.0, rgba8=True)
        out[f"stoch_{k}"] = np.rint(s * 255.0).astype(np.uint8)
        out[f"zstoch_{k}"] = np.rint(z.astype(np.float64) * 16777215.0).astype(np.uint32)
        g, gz, requested, overflow = O.glsl_gps_frame(ids, proj, W, H, 2, 16 << 20, 1.0)
        assert overflow == 0
        out[f"gps_{k}"] = np.rint(g * 255.0).astype(np.uint8)
        out[f"zgps_{k}"] = gz
        out[f"gpsw_{k}"] = np.uint32(requested)
    ids, keys, _, _, _ = O.glsl_cull(rows, cams[3])
    ties = np.random.default_rng(12).integers(0, 40, 5000).astype(np.uint32) * np.uint32(0x01010101)
    for name, k, i in (("cull", keys, ids), ("ties", ties, np.arange(ties.size, dtype=np.uint32))):
        ko, io = O.glsl_sort_pairs(k, i)
        out[f"sort_in_{name}"] = np.stack([k, i])
        out[f"sort_out_{name}"] = np.stack([ko, io])
    rng = np.random.default_rng(13)
    img = (rng.random((40, 64, 4)) * 3.0).astype(np.float16)
    img[0, :5, :3] = 0.0
    img[1, :5, :3] = np.float16(60000.0)
    img[2, :5, :3] = np.float16(6e-8)
    img[3, :5, :3] = np.float16(np.inf)
    lut = rng.integers(0, 65536, (17, 17, 17, 3), dtype=np.uint16)
    params = np.array([-12.0, 4.0, 1.5], np.float32)
    out["disp_in"], out["disp_lut"], out["disp_params"] = img, lut, params
    out["disp_out"] = O.glsl_display(img, lut, *params)
    out["blit_out"] = O.glsl_display(img, None, 0.0, 1.0, 0.0)
    deltas = scene.anim_deltas(5, N, 3)
    scales = np.linspace(0.002, 0.02, 48, dtype=np.float32)
    out["anim_scales"] = scales
    out["anim_states"] = ANIM_STATES
    for s, (a, b, w) in enumerate(ANIM_STATES):
        ids, _, proj, _, _ = O.glsl_cull(rows, cams[0], deltas=deltas, scales=scales, state_a=int(a),
                                         state_b=int(b), weight=float(w))
        out["anim_ids"] = ids
        out[f"anim_proj_{s}"] = proj
    dst = Path(__file__).with_name("shader_small.npz")
    np.savez_compressed(dst, **out)
    print(dst, dst.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
