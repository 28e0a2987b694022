"""Generate tests/golden/ref_small.npz from the reference's own CPU code.

Run in a checkout that has the reference sources (oracle/Makefile builds
oracle/_ref/libgsref.so from them):

    python tests/golden/make_golden.py

The fixture holds, for a 256-Gaussian seeded scene written as a 3DGS PLY:
  raw        : the PLY attributes (N x 59 float32)
  rows       : GpuGaussian rows produced by the reference loader
               (gaussian_load_ply + pack_gpu_gaussians)
  view/proj  : camera matrices from the reference camera code
               (camera_get_view_matrix / camera_get_proj_matrix) for 4 poses
  visible_k, depths_k, sorted_k : reference cull_gaussians + sort_gaussians
               output for pose k
Nothing here is read from the reference tree at test time.
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gamesplat_b200 import scene  # noqa: E402
from oracle import oracle as O  # noqa: E402

N = 256
POSES = [
    # (position, yaw, pitch, fov_y, width, height, z_up, ortho_blend)
    ((0.0, 0.0, 3.0), float(np.pi), 0.0, float(np.float32(np.pi / 3)), 1280, 720, 0, 0.0),
    ((0.3, 0.2, 0.6), 3.6, -0.2, float(np.float32(np.pi / 3)), 640, 480, 0, 0.0),
    ((0.0, -2.5, 0.2), 0.1, 0.15, float(np.float32(np.pi / 2)), 512, 512, 1, 0.0),
    ((0.2, 0.1, 2.5), 3.3, 0.05, float(np.float32(np.pi / 3)), 800, 600, 0, 0.5),
]


def main() -> None:
    O.build()
    ref = O.ref()
    raw = scene.small_scene(seed=7, n=N)
    out = {"raw": raw}
    with tempfile.TemporaryDirectory() as td:
        ply = str(Path(td) / "golden.ply").encode()
        scene.write_ply(ply.decode(), raw)
        n = ref.ref_load_ply_rows(ply, None, 0)
        assert n == N
        rows = np.empty((N, 64), np.float32)
        ref.ref_load_ply_rows(ply, rows.ctypes.data, N)
        out["rows"] = rows
        views, projs, meta = [], [], []
        for k, (pos, yaw, pitch, fov, w, h, zup, ob) in enumerate(POSES):
            v = np.empty(16, np.float32)
            p = np.empty(16, np.float32)
            ref.ref_camera_matrices(np.array(pos, np.float32), yaw, pitch, fov, 0.1, 100.0, zup, 1.0, ob,
                                    np.float32(w / h), v, p)
            views.append(v)
            projs.append(p)
            meta.append([pos[0], pos[1], pos[2], yaw, pitch, fov, w, h, zup, ob])
            vis = np.empty(N, np.uint32)
            dep = np.empty(N, np.float32)
            srt = np.empty(N, np.uint32)
            vc = ref.ref_cull_sort_ply(ply, v, p, np.float32(ob), vis, dep, srt)
            out[f"visible_{k}"] = vis[:vc].copy()
            out[f"depths_{k}"] = dep[:vc].copy()
            out[f"sorted_{k}"] = srt[:vc].copy()
        out["view"] = np.stack(views)
        out["proj"] = np.stack(projs)
        out["poses"] = np.array(meta, np.float64)
    np.savez_compressed(Path(__file__).with_name("ref_small.npz"), **out)
    print("wrote", Path(__file__).with_name("ref_small.npz"))


if __name__ == "__main__":
    main()
