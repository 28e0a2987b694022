"""Seeded synthetic scenes and cameras of the benchmark workloads.

No public dataset is involved: scenes are drawn with numpy's PCG64
(default_rng(seed)) in a fixed order and come out as raw 3DGS attributes
(N x 59 float32 in PLY property order: x y z, f_dc_0..2, f_rest_0..44
(channel-major: R0..14, G0..14, B0..14), opacity (logit), scale_0..2 (log),
rot_0..3 (w, x, y, z, unnormalised)).  gs_pack_raw / the reference PLY loader
turn them into 256-byte GpuGaussian rows.

Workloads:
  small  : 100k Gaussians, positions U[-1,1]^3, log-scale N(-4, 0.5), random
           quaternions, opacity logit N(0, 1.5), SH3 (DC N(0,0.5), rest
           N(0,0.05)); camera at (0,0,3) looking at the origin, 1280x720,
           vertical FOV 60 deg.
  room3m : 3M Gaussians: 70% in 256 anisotropic-size clusters (centres U[-5,5]^3,
           std U[0.05,0.5] m), 30% on the six faces of a +-7 m cube with 1 cm
           normal jitter; log-scale N(-4.5, 0.7); opacity logit N(0.5, 2); SH as
           above; 120-frame orbit at radius 6 m, 1920x1080, FOV 60 deg.
"""
from __future__ import annotations

import math
import struct

import numpy as np

RAW_FLOATS = 59


def _appearance(rng: np.random.Generator, n: int, log_scale_mu: float, log_scale_sd: float,
                op_mu: float, op_sd: float) -> dict:
    log_scale = rng.normal(log_scale_mu, log_scale_sd, size=(n, 3)).astype(np.float32)
    quat = rng.normal(0.0, 1.0, size=(n, 4)).astype(np.float32)
    opacity = rng.normal(op_mu, op_sd, size=n).astype(np.float32)
    dc = rng.normal(0.0, 0.5, size=(n, 3)).astype(np.float32)
    rest = rng.normal(0.0, 0.05, size=(n, 45)).astype(np.float32)
    return dict(log_scale=log_scale, quat=quat, opacity=opacity, dc=dc, rest=rest)


def _assemble(pos: np.ndarray, app: dict) -> np.ndarray:
    n = pos.shape[0]
    raw = np.empty((n, RAW_FLOATS), np.float32)
    raw[:, 0:3] = pos
    raw[:, 3:6] = app["dc"]
    raw[:, 6:51] = app["rest"]
    raw[:, 51] = app["opacity"]
    raw[:, 52:55] = app["log_scale"]
    raw[:, 55:59] = app["quat"]
    return raw


def small_scene(seed: int = 0, n: int = 100_000) -> np.ndarray:
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, size=(n, 3)).astype(np.float32)
    app = _appearance(rng, n, -4.0, 0.5, 0.0, 1.5)
    return _assemble(pos, app)


def room_scene(seed: int = 1, n: int = 3_000_000, clusters: int = 256, cluster_frac: float = 0.7,
               box: float = 5.0, room: float = 7.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n_c = int(round(n * cluster_frac))
    n_p = n - n_c
    centres = rng.uniform(-box, box, size=(clusters, 3))
    stds = rng.uniform(0.05, 0.5, size=clusters)
    which = rng.integers(0, clusters, size=n_c)
    pos_c = centres[which] + rng.normal(0.0, 1.0, size=(n_c, 3)) * stds[which, None]
    face = rng.integers(0, 6, size=n_p)
    uv = rng.uniform(-room, room, size=(n_p, 2))
    jitter = rng.normal(0.0, 0.01, size=n_p)
    axis = face // 2
    sign = np.where(face % 2 == 0, -1.0, 1.0)
    pos_p = np.empty((n_p, 3))
    for a in range(3):
        other = [b for b in range(3) if b != a]
        m = axis == a
        pos_p[m, a] = sign[m] * room + jitter[m]
        pos_p[m, other[0]] = uv[m, 0]
        pos_p[m, other[1]] = uv[m, 1]
    pos = np.concatenate([pos_c, pos_p]).astype(np.float32)
    app = _appearance(rng, n, -4.5, 0.7, 0.5, 2.0)
    return _assemble(pos, app)


def write_ply(path: str, raw: np.ndarray) -> None:
    """Binary little-endian 3DGS PLY with the 59 float properties of `raw`."""
    raw = np.ascontiguousarray(raw, dtype="<f4")
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{k}" for k in range(45)] + \
            ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    assert raw.shape[1] == len(names)
    header = "ply\nformat binary_little_endian 1.0\n" + f"element vertex {raw.shape[0]}\n" + \
             "".join(f"property float {nm}\n" for nm in names) + "end_header\n"
    with open(path, "wb") as f:
        f.write(header.encode())
        f.write(raw.tobytes())


def small_camera_pose():
    """(position, yaw, pitch): camera at (0,0,3) looking at the origin."""
    return (0.0, 0.0, 3.0), math.pi, 0.0


def orbit_pose(k: int, frames: int = 120, radius: float = 6.0):
    """Frame k of the orbit at `radius`, pitch 0, looking at the origin."""
    yaw = np.float32(2.0 * math.pi * k / frames)
    fwd = (math.sin(float(yaw)), 0.0, math.cos(float(yaw)))
    pos = tuple(float(np.float32(-radius * c)) for c in fwd)
    return pos, float(yaw), 0.0


def look_at_pose(position, target):
    """(yaw, pitch) of the reference fly camera (z_up off) at `position` looking
    at `target`: forward = (cos p sin y, sin p, cos p cos y) (src/camera.cpp:22-33)."""
    d = np.asarray(target, np.float64) - np.asarray(position, np.float64)
    d /= np.linalg.norm(d)
    return float(math.atan2(d[0], d[2])), float(math.asin(max(-1.0, min(1.0, d[1]))))


BATCH_VIEWPORTS = ((512, 512), (1280, 720), (1920, 1080))


def batch_cameras(seed: int = 3, count: int = 64):
    """The batched workload's cameras: positions uniform on the 4-8 m shell
    around the origin, each aimed at a point uniform in the 1 m ball, the
    viewport cycling through 512x512, 1280x720 and 1920x1080.  Returns
    [(position, yaw, pitch, width, height)]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        r = rng.uniform(4.0, 8.0)
        t = rng.normal(size=3)
        t *= rng.uniform(0.0, 1.0) ** (1.0 / 3.0) / np.linalg.norm(t)
        pos = tuple(float(np.float32(v)) for v in d * r)
        yaw, pitch = look_at_pose(pos, t)
        w, h = BATCH_VIEWPORTS[k % len(BATCH_VIEWPORTS)]
        out.append((pos, yaw, pitch, w, h))
    return out


def anim_deltas(seed: int, n: int, states: int) -> np.ndarray:
    """gsanim appearance states of the batched workload: int8 SH deltas
    round(N(0, 20)) clipped to [-127, 127], (states, n, 48), for a scale of 1/256."""
    rng = np.random.default_rng(seed)
    out = np.empty((states, n, 48), np.int8)
    for s in range(states):
        out[s] = np.clip(np.rint(rng.normal(0.0, 20.0, size=(n, 48))), -127, 127).astype(np.int8)
    return out

