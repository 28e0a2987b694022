"""Float64 restatement of the splatting equations (test infrastructure only).

The FP32 oracle (gs_oracle.c) and the CUDA kernels evaluate the reference's
shaders in single precision, in the shaders' operand order, which is what
makes them bit-exact with each other.  This module evaluates the same
equations in double precision, so a test can state how far the single-
precision path is from the exact arithmetic, per image:

* cull / covariance / conic / radius / centre / SH colour of
  shaders/cull.glsl:209-423 (the same formulas as gs_oracle.c:cull_one);
* far-to-near order of the depth keys (ties by index, shaders/sort.glsl);
* quad coverage of shaders/splat.glsl:39-75 with the GL viewport transform,
  1/256-pixel snapping and top-left fill rule of oc_quad_rect;
* the fragment Gaussian, alpha cut-off and premultiplied back-to-front
  blend of shaders/splat.glsl:88-104 and src/renderer.cpp:276-288.

Everything is float64 except the inputs, which are the float32 rows and
camera.  Vectorised over splats for the projection; the composite loops over
splats in order (small scenes only).
"""
from __future__ import annotations

import numpy as np

SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199
SH_C2 = (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396)
SH_C3 = (-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
         1.445305721320277, -0.5900435899266435)


def _mix(a, b, t):
    return a * (1.0 - t) + b * t


def camera64(cam) -> dict:
    """The 40-float CameraUniforms array (view, proj, viewport, orthographic,
    persp_focal, ortho_focal, clip_y_sign, clip_z_01, pad) as float64 fields."""
    c = np.asarray(cam, dtype=np.float32).reshape(-1).astype(np.float64)
    return dict(view=c[0:16], proj=c[16:32], vp=c[32:34], ortho=c[34], fxp=c[35], fxo=c[36], ysign=c[37],
                z01=c[38])


def project64(rows: np.ndarray, cam, sh_degree: int = 3):
    """(visible mask, positive view depth, N x 16 float64 projected records)."""
    r = np.asarray(rows, dtype=np.float32).reshape(-1, 64).astype(np.float64)
    k = camera64(cam)
    V, P, t = k["view"], k["proj"], k["ortho"]
    px, py, pz, op = r[:, 0], r[:, 1], r[:, 2], r[:, 3]
    vx = V[0] * px + V[4] * py + V[8] * pz + V[12]
    vy = V[1] * px + V[5] * py + V[9] * pz + V[13]
    vz = V[2] * px + V[6] * py + V[10] * pz + V[14]
    vis = vz <= -0.2
    with np.errstate(divide="ignore", invalid="ignore"):
        inv_z = -1.0 / vz
        ndc_x = P[0] * vx * inv_z * (1.0 - t) + P[0] * vx * t
        ndc_y = P[5] * vy * inv_z * (1.0 - t) + P[5] * vy * t
    vis &= (np.abs(ndc_x) <= 1.3) & (np.abs(ndc_y) <= 1.3)

    qw, qx, qy, qz = r[:, 8], r[:, 9], r[:, 10], r[:, 11]
    R = np.empty((r.shape[0], 3, 3))            # R[:, column, row]
    R[:, 0, 0] = 1 - 2 * (qy * qy + qz * qz)
    R[:, 0, 1] = 2 * (qx * qy + qw * qz)
    R[:, 0, 2] = 2 * (qx * qz - qw * qy)
    R[:, 1, 0] = 2 * (qx * qy - qw * qz)
    R[:, 1, 1] = 1 - 2 * (qx * qx + qz * qz)
    R[:, 1, 2] = 2 * (qy * qz + qw * qx)
    R[:, 2, 0] = 2 * (qx * qz + qw * qy)
    R[:, 2, 1] = 2 * (qy * qz - qw * qx)
    R[:, 2, 2] = 1 - 2 * (qx * qx + qy * qy)
    M = R * r[:, 4:7][:, :, None]               # column c scaled by scale[c]
    cov = np.einsum("nkr,nkc->ncr", M, M)       # cov[c][r] = sum_k M[k][r] M[k][c]
    W = np.array([[V[c * 4 + rr] for rr in range(3)] for c in range(3)])
    A = np.einsum("kr,nck->ncr", W, cov)        # A[c][r] = sum_k W[k][r] cov[c][k]
    B = np.einsum("nkr,kc->ncr", A, W)          # B[c][r] = sum_k A[k][r] W[k][c]
    fxp, fxo = k["fxp"], k["fxo"]
    with np.errstate(divide="ignore", invalid="ignore"):
        J00 = _mix(fxp / vz, -fxo, t)
        J11 = _mix(fxp / vz, -fxo, t)
        J02 = _mix(-fxp * vx / (vz * vz), 0.0, t)
        J12 = _mix(-fxp * vy / (vz * vz), 0.0, t)
    a = J00 * J00 * B[:, 0, 0] + 2 * J00 * J02 * B[:, 0, 2] + J02 * J02 * B[:, 2, 2] + 0.3
    b = J00 * J11 * B[:, 0, 1] + J00 * J12 * B[:, 0, 2] + J02 * J11 * B[:, 1, 2] + J02 * J12 * B[:, 2, 2]
    c = J11 * J11 * B[:, 1, 1] + 2 * J11 * J12 * B[:, 1, 2] + J12 * J12 * B[:, 2, 2] + 0.3
    det = np.maximum(a * c - b * b, 1e-6)
    vpx, vpy = k["vp"]
    with np.errstate(divide="ignore", invalid="ignore"):
        cx = _mix(fxp * vx / vz + vpx * 0.5, -fxo * vx + vpx * 0.5, t)
        cy = _mix(vpy * 0.5 + fxp * vy / vz, vpy * 0.5 - fxo * vy, t)
        ndc_z = (P[10] * vz + P[14]) / (-vz)
    ndc_z = _mix(ndc_z, ndc_z * 0.5 + 0.5, k["z01"])
    y_flip = (1.0 - k["ysign"]) * 0.5
    camw = -(W @ V[12:15])
    d = r[:, 0:3] - camw
    x, y, z = (d / np.linalg.norm(d, axis=1)[:, None]).T
    sh = r[:, 16:61].reshape(-1, 15, 3)
    res = SH_C0 * r[:, 12:15]
    if sh_degree >= 1:
        res = res - SH_C1 * y[:, None] * sh[:, 0] + SH_C1 * z[:, None] * sh[:, 1] - SH_C1 * x[:, None] * sh[:, 2]
    if sh_degree >= 2:
        xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
        for k2, f in enumerate([xy, yz, 2 * zz - xx - yy, xz, xx - yy]):
            res = res + (SH_C2[k2] * f)[:, None] * sh[:, 3 + k2]
    if sh_degree >= 3:
        fs = [y * (3 * xx - yy), xy * z, y * (4 * zz - xx - yy), z * (2 * zz - 3 * xx - 3 * yy),
              x * (4 * zz - xx - yy), z * (xx - yy), x * (xx - 3 * yy)]
        for k3, f in enumerate(fs):
            res = res + (SH_C3[k3] * f)[:, None] * sh[:, 8 + k3]
    rgb = np.maximum(res + 0.5, 0.0)
    out = np.zeros((r.shape[0], 16))
    out[:, 0:3] = rgb
    out[:, 3] = op
    out[:, 4] = cx
    out[:, 5] = _mix(cy, vpy - cy, y_flip)
    with np.errstate(invalid="ignore"):
        out[:, 6] = np.ceil(3 * np.sqrt(a))
        out[:, 7] = np.ceil(3 * np.sqrt(c))
    out[:, 8] = c / det
    out[:, 9] = -b / det * k["ysign"]
    out[:, 10] = a / det
    out[:, 11] = ndc_z
    out[:, 12], out[:, 13], out[:, 14], out[:, 15] = a, b * k["ysign"], c, det
    return vis, np.maximum(-vz, 0.0), out


def quad_rect64(p, vp_w, vp_h, ysign, width, height):
    """Covered pixel columns [i0, i1) and GL rows [j0, j1), or None."""
    if not (-1.0 <= p[11] <= 1.0):
        return None
    hw, hh = width * 0.5, height * 0.5
    xa, xb = p[4] - p[6], p[4] + p[6]
    ya, yb = p[5] - p[7], p[5] + p[7]
    X = sorted(int(np.rint(((2 * v / vp_w - 1) * hw + hw) * 256)) for v in (xa, xb))
    Y = sorted(int(np.rint((((2 * v / vp_h - 1) * ysign) * hh + hh) * 256)) for v in (ya, yb))
    i0, i1 = -((128 - X[0]) // 256), -((128 - X[1]) // 256)        # ceil((X - 128) / 256)
    j0, j1 = (Y[0] - 128) // 256 + 1, (Y[1] - 128) // 256 + 1
    i0, j0, i1, j1 = max(i0, 0), max(j0, 0), min(i1, width), min(j1, height)
    return None if (i1 <= i0 or j1 <= j0) else (i0, i1, j0, j1)


def frame64(rows: np.ndarray, cam, width: int, height: int, bg: float = 0.0, sh_degree: int = 3) -> np.ndarray:
    """H x W x 4 float64 RGBA, top row first: the sorted-alpha frame in double precision."""
    vis, depth, proj = project64(rows, cam, sh_degree)
    k = camera64(cam)
    ids = np.nonzero(vis)[0]
    order = ids[np.lexsort((ids, -depth[ids]))]             # far to near, ties by index
    img = np.zeros((height, width, 4))
    img[..., :3] = bg
    for i in order:
        p = proj[i]
        rect = quad_rect64(p, k["vp"][0], k["vp"][1], k["ysign"], width, height)
        if rect is None:
            continue
        i0, i1, j0, j1 = rect
        fx = np.arange(i0, i1) + 0.5 - p[4]
        fy = np.arange(j0, j1) + 0.5 - p[5]
        dx, dy = np.meshgrid(fx, fy)
        power = -0.5 * (p[8] * dx * dx + 2 * p[9] * dx * dy + p[10] * dy * dy)
        cutoff = np.log((1.0 / 255.0) / max(p[3], 1e-8))
        keep = (power <= 0.0) & (power >= cutoff)
        alpha = np.where(keep, np.minimum(p[3] * np.exp(np.minimum(power, 0.0)), 0.99), 0.0)[..., None]
        dst = img[j0:j1, i0:i1]
        dst[..., :3] = p[0:3] * alpha + (1 - alpha) * dst[..., :3]
        dst[..., 3:] = alpha + (1 - alpha) * dst[..., 3:]
    return img[::-1]
