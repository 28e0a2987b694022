"""Train the stochastic-splat denoiser on pairs the renderer generates itself.

A pair is the denoiser input of a frame (two un-jittered stochastic samples
per pixel, their TAA history built over a short run of frames up to the
camera, and the features, from gs_render_features) and the sorted-alpha
frame of the same camera (the target).  Cameras are random positions on the
benchmark orbit (radius 6 m around the origin, looking at it); the history
comes from `history_frames` frames that approach the camera along the orbit
at the benchmark's speed (3 degrees per frame).  Each training step renders
one pair at full resolution every `batches_per_pair` steps and takes a batch of
random crops from it at every step.

All compute runs in libgs_cuda.so (renderer and the denoiser's kernels);
torch only holds device buffers and slices the crops.

    python -m gamesplat_b200.train_denoiser --out weights.f32 [--pairs 2000]
"""
from __future__ import annotations

import argparse
import math
import time

import numpy as np

ORBIT_FRAMES = 120
ORBIT_RADIUS = 6.0


def orbit_camera(angle: float, width: int, height: int):
    """Camera on the benchmark orbit at `angle` radians (the pose of
    scene.orbit_pose for a fractional frame)."""
    from . import renderer as R

    yaw = np.float32(angle)
    fwd = (math.sin(float(yaw)), 0.0, math.cos(float(yaw)))
    pos = tuple(float(np.float32(-ORBIT_RADIUS * c)) for c in fwd)
    return R.camera_uniforms(pos, float(yaw), 0.0, width, height)


class PairSource:
    """Renders (features, target) pairs of a scene at width x height."""

    def __init__(self, rows, width: int, height: int, history_frames: int = 16, device: int = 0):
        import torch

        from .renderer import Renderer

        self.w, self.h, self.k = width, height, history_frames
        self.feat_r = Renderer(device)
        self.feat_r.set(splat_render_mode="denoised", black_background=1)
        self.feat_r.upload_gaussians(rows)
        self.alpha_r = Renderer(device)
        self.alpha_r.set(splat_render_mode="alpha", black_background=1)
        self.alpha_r.upload_gaussians(rows)
        self.features = torch.zeros(height, width, 16, dtype=torch.bfloat16, device="cuda")
        self.target16 = torch.zeros(height, width, 4, dtype=torch.float16, device="cuda")

    def render(self, angle: float):
        """Features and float target of the camera at `angle` (device tensors)."""
        step = 2.0 * math.pi / ORBIT_FRAMES
        self.feat_r.reset_stochastic_accumulation()
        for i in range(self.k, -1, -1):
            self.feat_r.render_features(orbit_camera(angle - i * step, self.w, self.h), self.features.data_ptr())
        self.alpha_r.draw_frame(orbit_camera(angle, self.w, self.h), out_ptr=self.target16.data_ptr())
        return self.features, self.target16.float()

    def close(self):
        self.feat_r.destroy()
        self.alpha_r.destroy()


def train(rows, pairs: int = 2000, epochs: int = 2, batch: int = 8, crop: int = 256, lr: float = 1e-3,
          width: int = 1920, height: int = 1080, seed: int = 4, log_every: int = 500, denoiser=None,
          batches_per_pair: int = 4):
    """Train a denoiser (new, seeded, unless one is given) on `pairs` random
    orbit cameras, `batches_per_pair` batches of random crops from each
    rendered pair; returns (denoiser, loss history)."""
    import torch

    from .denoiser import Denoiser

    rng = np.random.default_rng(seed)
    angles = rng.uniform(0.0, 2.0 * math.pi, size=pairs)
    d = denoiser or Denoiser(0)
    if denoiser is None:
        d.init_params(seed)
    src = PairSource(rows, width, height)
    xb = torch.zeros(batch, crop, crop, 16, dtype=torch.bfloat16, device="cuda")
    tb = torch.zeros(batch, crop, crop, 4, dtype=torch.float32, device="cuda")
    history = []
    t0 = time.perf_counter()
    steps = pairs * epochs * batches_per_pair
    for it in range(steps):
        if it % batches_per_pair == 0:
            feats, target = src.render(float(angles[(it // batches_per_pair) % pairs]))
        ys = rng.integers(0, height - crop + 1, size=batch)
        xs = rng.integers(0, width - crop + 1, size=batch)
        for b in range(batch):
            xb[b].copy_(feats[ys[b]:ys[b] + crop, xs[b]:xs[b] + crop])
            tb[b].copy_(target[ys[b]:ys[b] + crop, xs[b]:xs[b] + crop])
        # cosine decay to 10 % of the rate
        cur = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * it / steps)))
        want = (it % log_every == 0) or it == steps - 1
        parts = d.train_step(xb.data_ptr(), tb.data_ptr(), batch, crop, crop, cur, want_loss=want)
        if want:
            history.append((it, float(parts[3]), float(parts[0]), float(parts[1]), time.perf_counter() - t0))
    torch.cuda.synchronize()
    src.close()
    return d, history


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="where to write the parameters (float32, little-endian)")
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=2)
    ap.add_argument("--batches-per-pair", type=int, default=4)
    ap.add_argument("--gaussians", type=int, default=3_000_000)
    ap.add_argument("--lr", type=float, default=1e-3)
    args = ap.parse_args()
    from . import renderer as R
    from . import scene

    rows = R.pack_raw(scene.room_scene(1, args.gaussians))
    d, hist = train(rows, pairs=args.pairs, epochs=args.epochs, lr=args.lr, batches_per_pair=args.batches_per_pair)
    for it, loss, l1, ssim, t in hist:
        print(f"step {it:6d}  loss {loss:.5f}  l1 {l1:.5f}  ssim {ssim:.4f}  {t:7.1f} s", flush=True)
    d.params().astype("<f4").tofile(args.out)
    d.close()


if __name__ == "__main__":
    main()
