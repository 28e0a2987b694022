"""Benchmark of the per-frame splatting path on B200.

Workload (the one the headline metric is quoted on): 3M SH3 Gaussians
("room3m": 256 clusters + 6 room planes, seed 1), 1920x1080, 120-frame orbit
at radius 6 m, sorted-alpha mode, RGBA16F output.  One step = one frame of
the orbit (cull/SH/project -> depth sort -> bin -> tile sort -> raster).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Timing: W untimed frames, then K frames between CUDA events on the render
stream, barrier + synchronize on both sides, max over ranks.  The scene rows
(768 MB) are larger than L2, so no L2 flush is inserted.  Multi-GPU runs are
replicas (each rank renders its own orbit frames; no collective on the data
path), value = total frames / max time.  `e2e` re-times K frames through
gs_render_host_submit (camera host->device, image device->host each frame,
two frames in flight; all images in host memory when the clock stops), with
the synchronous gs_render_host beside it.
The reference arm (--impl reference) times the CPU oracle port of the same
frame on all host cores, on rows and cameras built by the reference's own
loader and camera code, without loading libgs_cuda.so (the reference's own
CPU code covers only cull + sort; its cull+sort timing is reported beside it).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "1080p fps at 3M splats: sorted-alpha vs denoised stochastic @PSNR≥40dB"
WIDTH, HEIGHT, FRAMES = 1920, 1080, 120
WORKLOAD = "room3m_sh3_1080p_orbit120_sorted_alpha"


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic(*kernels: str):
    """DRAM bytes per launch of the named kernels together (one launch each)
    from the committed ncu capture of the benchmark workload
    (profiles/traffic_room3m_1080p.txt), or None if one is missing."""
    p = ROOT / "profiles" / "traffic_room3m_1080p.txt"
    if not p.exists():
        return None
    found = {}
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0] in kernels:
            found[parts[0]] = int(parts[1])
    if len(found) != len(kernels):
        return None
    return sum(found.values())


def orbit_cameras(width=WIDTH, height=HEIGHT):
    from gamesplat_b200 import renderer as R
    from gamesplat_b200 import scene

    return [R.camera_uniforms(*scene.orbit_pose(k, FRAMES), width, height) for k in range(FRAMES)]


def make_rows(n=3_000_000):
    from gamesplat_b200 import renderer as R
    from gamesplat_b200 import scene

    raw = scene.room_scene(1, n)
    rows = R.pack_raw(raw)
    del raw
    return rows


def bench_config(n, world):
    """The workload, identical in both arms."""
    return {"workload": WORKLOAD, "gaussians": n, "width": WIDTH, "height": HEIGHT, "mode": "alpha",
            "output": "RGBA16F", "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (768 MB of rows), no flush"}


def _scene_module():
    """gamesplat_b200/scene.py (numpy only) loaded by path, so that the
    reference arm never imports the package that wraps libgs_cuda.so."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_bench_scene", ROOT / "gamesplat_b200" / "scene.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_inputs(n=3_000_000):
    """Rows and orbit cameras of the benchmark workload built by the
    reference's own CPU code only (oracle/_ref, compiled from its sources):
    the seeded scene goes through a PLY file into gaussian_load_ply +
    pack_gpu_gaussians, and the cameras come from camera_get_view_matrix /
    camera_get_proj_matrix with the frame setup of src/main.cpp:1264-1281."""
    from oracle import oracle as O

    sc = _scene_module()
    rows = O.ref_rows_from_raw(sc.room_scene(1, n))
    cams = [O.ref_camera_uniforms(*sc.orbit_pose(k, FRAMES), WIDTH, HEIGHT) for k in range(FRAMES)]
    return rows, cams


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        # ranks do the same work between collectives: a short timeout turns a lost rank into an error
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def cpu_frame(rows, cam, threads=None):
    """One oracle frame (cull + sort + composite) on the host; seconds."""
    from oracle import oracle as O

    t = time.perf_counter()
    ids, keys, proj, vc, _ = O.cull(rows, cam, collect_stats=False)
    _, si = O.sort_pairs(keys, ids)
    O.composite_alpha(si, proj, WIDTH, HEIGHT, cam, bg=0.0)
    return time.perf_counter() - t


def reference_cull_sort(rows, cam):
    """The reference's own CPU cull_gaussians + sort_gaussians
    (src/gaussian.cpp:77-181, single-threaded, compiled from its sources into
    oracle/_ref) on the benchmark scene: a reported figure beside the frame
    baseline, or a note of why it is missing.  Never raises."""
    try:
        from oracle import oracle as O

        if not O.ref_available():
            return {"unavailable": "oracle/_ref not built (needs the reference sources)"}
        sec, vis = O.ref_cull_sort_seconds(rows, cam)
        return {"ms": 1000.0 * sec, "threads": 1, "visible": vis, "camera": "orbit frame 0",
                "source": "cull_gaussians + sort_gaussians, src/gaussian.cpp:77-181"}
    except Exception as e:  # a reported extra, never the reason a bench line is missing
        return {"unavailable": f"{type(e).__name__}: {e}"[:200]}


def run_reference(args):
    """The reference arm: the same frames on the host cores.  The reference's
    own renderer draws through GL (unavailable on this box), so each frame is
    the CPU oracle's restatement of that path (cull + SH + sort + composite,
    kind "port"), with rows and cameras built by the reference's own loader
    and camera code; the reference's own CPU cull + sort is timed beside it.
    Rank 0 alone runs; the other ranks exit without work."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    rows, cams = reference_inputs(args.gaussians)
    for i in range(args.warmup):
        cpu_frame(rows, cams[i % FRAMES])
    t0 = time.perf_counter()
    for i in range(args.steps):
        cpu_frame(rows, cams[(args.warmup + i) % FRAMES])
    dt = time.perf_counter() - t0
    fps = args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded room3m scene: 3M SH3 Gaussians, 120-frame orbit cameras)",
        "config": bench_config(rows.shape[0], world),
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full frames of the orbit, oracle cull+SH+sort+composite, "
                                   f"OpenMP on {cores} threads; rows and cameras from the reference's own "
                                   f"PLY loader and camera code"},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cpu_cull_sort": reference_cull_sort(rows, cams[0]),
    }
    print(json.dumps(line), flush=True)


DENOISER_WEIGHTS = ROOT / "gamesplat_b200" / "denoiser_room3m.f32"


def _ssim_psnr(a, b):
    """PSNR (RGBA) and mean SSIM (RGB, 11-tap Gaussian window, sigma 1.5) of
    two H x W x 4 float tensors on the device."""
    import torch
    import torch.nn.functional as F

    mse = float(((a - b) ** 2).mean())
    psnr = float("inf") if mse == 0 else 10.0 * np.log10(1.0 / mse)
    k = torch.exp(-torch.arange(-5, 6, device=a.device, dtype=torch.float32) ** 2 / 4.5)
    k = (k / k.sum()).view(1, 1, 1, 11).repeat(3, 1, 1, 1)

    def blur(t):
        t = F.conv2d(t, k, padding=(0, 5), groups=3)
        return F.conv2d(t, k.transpose(2, 3), padding=(5, 0), groups=3)

    x = a[..., :3].permute(2, 0, 1).unsqueeze(0)
    y = b[..., :3].permute(2, 0, 1).unsqueeze(0)
    mx, my = blur(x), blur(y)
    sxx, syy, sxy = blur(x * x) - mx * mx, blur(y * y) - my * my, blur(x * y) - mx * my
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    s = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
    return psnr, float(s[..., 5:-5, 5:-5].mean())


def denoised_mode(r, stream, out, frame, args, rank):
    """The denoised stochastic mode on the benchmark scene: frame time over the
    orbit (two stochastic samples per pixel, TAA history, the denoiser and
    the sorted-alpha fallback of tiles over the 40 dB budget), and its quality
    against the sorted-alpha frame on held-out random orbit cameras (each
    after `history` frames approaching it along the orbit): PSNR and SSIM with
    and without the fallback, and the fallback rate."""
    import torch

    from gamesplat_b200 import Denoiser
    from gamesplat_b200.train_denoiser import ORBIT_FRAMES, orbit_camera

    if not DENOISER_WEIGHTS.exists():
        return {"unavailable": "no trained denoiser parameters (gamesplat_b200/denoiser_room3m.f32)"}
    d = Denoiser(0, stream=stream.cuda_stream)
    d.set_params(np.fromfile(DENOISER_WEIGHTS, dtype="<f4"))
    r.set_denoiser(d)
    r.set_denoise_budget(1e-4, True)
    r.set(splat_render_mode="denoised", black_background=1)
    r.reset_stochastic_accumulation()
    nm = min(args.steps, 20) if args.denoise_frames is None else args.denoise_frames
    for i in range(5):
        r.draw_frame(frame(i), out_ptr=out.data_ptr())
    stream.synchronize()
    r.profile(True)
    r.stage_times(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fb = 0
    for i in range(nm):
        r.draw_frame(frame(args.warmup + i), out_ptr=out.data_ptr())
    e1.record(stream)
    stream.synchronize()
    mms = e0.elapsed_time(e1) / nm
    st_m = {k: round(v[0] / nm, 4) for k, v in r.stage_times(reset=True).items() if v[0] > 0}
    r.profile(False)
    entry = {"ms_per_frame": mms, "fps": 1000.0 / mms, "frames": nm, "stages_ms_per_frame": st_m,
             "samples_per_pixel": 2, "tile_budget_db": 40.0, "denoiser": "5 x 3x3 conv, 32 ch, U-Net skip, bf16 "
             "tensor cores (tcgen05), fp32 accumulation"}
    # quality on held-out cameras
    cams = args.denoise_eval_cameras
    if cams > 0 and rank == 0:
        rng = np.random.default_rng(5)          # training cameras use seed 4
        angles = rng.uniform(0.0, 2.0 * np.pi, size=cams)
        step = 2.0 * np.pi / ORBIT_FRAMES
        W, H = WIDTH, HEIGHT
        alpha_r = type(r)(0, stream=stream.cuda_stream)
        alpha_r.set(splat_render_mode="alpha", black_background=1)
        alpha_r.upload_gaussians(_bench_rows_cache[0])
        ref = torch.empty(H, W, 4, dtype=torch.float16, device="cuda")
        img_fb = torch.empty(H, W, 4, dtype=torch.float16, device="cuda")
        img_nf = torch.empty(H, W, 4, dtype=torch.float16, device="cuda")
        ps_fb, ss_fb, ps_nf, ss_nf, fbt = [], [], [], [], []
        tiles = ((W + 15) // 16) * ((H + 15) // 16)
        for a in angles:
            for budget_fb, img in ((True, img_fb), (False, img_nf)):
                r.set_denoise_budget(1e-4, budget_fb)
                r.reset_stochastic_accumulation()
                for k in range(args.denoise_history, -1, -1):
                    r.draw_frame(orbit_camera(float(a) - k * step, W, H), out_ptr=img.data_ptr())
                if budget_fb:
                    fbt.append(r.stats().denoise_fallback_tiles / tiles)
            alpha_r.draw_frame(orbit_camera(float(a), W, H), out_ptr=ref.data_ptr())
            stream.synchronize()
            p, s_ = _ssim_psnr(img_fb.float(), ref.float())
            ps_fb.append(p)
            ss_fb.append(s_)
            p, s_ = _ssim_psnr(img_nf.float(), ref.float())
            ps_nf.append(p)
            ss_nf.append(s_)
        alpha_r.destroy()
        entry["quality"] = {
            "cameras": cams, "history_frames": args.denoise_history, "seed": 5,
            "psnr_db_mean": float(np.mean(ps_fb)), "psnr_db_min": float(np.min(ps_fb)),
            "ssim_mean": float(np.mean(ss_fb)), "fallback_tile_rate": float(np.mean(fbt)),
            "frames_at_or_above_40db": float(np.mean(np.asarray(ps_fb) >= 40.0)),
            "denoiser_only_psnr_db_mean": float(np.mean(ps_nf)), "denoiser_only_ssim_mean": float(np.mean(ss_nf)),
            "denoiser_only_frames_at_or_above_40db": float(np.mean(np.asarray(ps_nf) >= 40.0)),
        }
    r.set_denoiser(None)
    d.close()
    return entry


_bench_rows_cache = []


def batched_mode(r, stream, args):
    """Batched variant on the benchmark scene: 64 cameras (4-8 m shell, aimed
    within 1 m of the origin, viewports cycling 512x512 / 1280x720 /
    1920x1080) in one gs_render_batch, against the same frames one gs_render
    each; and gsanim appearance states (1M Gaussians x 256 int8 states, 32 per
    gs_render_anim_batch) against one frame per state."""
    import torch

    from gamesplat_b200 import Renderer
    from gamesplat_b200 import renderer as R
    from gamesplat_b200 import scene

    out = {}
    cams = [R.camera_uniforms(p, y, pt, w, h) for p, y, pt, w, h in scene.batch_cameras(3, 64)]
    bufs = [torch.empty(int(c[32]) * int(c[33]) * 4, dtype=torch.float16, device="cuda") for c in cams]
    ptrs = [b.data_ptr() for b in bufs]
    r.set(splat_render_mode="alpha", black_background=1)

    def timed(fn, reps):
        fn()
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / reps

    # the autotuner picks the tile shape and the frames per raster launch
    import ctypes as C

    from gamesplat_b200 import _lib as L

    arr = (L.GsCamera * len(cams))(*[R.camera_from_array(c) for c in cams])
    cptr = (C.c_void_p * len(cams))(*[C.c_void_p(p) for p in ptrs])
    tune = L.GsTuneResult()
    L.check(L.lib().gs_autotune_batch(r._ctx, arr, len(cams), cptr, C.byref(tune)), "gs_autotune_batch")
    out["autotuner"] = {"tile": f"{tune.tile_w}x{tune.tile_h}", "batch_depth": int(tune.batch_depth),
                        "best_ms": float(tune.best_ms),
                        "tried": [{"tile": f"{tune.tried_tile_w[i]}x{tune.tried_tile_h[i]}",
                                   "batch_depth": int(tune.tried_depth[i]), "ms": float(tune.tried_ms[i])}
                                  for i in range(tune.tried)]}
    reps = 3
    t_batch = timed(lambda: r.render_batch(cams, ptrs), reps)
    t_seq = timed(lambda: [r.draw_frame(c, out_ptr=p) for c, p in zip(cams, ptrs)], reps)
    # the same frames one gs_render each, grouped by viewport (the context's targets
    # are re-sized 3 times per batch instead of at every frame)
    order = sorted(range(len(cams)), key=lambda k: (int(cams[k][32]), int(cams[k][33])))
    t_seq_grouped = timed(lambda: [r.draw_frame(cams[k], out_ptr=ptrs[k]) for k in order], reps)
    mix = {}
    for (w, h) in scene.BATCH_VIEWPORTS:
        sel = [(c, p) for c, p in zip(cams, ptrs) if int(c[32]) == w and int(c[33]) == h]
        tb = timed(lambda: r.render_batch([c for c, _ in sel], [p for _, p in sel]), reps)
        mix[f"{w}x{h}"] = {"cameras": len(sel), "batch_frames_per_s": 1000.0 * len(sel) / tb}
    out["cameras"] = {"count": len(cams), "viewports": "512x512 / 1280x720 / 1920x1080 cycling",
                      "batch_ms": t_batch, "batch_frames_per_s": 1000.0 * len(cams) / t_batch,
                      "sequential_ms": t_seq, "sequential_frames_per_s": 1000.0 * len(cams) / t_seq,
                      "sequential_note": "one gs_render per camera in the batch's order: the viewport changes "
                                         "at every frame, so the context re-sizes its targets every frame",
                      "sequential_grouped_ms": t_seq_grouped,
                      "sequential_grouped_frames_per_s": 1000.0 * len(cams) / t_seq_grouped,
                      "per_viewport": mix}
    # gsanim states: 1M Gaussians x 256 states, 32 per launch
    n_anim, states, per = args.anim_gaussians, 256, 32
    if n_anim > 0:
        rows = R.pack_raw(scene.room_scene(1, n_anim))
        # round(N(0, 20)) clipped to [-127, 127], drawn on the device (12 GB: numpy would take minutes)
        g = torch.Generator(device="cuda").manual_seed(3)
        deltas = np.empty((states - 1, n_anim, 48), np.int8)
        for sidx in range(states - 1):
            d = torch.randn(n_anim, 48, device="cuda", generator=g).mul_(20.0).round_().clamp_(-127, 127)
            deltas[sidx] = d.to(torch.int8).cpu().numpy()
        ra = Renderer(0, stream=stream.cuda_stream)
        ra.set(splat_render_mode="alpha", black_background=1)
        ra.upload_gaussians(rows)
        ra.upload_animation(deltas, np.full(48, 1.0 / 256.0, np.float32))
        del deltas
        cam = R.camera_uniforms(*scene.orbit_pose(0, FRAMES), WIDTH, HEIGHT)
        imgs = [torch.empty(WIDTH * HEIGHT * 4, dtype=torch.float16, device="cuda") for _ in range(per)]
        iptr = [b.data_ptr() for b in imgs]

        def all_states_batched():
            for b0 in range(0, states, per):
                ra.render_anim_batch(cam, list(range(b0, b0 + per)), iptr)

        def all_states_single():
            for sidx in range(states):
                ra.set_animation_state(sidx)
                ra.draw_frame(cam, out_ptr=iptr[sidx % per])

        tb = timed(all_states_batched, 1)
        ts = timed(all_states_single, 1)
        ra.destroy()
        out["gsanim_states"] = {"gaussians": n_anim, "states": states, "states_per_launch": per,
                                "viewport": f"{WIDTH}x{HEIGHT}", "batch_ms": tb,
                                "batch_states_per_s": 1000.0 * states / tb, "sequential_ms": ts,
                                "sequential_states_per_s": 1000.0 * states / ts}
    return out


def precision_variant(args):
    """The FP16-SH row format on the larger workload: 6M Gaussians drawn as the
    3M scene (seed 2), 3840x2160, 8 orbit cameras (frames 0, 15, ..., 105).
    Frame time and the cull roofline with 144-byte rows beside the FP32 rows,
    and the error of the FP16-SH frames against the FP32 frames of the same
    cameras (the FP32 path's own distance from float64 is stated by the
    test suite on reduced scenes)."""
    import torch

    from gamesplat_b200 import Renderer
    from gamesplat_b200 import renderer as R
    from gamesplat_b200 import scene

    n = args.precision_gaussians
    W, H = 3840, 2160
    raw = scene.room_scene(2, n)
    rows = R.pack_raw(raw)
    del raw
    cams = [R.camera_uniforms(*scene.orbit_pose(15 * k, FRAMES), W, H) for k in range(8)]
    stream = torch.cuda.Stream()
    imgs, out = {}, {}
    hbm_peak = load_peaks()[0]
    for fmt in ("fp32", "fp16_sh"):
        r = Renderer(0, stream=stream.cuda_stream)
        r.set(splat_render_mode="alpha", black_background=1)
        r.set_row_format(fmt == "fp16_sh")
        r.upload_gaussians(rows)
        o = torch.empty(H * W * 4, dtype=torch.float16, device="cuda")
        for c in cams[:3]:
            r.draw_frame(c, out_ptr=o.data_ptr())
        stream.synchronize()
        r.profile(True)
        r.stage_times(reset=True)
        reps = 3
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            for c in cams:
                r.draw_frame(c, out_ptr=o.data_ptr())
        e1.record(stream)
        stream.synchronize()
        frames = reps * len(cams)
        ms = e0.elapsed_time(e1) / frames
        st = {k: v[0] / frames for k, v in r.stage_times(reset=True).items() if v[0] > 0}
        r.profile(False)
        vis = []
        r.set(splat_diagnostics_enabled=0)
        frames_img = []
        for c in cams:
            r.draw_frame(c, out_ptr=o.data_ptr())
            vis.append(r.stats().visible_count)
            frames_img.append(o.view(H, W, 4).float().clone())
        imgs[fmt] = frames_img
        n_vis = float(np.mean(vis))
        row_rest = 240.0 if fmt == "fp32" else 128.0   # bytes of a visible row beyond its 16-byte head
        alg = 16.0 * n + (row_rest + 64.0) * n_vis + 8.0 * n
        ach = alg / (st["cull"] / 1000.0) / 1e9
        out[fmt] = {"ms_per_frame": ms, "fps": 1000.0 / ms, "stages_ms_per_frame": {k: round(v, 4) for k, v in
                                                                                     st.items()},
                    "row_bytes": 256 if fmt == "fp32" else 144, "visible_per_frame": n_vis,
                    "cull_roofline": {"achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                                      "algorithmic_bytes": alg}}
        r.destroy()
    errs = []
    for a, b in zip(imgs["fp16_sh"], imgs["fp32"]):
        d = (a - b).abs()
        mse = float((d ** 2).mean())
        errs.append({"max_abs": float(d.max()), "psnr_db": float("inf") if mse == 0 else 10 * np.log10(1 / mse),
                     "frac_over_2^-9": float((d > 2.0 ** -9).float().mean())})
    return {"workload": f"room{n // 1_000_000}m_sh3_2160p_8cams", "gaussians": n, "width": W, "height": H,
            "formats": out, "fp16_vs_fp32_per_camera": errs,
            "sh_eval": "SH3 basis (hi + lo FP16) x FP16 coefficients on the tensor cores (mma.m16n8k16, FP32 "
                       "accumulation); covariance, conic and compositing FP32"}


def run_ours(args):
    import torch

    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from gamesplat_b200 import Renderer, replicas

    rows = make_rows(args.gaussians)
    _bench_rows_cache.append(rows)
    n = rows.shape[0]
    cams = orbit_cameras()
    stream = torch.cuda.Stream()
    r = Renderer(local, stream=stream.cuda_stream)
    r.set(splat_render_mode="alpha", black_background=1)
    r.upload_gaussians(rows)
    out = torch.empty(WIDTH * HEIGHT * 4, dtype=torch.float16, device="cuda")

    def frame(i):
        return cams[replicas.frame_index(rank, world, i, FRAMES)]

    if args.only_mode:
        # one secondary figure alone (for profiling captures): no headline line
        if args.only_mode == "denoised":
            res = denoised_mode(r, stream, out, frame, args, rank)
        elif args.only_mode == "precision":
            res = precision_variant(args)
        else:
            res = batched_mode(r, stream, args)
        r.destroy()
        if rank == 0:
            print(json.dumps({"only_mode": args.only_mode, "result": res}), flush=True)
        return

    # untimed warm-up (also sizes the tile-entry buffers via the host path)
    r.draw_frame(frame(0))
    for i in range(args.warmup):
        r.draw_frame(frame(i), out_ptr=out.data_ptr())
    stream.synchronize()
    launches_per_frame = r.stats().kernel_launches
    sampler = ClockSampler(local) if rank == 0 else None

    def barrier():
        if pg:
            pg.barrier()

    barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    vis_sum = 0
    for i in range(args.steps):
        r.draw_frame(frame(args.warmup + i), out_ptr=out.data_ptr())
    ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if sampler else None
    ms = ev0.elapsed_time(ev1)
    stats = r.stats()
    # Per-stage device times: the same frames again with the library's stage
    # events on (kept out of the timed region above, whose frames run without
    # events between their kernels).
    r.profile(True)
    r.stage_times(reset=True)
    for i in range(args.steps):
        r.draw_frame(frame(args.warmup + i), out_ptr=out.data_ptr())
    stream.synchronize()
    stages = r.stage_times(reset=True)
    r.profile(False)
    ms_max = replicas.reduce_max(ms, pg, "cuda")
    fps = replicas.whole_job_rate(args.steps, world, ms_max / 1000.0)

    # visible count and quad-area diagnostics over the timed frames' cameras
    # (outside the timed region) for the roofline units
    vis_counts, quad_frags = [], []
    r.set(splat_diagnostics_enabled=1)
    for i in range(min(args.steps, 8)):
        r.draw_frame(frame(args.warmup + i), out_ptr=out.data_ptr())
        st_i = r.stats()
        vis_counts.append(st_i.visible_count)
        quad_frags.append(st_i.diagnostics[0] * 1024.0)   # shaders/cull.glsl:297-299 (kpix)
    r.set(splat_diagnostics_enabled=0)
    n_vis = float(np.mean(vis_counts))
    frags = float(np.mean(quad_frags))

    # e2e through the public API with host buffers: the camera from host
    # memory, the RGBA16F image read back every frame into a page-locked host
    # buffer (a renderer's readback buffers), streamed (gs_render_host_submit:
    # a frame's copy overlaps the next frame's kernels); beside it the
    # synchronous gs_render_host into page-locked and into pageable memory.
    e2e_fps = e2e_sync_fps = e2e_pageable_fps = None
    if not args.no_e2e:
        from gamesplat_b200 import _lib as L
        from gamesplat_b200.renderer import camera_from_array
        import ctypes as C

        camsC = [camera_from_array(c) for c in cams]

        def e2e_run(ptr):
            for i in range(2):
                L.lib().gs_render_host(r._ctx, C.byref(camsC[i]), ptr)
            barrier()
            t0 = time.perf_counter()
            for i in range(args.steps):
                st = L.lib().gs_render_host(r._ctx, C.byref(camsC[replicas.frame_index(rank, world, args.warmup + i,
                                                                                        FRAMES)]), ptr)
                L.check(st, "gs_render_host", r._ctx)
            dt = time.perf_counter() - t0
            return replicas.whole_job_rate(args.steps, world, replicas.reduce_max(dt, pg, "cuda"))

        def e2e_stream(bufs):
            # gs_render_host_submit per frame into page-locked buffers in turn
            # (two frames in flight: frame i's image is copied while frame
            # i + 1 renders); the timed region ends when every image is in
            # host memory
            for i in range(2):
                L.check(L.lib().gs_render_host_submit(r._ctx, C.byref(camsC[i]), bufs[i % len(bufs)].data_ptr()),
                        "gs_render_host_submit", r._ctx)
            L.check(L.lib().gs_render_host_wait(r._ctx, None), "gs_render_host_wait", r._ctx)
            barrier()
            t0 = time.perf_counter()
            for i in range(args.steps):
                cam_i = camsC[replicas.frame_index(rank, world, args.warmup + i, FRAMES)]
                L.check(L.lib().gs_render_host_submit(r._ctx, C.byref(cam_i), bufs[i % len(bufs)].data_ptr()),
                        "gs_render_host_submit", r._ctx)
            L.check(L.lib().gs_render_host_wait(r._ctx, None), "gs_render_host_wait", r._ctx)
            dt = time.perf_counter() - t0
            return replicas.whole_job_rate(args.steps, world, replicas.reduce_max(dt, pg, "cuda"))

        pinned_img = torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float16, pin_memory=True)
        stream_bufs = [pinned_img, torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float16, pin_memory=True)]
        e2e_fps = e2e_stream(stream_bufs)
        e2e_sync_fps = e2e_run(pinned_img.data_ptr())
        host_img = np.empty((HEIGHT, WIDTH, 4), np.float16)
        e2e_pageable_fps = e2e_run(host_img.ctypes.data)

    # The path's other render modes on the same scene and cameras, with the
    # renderer's defaults (stochastic: TAA, 4 samples per frame; GPS:
    # supersample 2, 16 Mi work items): secondary figures, not the headline.
    modes = {}
    if not args.no_modes:
        nm = min(args.steps, 20)
        for mode in ("stochastic", "gps"):
            r.set(splat_render_mode=mode, black_background=1)
            r.reset_stochastic_accumulation()
            for i in range(3):
                r.draw_frame(frame(i), out_ptr=out.data_ptr())
            stream.synchronize()
            r.profile(True)
            r.stage_times(reset=True)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(nm):
                r.draw_frame(frame(args.warmup + i), out_ptr=out.data_ptr())
            e1.record(stream)
            stream.synchronize()
            mms = e0.elapsed_time(e1) / nm
            st_m = {k: round(v[0] / nm, 4) for k, v in r.stage_times(reset=True).items() if v[0] > 0}
            r.profile(False)
            sm = r.stats()
            entry = {"ms_per_frame": mms, "fps": 1000.0 / mms, "frames": nm, "stages_ms_per_frame": st_m}
            if mode == "stochastic":
                k = r.knobs()
                entry["samples_per_frame"] = int(k.stochastic_taa_current_samples if k.stochastic_taa_enabled
                                                 else k.stochastic_samples_per_frame)
            else:
                k = r.knobs()
                ss = int(k.gps_supersample_factor)
                work = min(int(sm.gps_requested_work_items), int(sm.gps_max_work_items))
                gps_ms = st_m.get("gps", mms)
                entry.update({"supersample": ss, "work_items_per_frame": work,
                              "points_per_s": work * ss * ss / (gps_ms / 1000.0),
                              "atomics_per_s": work * ss * ss / (gps_ms / 1000.0),
                              "budget_exhausted": int(sm.gps_budget_exhausted)})
            modes[mode] = entry
        r.set(splat_render_mode="alpha", black_background=1)

    precision = None
    if not args.no_modes and args.precision_gaussians > 0 and rank == 0:
        precision = precision_variant(args)
    if not args.no_modes and rank == 0:
        modes["batched"] = batched_mode(r, stream, args)
        from gamesplat_b200 import _lib as L

        L.check(L.lib().gs_set_tile_shape(r._ctx, 16, 16), "gs_set_tile_shape")
        L.check(L.lib().gs_set_batch_depth(r._ctx, 0), "gs_set_batch_depth")
    if not args.no_modes:
        den = denoised_mode(r, stream, out, frame, args, rank)
        if den is not None:
            modes["denoised"] = den
        r.set(splat_render_mode="alpha", black_background=1)

    r.destroy()
    if pg:
        pg.destroy_process_group()
    if rank != 0:
        return

    hbm_peak, tflops_peak, peak_src = load_peaks()
    # dominant stage and its roofline (per launch = per frame)
    per_frame = {k: v[0] / args.steps for k, v in stages.items() if v[0] > 0}
    dominant = max(per_frame, key=per_frame.get)
    # algorithmic bytes per frame (per-unit figures of the scope table):
    #   cull: 16 N + 272 N_vis + 8 N; sort: 68 N_vis (compacted sort length)
    alg = {
        "cull": 16.0 * n + 272.0 * n_vis + 8.0 * n,
        "sort": 68.0 * n_vis,
    }
    # The roofline kernel is the HBM-bound cull (its two launches, visibility
    # and projection, timed together as the cull stage); the raster (the
    # dominant stage) is issue-bound and reported separately in fragments/s.
    roof_stage = "cull"
    achieved = alg[roof_stage] / (per_frame[roof_stage] / 1000.0) / 1e9
    traffic = profiled_traffic("cull_visible_kernel", "cull_project_kernel") if n == 3_000_000 else None
    roofline = {"bound": "hbm", "kernel": "cull_visible_kernel + cull_project_kernel<16>", "achieved": achieved,
                "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": traffic,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": alg[roof_stage],
                "traffic_source": "profiles/cull_visible_kernel_room3m_1080p.md + "
                                  "profiles/cull_project_kernel_room3m_1080p.md" if traffic else None}
    raster = {"kernel": "raster_kernel<0>", "ms_per_frame": per_frame.get("raster"),
              "share_of_frame": per_frame.get("raster", 0.0) / (ms_max / args.steps),
              "bound": "instruction issue (ALU pipe)", "quad_fragments_per_frame": frags,
              "reference_equivalent_fragments_per_s": frags / (per_frame["raster"] / 1000.0)
              if per_frame.get("raster") else None}
    hbm_stages = {}
    for k in alg:
        if k in per_frame:
            a = alg[k] / (per_frame[k] / 1000.0) / 1e9
            hbm_stages[k] = {"ms": per_frame[k], "achieved_gbs": a, "frac": a / hbm_peak}

    cpu = None
    ref_cull_sort = None
    if not args.no_cpu_baseline and world == 1:
        cores = os.cpu_count() or 1
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
        t = cpu_frame(rows, cams[0])
        cpu = {"value": 1.0 / t, "unit": "frames/s", "cores": cores, "kind": "port",
               "sample": f"1 full frame (orbit frame 0), oracle cull+SH+sort+composite on {cores} threads"}
        ref_cull_sort = reference_cull_sort(rows, cams[0])

    line = {
        "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded room3m scene: 3M SH3 Gaussians, 120-frame orbit cameras)",
        "config": bench_config(n, world),
        "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": 160,
                "d2h_bytes_per_step": WIDTH * HEIGHT * 8, "host_buffer": "page-locked",
                "api": "gs_render_host_submit per frame (two frames in flight), gs_render_host_wait at the end",
                "sync_value": e2e_sync_fps, "sync_api": "gs_render_host per frame (returns with the image)",
                "pageable_value": e2e_pageable_fps},
        "gpu_launches": int(launches_per_frame) * args.steps,
        "roofline": roofline,
        "dominant_stage": dominant,
        "raster": raster,
        "modes": modes or None,
        "precision_variant": precision,
        "stages_ms_per_frame": per_frame,
        "hbm_stages": hbm_stages,
        "visible_per_frame": n_vis,
        "tile_entries_last_frame": int(stats.tile_entries),
        "clocks": clocks,
        "cpu_baseline": cpu,
        "reference_cpu_cull_sort": ref_cull_sort,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-modes", action="store_true", help="skip the stochastic and GPS mode figures")
    ap.add_argument("--only-mode", choices=["denoised", "precision", "batched"], default=None,
                    help="run one secondary figure alone and print it (profiling captures), no headline line")
    ap.add_argument("--denoise-eval-cameras", type=int, default=200,
                    help="held-out cameras of the denoised mode's quality figures (0: skip)")
    ap.add_argument("--denoise-history", type=int, default=16,
                    help="frames along the orbit before each held-out camera (the TAA history)")
    ap.add_argument("--denoise-frames", type=int, default=None, help="timed denoised frames (default min(steps, 20))")
    ap.add_argument("--precision-gaussians", type=int, default=6_000_000,
                    help="scene size of the FP16-SH row format figures (0: skip)")
    ap.add_argument("--anim-gaussians", type=int, default=1_000_000,
                    help="scene size of the gsanim state batches (0: skip)")
    ap.add_argument("--gaussians", type=int, default=3_000_000,
                    help="scene size (the benchmark workload is 3M; smaller only for profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
