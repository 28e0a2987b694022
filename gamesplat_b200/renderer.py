"""Python face of the reference renderer interface (src/renderer.h:249-266),
backed by libgs_cuda.so.  Method names follow the reference functions:

    renderer_init                          -> Renderer(device, stream)
    renderer_upload_gaussians              -> upload_gaussians(rows)
    renderer_set_gps_work_budget           -> set_gps_work_budget(n)
    renderer_reset_stochastic_accumulation -> reset_stochastic_accumulation()
    renderer_draw_frame                    -> draw_frame(cam[, out])
    renderer_destroy                       -> destroy()

Renderer knobs (src/renderer.h:121-247) are attributes: splat_render_mode,
sh_degree, sh_lod_distance, gps_supersample_factor, ... .  Errors raise
GsError (the reference returns false and logs).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

MODE_NAMES = {"alpha": L.GS_MODE_ALPHA, "stochastic": L.GS_MODE_STOCHASTIC, "gps": L.GS_MODE_GPS,
              "denoised": L.GS_MODE_DENOISED}
KNOB_FIELDS = [f for f, _ in L.GsKnobs._fields_ if f != "reserved"]


def _host_ptr(buf) -> int:
    """Address of a host buffer: a torch tensor (data_ptr) or a numpy array."""
    return int(buf.data_ptr()) if hasattr(buf, "data_ptr") else int(buf.ctypes.data)


def camera_from_array(cam) -> L.GsCamera:
    if isinstance(cam, L.GsCamera):
        return cam
    a = np.ascontiguousarray(cam, dtype=np.float32)
    if a.shape != (40,):
        raise ValueError("camera must be 40 float32 (CameraUniforms)")
    s = L.GsCamera()
    C.memmove(C.addressof(s), a.ctypes.data, 160)
    return s


def camera_to_array(cam: L.GsCamera) -> np.ndarray:
    out = np.empty(40, np.float32)
    C.memmove(out.ctypes.data, C.addressof(cam), 160)
    return out


def camera_uniforms(position, yaw: float, pitch: float, width: int, height: int, fov_y: float = np.pi / 3,
                    near_plane: float = 0.1, far_plane: float = 100.0, z_up: bool = False,
                    ortho_size: float = 1.0, ortho_blend: float = 0.0, webgpu: bool = False) -> np.ndarray:
    """CameraUniforms of the reference fly camera (src/camera.cpp:137-245,
    src/main.cpp:1264-1281) as 40 float32."""
    pos = (C.c_float * 3)(*[float(v) for v in position])
    out = L.GsCamera()
    st = L.lib().gs_camera_uniforms(pos, float(yaw), float(pitch), float(fov_y), float(near_plane),
                                    float(far_plane), int(bool(z_up)), float(ortho_size), float(ortho_blend),
                                    int(width), int(height), int(bool(webgpu)), C.byref(out))
    L.check(st, "gs_camera_uniforms")
    return camera_to_array(out)


def load_ply(path: str) -> np.ndarray:
    """GpuGaussian rows (N x 64 float32) of a 3DGS PLY, reference loader transforms."""
    n = L.lib().gs_load_ply(str(path).encode(), None, 0)
    if n < 0:
        raise L.GsError(int(n), "gs_load_ply", str(path))
    rows = np.empty((n, 64), np.float32)
    got = L.lib().gs_load_ply(str(path).encode(), rows.ctypes.data, n)
    if got != n:
        raise L.GsError(int(got) if got < 0 else L.GS_ERR_BAD_ARG, "gs_load_ply", str(path))
    return rows


def load_scene(path: str) -> np.ndarray:
    """GpuGaussian rows (N x 64 float32) of a .ply, .sog or .gsanim file, chosen by extension
    (load_gaussian_scene)."""
    n = L.lib().gs_load_scene(str(path).encode(), None, 0)
    if n < 0:
        raise L.GsError(int(n), "gs_load_scene", str(path))
    rows = np.empty((n, 64), np.float32)
    got = L.lib().gs_load_scene(str(path).encode(), rows.ctypes.data, n)
    if got != n:
        raise L.GsError(int(got) if got < 0 else L.GS_ERR_BAD_ARG, "gs_load_scene", str(path))
    return rows


def load_sog(path: str) -> np.ndarray:
    """GpuGaussian rows (N x 64 float32) of a SOG archive, reference loader decode."""
    n = L.lib().gs_load_sog(str(path).encode(), None, 0)
    if n < 0:
        raise L.GsError(int(n), "gs_load_sog", str(path))
    rows = np.empty((n, 64), np.float32)
    got = L.lib().gs_load_sog(str(path).encode(), rows.ctypes.data, n)
    if got != n:
        raise L.GsError(int(got) if got < 0 else L.GS_ERR_BAD_ARG, "gs_load_sog", str(path))
    return rows


def webp_decode(data: bytes) -> np.ndarray:
    """H x W x 4 uint8 RGBA pixels of a lossless WebP image (the SOG image format)."""
    w, h = C.c_int32(), C.c_int32()
    L.check(L.lib().gs_webp_decode_rgba(data, len(data), C.byref(w), C.byref(h), None, 0), "gs_webp_decode_rgba")
    out = np.empty((h.value, w.value, 4), np.uint8)
    L.check(L.lib().gs_webp_decode_rgba(data, len(data), C.byref(w), C.byref(h), out.ctypes.data, out.size),
            "gs_webp_decode_rgba")
    return out


def pack_raw(raw: np.ndarray) -> np.ndarray:
    """Raw 3DGS attributes (N x 59: xyz, f_dc, f_rest, opacity, scale, rot) -> GpuGaussian rows."""
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    if raw.ndim != 2 or raw.shape[1] != 59:
        raise ValueError("raw must be N x 59 float32")
    rows = np.empty((raw.shape[0], 64), np.float32)
    L.check(L.lib().gs_pack_raw(raw.ctypes.data, raw.shape[0], rows.ctypes.data), "gs_pack_raw")
    return rows


class Renderer:
    """One gs_ctx: a renderer on one CUDA device and stream."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._ctx = C.c_void_p()
        L.check(L.lib().gs_create(C.byref(self._ctx), int(device), C.c_void_p(stream or 0)), "gs_create")
        self.width = 0
        self.height = 0

    # -- lifetime -----------------------------------------------------------
    def destroy(self) -> None:
        if self._ctx:
            L.lib().gs_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- knobs ----------------------------------------------------------------
    def knobs(self) -> L.GsKnobs:
        k = L.GsKnobs()
        L.check(L.lib().gs_get_knobs(self._ctx, C.byref(k)), "gs_get_knobs", self._ctx)
        return k

    def set(self, **kw) -> None:
        k = self.knobs()
        for name, val in kw.items():
            if name == "splat_render_mode":
                name, val = "render_mode", MODE_NAMES.get(val, val) if isinstance(val, str) else val
            if name not in KNOB_FIELDS:
                raise AttributeError(name)
            setattr(k, name, val)
        L.check(L.lib().gs_set_knobs(self._ctx, C.byref(k)), "gs_set_knobs", self._ctx)

    @property
    def splat_render_mode(self) -> int:
        return self.knobs().render_mode

    @splat_render_mode.setter
    def splat_render_mode(self, mode) -> None:
        self.set(splat_render_mode=mode)

    # -- scene ----------------------------------------------------------------
    def upload_gaussians(self, rows: np.ndarray) -> None:
        rows = np.ascontiguousarray(rows, dtype=np.float32)
        if rows.ndim != 2 or rows.shape[1] != 64:
            raise ValueError("rows must be N x 64 float32 GpuGaussian rows")
        L.check(L.lib().gs_upload_rows(self._ctx, rows.ctypes.data, rows.shape[0]), "gs_upload_rows", self._ctx)

    def upload_rows_range(self, rows: np.ndarray, first: int) -> None:
        """Replace rows [first, first + len(rows)) of the resident scene."""
        rows = np.ascontiguousarray(rows, dtype=np.float32)
        if rows.ndim != 2 or rows.shape[1] != 64:
            raise ValueError("rows must be N x 64 float32 GpuGaussian rows")
        L.check(L.lib().gs_upload_rows_range(self._ctx, rows.ctypes.data, int(first), rows.shape[0]),
                "gs_upload_rows_range", self._ctx)

    def upload_gaussians_device(self, ptr: int, count: int) -> None:
        L.check(L.lib().gs_upload_rows_device(self._ctx, C.c_void_p(ptr), count), "gs_upload_rows_device",
                self._ctx)

    def upload_animation(self, deltas: np.ndarray, scales: np.ndarray) -> None:
        """gsanim int8 appearance deltas: (states, N, 48) int8 and 48 float32 scales."""
        deltas = np.ascontiguousarray(deltas, dtype=np.int8)
        scales = np.ascontiguousarray(scales, dtype=np.float32)
        if deltas.ndim != 3 or deltas.shape[2] != 48 or scales.shape != (48,):
            raise ValueError("deltas must be (states, N, 48) int8 and scales 48 float32")
        L.check(L.lib().gs_upload_anim(self._ctx, deltas.ctypes.data, deltas.shape[0], scales.ctypes.data),
                "gs_upload_anim", self._ctx)

    def set_animation_state(self, state_a: int, state_b: int = 0, weight: float = 0.0) -> None:
        L.check(L.lib().gs_set_anim_state(self._ctx, int(state_a), int(state_b), float(weight)),
                "gs_set_anim_state", self._ctx)

    def upload_layers(self, halves: np.ndarray) -> None:
        """gsanim 0.3 appearance layers: (layers, N, 48) uint16 IEEE half bits; 0 layers removes them."""
        halves = np.ascontiguousarray(halves, dtype=np.uint16)
        if halves.ndim != 3 or halves.shape[2] != 48:
            raise ValueError("halves must be (layers, N, 48) uint16")
        L.check(L.lib().gs_upload_layers(self._ctx, halves.ctypes.data, halves.shape[0]), "gs_upload_layers",
                self._ctx)

    def set_layer_weights(self, weights: np.ndarray) -> None:
        """RGB weight per layer for the next frames ((count, 3) float32); an empty array turns layers off."""
        weights = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1, 3)
        L.check(L.lib().gs_set_layer_weights(self._ctx, weights.ctypes.data, weights.shape[0]),
                "gs_set_layer_weights", self._ctx)

    def set_gps_work_budget(self, max_work_items: int) -> bool:
        st = L.lib().gs_set_gps_budget(self._ctx, int(max_work_items))
        if st == L.GS_ERR_BUDGET_REFUSED:
            return False
        L.check(st, "gs_set_gps_budget", self._ctx)
        return True

    # -- batches ---------------------------------------------------------------
    def render_batch(self, cams, out_ptrs) -> None:
        """Alpha frames of several cameras (any viewports) into device images
        (out_ptrs[k]: W_k * H_k * 4 halves), one persistent raster launch."""
        n = len(cams)
        arr = (L.GsCamera * n)(*[camera_from_array(c) for c in cams])
        outs = (C.c_void_p * n)(*[C.c_void_p(p) for p in out_ptrs])
        L.check(L.lib().gs_render_batch(self._ctx, arr, n, outs), "gs_render_batch", self._ctx)

    def render_anim_batch(self, cam, states_a, out_ptrs, states_b=None, weights=None) -> None:
        """gsanim appearance states of one camera into device images."""
        n = len(states_a)
        a = np.ascontiguousarray(states_a, np.int32)
        b = np.ascontiguousarray(states_b if states_b is not None else np.zeros(n), np.int32)
        w = np.ascontiguousarray(weights if weights is not None else np.zeros(n), np.float32)
        outs = (C.c_void_p * n)(*[C.c_void_p(p) for p in out_ptrs])
        c = camera_from_array(cam)
        L.check(L.lib().gs_render_anim_batch(self._ctx, C.byref(c), a.ctypes.data, b.ctypes.data, w.ctypes.data, n,
                                             outs), "gs_render_anim_batch", self._ctx)

    def set_row_format(self, fp16_sh: bool) -> None:
        """Row format of the next upload: FP16 SH coefficients (144-byte rows,
        SH3 on the tensor cores) or the FP32 GpuGaussian rows."""
        L.check(L.lib().gs_set_row_format(self._ctx, int(bool(fp16_sh))), "gs_set_row_format", self._ctx)

    # -- denoised mode ---------------------------------------------------------
    def set_denoiser(self, denoiser) -> None:
        """Attach a gamesplat_b200.denoiser.Denoiser (kept alive by the caller) for the denoised mode."""
        self._denoiser = denoiser
        L.check(L.lib().gs_set_denoiser(self._ctx, denoiser.handle if denoiser is not None else None),
                "gs_set_denoiser", self._ctx)

    def set_denoise_budget(self, tile_mse: float = 1e-4, fallback: bool = True) -> None:
        L.check(L.lib().gs_set_denoise_budget(self._ctx, float(tile_mse), int(bool(fallback))),
                "gs_set_denoise_budget", self._ctx)

    def render_features(self, cam, features_ptr: int) -> None:
        """The denoiser input of the next frame into device memory (H x W x 16 bf16)."""
        c = camera_from_array(cam)
        L.check(L.lib().gs_render_features(self._ctx, C.byref(c), C.c_void_p(features_ptr)), "gs_render_features",
                self._ctx)

    def reset_stochastic_accumulation(self) -> None:
        L.check(L.lib().gs_reset_accumulation(self._ctx), "gs_reset_accumulation", self._ctx)

    # -- display transform ----------------------------------------------------
    def set_display_lut(self, lut, log2_min: float = 0.0, log2_max: float = 1.0) -> None:
        """gsanim 0.3 display LUT: (n, n, n, 3) uint16 indexed [z, y, x, rgb]; None removes it."""
        if lut is None:
            L.check(L.lib().gs_set_display_lut(self._ctx, None, 0, 0.0, 0.0), "gs_set_display_lut", self._ctx)
            return
        lut = np.ascontiguousarray(lut, dtype=np.uint16)
        n = lut.shape[0]
        if lut.shape != (n, n, n, 3):
            raise ValueError("lut must be (n, n, n, 3) uint16")
        L.check(L.lib().gs_set_display_lut(self._ctx, lut.ctypes.data, n, float(log2_min), float(log2_max)),
                "gs_set_display_lut", self._ctx)

    def display(self, in_ptr: int, out_ptr: int, width: int, height: int, exposure_ev: float = 0.0) -> None:
        """Display pass of a gs_render frame (device addresses; stream-ordered)."""
        L.check(L.lib().gs_display(self._ctx, C.c_void_p(in_ptr), C.c_void_p(out_ptr), int(width), int(height),
                                   float(exposure_ev)), "gs_display", self._ctx)

    # -- frames ---------------------------------------------------------------
    def draw_frame(self, cam, out_ptr: int | None = None) -> np.ndarray | None:
        """Render one frame.  With out_ptr (device address of W*H*4 halves) the
        call is stream-ordered and returns None; otherwise it returns the
        RGBA16F image (H x W x 4 float16, top row first) copied to the host."""
        c = camera_from_array(cam)
        if out_ptr is not None:
            L.check(L.lib().gs_render(self._ctx, C.byref(c), C.c_void_p(out_ptr)), "gs_render", self._ctx)
            return None
        w, h = int(c.viewport[0] + 0.5), int(c.viewport[1] + 0.5)
        img = np.empty((h, w, 4), np.float16)
        L.check(L.lib().gs_render_host(self._ctx, C.byref(c), img.ctypes.data), "gs_render_host", self._ctx)
        return img

    def submit_frame(self, cam, host_image) -> None:
        """Queue a frame whose RGBA16F image is copied into the page-locked
        host tensor host_image (H x W x 4 float16, e.g. torch.empty(...,
        pin_memory=True)) while the next frame renders (gs_render_host_submit);
        the image is there after wait_frames(host_image)."""
        c = camera_from_array(cam)
        L.check(L.lib().gs_render_host_submit(self._ctx, C.byref(c), C.c_void_p(_host_ptr(host_image))),
                "gs_render_host_submit", self._ctx)

    def wait_frames(self, host_image=None) -> None:
        """Wait until the submitted frame(s) for host_image (None: all) are in host memory."""
        ptr = None if host_image is None else C.c_void_p(_host_ptr(host_image))
        L.check(L.lib().gs_render_host_wait(self._ctx, ptr), "gs_render_host_wait", self._ctx)

    def stats(self) -> L.GsStats:
        s = L.GsStats()
        L.check(L.lib().gs_read_stats(self._ctx, C.byref(s)), "gs_read_stats", self._ctx)
        return s

    def debug_read(self, which: int, count: int, dtype=np.uint32, shape=None) -> np.ndarray:
        out = np.empty(count, dtype)
        L.check(L.lib().gs_debug_read(self._ctx, int(which), out.ctypes.data, out.nbytes), "gs_debug_read",
                self._ctx)
        return out.reshape(shape) if shape is not None else out

    # -- profiling ------------------------------------------------------------
    def profile(self, enable: bool = True) -> None:
        L.check(L.lib().gs_profile_enable(self._ctx, int(bool(enable))), "gs_profile_enable", self._ctx)

    def stage_times(self, reset: bool = False) -> dict:
        names = L.lib().gs_stage_names().decode().split(",")
        ms = (C.c_float * len(names))()
        launches = (C.c_uint32 * len(names))()
        n = L.lib().gs_stage_times(self._ctx, ms, launches, len(names), int(bool(reset)))
        if n < 0:
            L.check(n, "gs_stage_times", self._ctx)
        return {names[i]: (float(ms[i]), int(launches[i])) for i in range(len(names))}


def sort_pairs_scratch_bytes(n: int) -> int:
    return int(L.lib().gs_sort_pairs_scratch_bytes(int(n)))


def sort_pairs(keys_in: int, vals_in: int, keys_out: int, vals_out: int, n: int, scratch: int,
               scratch_bytes: int, begin_bit: int = 0, end_bit: int = 32, stream: int | None = None) -> None:
    """Stable radix sort of device buffers (device addresses)."""
    st = L.lib().gs_sort_pairs(C.c_void_p(keys_in), C.c_void_p(vals_in), C.c_void_p(keys_out),
                               C.c_void_p(vals_out), int(n), int(begin_bit), int(end_bit), C.c_void_p(scratch),
                               int(scratch_bytes), C.c_void_p(stream or 0))
    L.check(st, "gs_sort_pairs")
