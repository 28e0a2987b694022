"""ctypes bindings of libgs_cuda.so (include/gs_api.h).

The library is loaded from the package directory only; there is no fallback:
if it is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgs_cuda.so"

GS_OK = 0
GS_ERR_BAD_ARG = -1
GS_ERR_OOM = -2
GS_ERR_CUDA = -3
GS_ERR_DEVICE_TIMEOUT = -4
GS_ERR_NO_SCENE = -5
GS_ERR_BUDGET_REFUSED = -6
GS_ERR_NO_DEVICE = -7
GS_ERR_TOO_LARGE = -8
GS_ERR_FORMAT = -9

GS_MODE_ALPHA = 0
GS_MODE_STOCHASTIC = 1
GS_MODE_GPS = 2
GS_MODE_DENOISED = 3

GS_DEBUG_IDS = 0
GS_DEBUG_KEYS = 1
GS_DEBUG_PROJECTED = 2
GS_DEBUG_SORTED_IDS = 3
GS_DEBUG_SORTED_KEYS = 4
GS_DEBUG_ACCUM = 5
GS_DEBUG_SAMPLE = 6
GS_DEBUG_DEPTH = 7

# Every function include/gs_api.h declares (checked by the CPU test suite).
EXPORTS = (
    "gs_create", "gs_destroy", "gs_get_knobs", "gs_set_knobs", "gs_set_mode", "gs_upload_rows",
    "gs_upload_rows_device", "gs_set_gps_budget", "gs_reset_accumulation", "gs_render", "gs_render_host", "gs_render_host_submit", "gs_render_host_wait",
    "gs_read_stats", "gs_debug_read", "gs_profile_enable", "gs_stage_times", "gs_stage_names", "gs_status_str",
    "gs_last_error", "gs_camera_uniforms", "gs_load_ply", "gs_pack_raw", "gs_sort_pairs_scratch_bytes",
    "gs_sort_pairs", "gs_sort_pairs_noalloc", "gs_upload_anim", "gs_set_anim_state", "gs_set_display_lut",
    "gs_display", "gs_debug_wait_probe", "gs_pack_raw_device", "gs_gsanim_load", "gs_gsanim_free",
    "gs_gsanim_get_info", "gs_gsanim_rows", "gs_gsanim_deltas", "gs_gsanim_layer_data", "gs_gsanim_display_lut",
    "gs_gsanim_layer_name", "gs_gsanim_sample", "gs_gsanim_layer_weights", "gs_webp_decode_rgba",
    "gs_load_sog", "gs_upload_layers", "gs_set_layer_weights", "gs_debug_fail_alloc",
    "gs_load_scene", "gs_scene_device_bytes", "gs_upload_rows_range",
    "gs_denoiser_param_count", "gs_denoiser_create", "gs_denoiser_destroy", "gs_denoiser_init_params",
    "gs_denoiser_set_params", "gs_denoiser_get_params", "gs_denoiser_get_grads", "gs_denoiser_forward",
    "gs_denoiser_backward", "gs_denoiser_loss", "gs_denoiser_adam", "gs_denoiser_train_step", "gs_denoiser_status",
    "gs_conv3x3_scratch_bytes", "gs_conv3x3_bf16", "gs_conv3x3_wgrad_bf16",
    "gs_set_denoiser", "gs_set_denoise_budget", "gs_render_features", "gs_set_row_format",
    "gs_render_batch", "gs_render_anim_batch", "gs_set_tile_shape", "gs_set_batch_depth", "gs_autotune_batch",
)


class GsCamera(C.Structure):
    """CameraUniforms (src/camera.h:23-38)."""

    _fields_ = [
        ("view", C.c_float * 16),
        ("proj", C.c_float * 16),
        ("viewport", C.c_float * 2),
        ("orthographic", C.c_float),
        ("persp_focal", C.c_float),
        ("ortho_focal", C.c_float),
        ("clip_y_sign", C.c_float),
        ("clip_z_01", C.c_float),
        ("pad", C.c_float * 1),
    ]


class GsKnobs(C.Structure):
    _fields_ = [
        ("render_mode", C.c_int32),
        ("sh_degree", C.c_int32),
        ("sh_lod_distance", C.c_float),
        ("gps_supersample_factor", C.c_uint32),
        ("stochastic_samples_per_frame", C.c_uint32),
        ("stochastic_taa_current_samples", C.c_uint32),
        ("stochastic_accumulation_enabled", C.c_int32),
        ("stochastic_taa_enabled", C.c_int32),
        ("black_background", C.c_int32),
        ("splat_diagnostics_enabled", C.c_int32),
        ("linear_color", C.c_int32),
        ("write_invisible_records", C.c_int32),
        ("gpu_budget_mb", C.c_uint32),
        ("reserved", C.c_int32 * 3),
    ]


class GsStats(C.Structure):
    _fields_ = [
        ("gaussian_count", C.c_uint32),
        ("visible_count", C.c_uint32),
        ("tile_entries", C.c_uint32),
        ("tile_overflow", C.c_uint32),
        ("diagnostics", C.c_uint32 * 8),
        ("gps_requested_work_items", C.c_uint32),
        ("gps_budget_exhausted", C.c_uint32),
        ("gps_max_work_items", C.c_uint32),
        ("sample_count", C.c_uint32),
        ("frame_seed", C.c_uint32),
        ("error_flags", C.c_uint32),
        ("kernel_launches", C.c_uint32),
        ("denoise_fallback_tiles", C.c_uint32),
        ("reserved", C.c_uint32 * 4),
    ]


class GsGsanimInfo(C.Structure):
    """gs_gsanim_info (include/gs_api.h)."""

    _fields_ = [
        ("version", C.c_uint32),
        ("gaussian_count", C.c_uint32),
        ("state_count", C.c_uint32),
        ("layer_count", C.c_uint32),
        ("key_count", C.c_uint32),
        ("lut_size", C.c_uint32),
        ("linear", C.c_int32),
        ("log2_min", C.c_float),
        ("log2_max", C.c_float),
        ("duration_seconds", C.c_double),
    ]


class GsTuneResult(C.Structure):
    """gs_tune_result (include/gs_api.h)."""

    _fields_ = [
        ("tile_w", C.c_int32),
        ("tile_h", C.c_int32),
        ("batch_depth", C.c_uint32),
        ("best_ms", C.c_float),
        ("tried", C.c_uint32),
        ("tried_tile_w", C.c_int32 * 32),
        ("tried_tile_h", C.c_int32 * 32),
        ("tried_depth", C.c_uint32 * 32),
        ("tried_ms", C.c_float * 32),
    ]


assert C.sizeof(GsCamera) == 160
assert C.sizeof(GsKnobs) == 64

_lib = None


class GsError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where} failed: {status_str(status)} ({status})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


def lib() -> C.CDLL:
    """Load libgs_cuda.so; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m gamesplat_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp, u32, u64, i32, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_float
    sig = {
        "gs_create": (i32, [C.POINTER(vp), i32, vp]),
        "gs_destroy": (None, [vp]),
        "gs_get_knobs": (i32, [vp, C.POINTER(GsKnobs)]),
        "gs_set_knobs": (i32, [vp, C.POINTER(GsKnobs)]),
        "gs_set_mode": (i32, [vp, i32]),
        "gs_upload_rows": (i32, [vp, vp, u64]),
        "gs_upload_rows_device": (i32, [vp, vp, u64]),
        "gs_upload_rows_range": (i32, [vp, vp, u64, u64]),
        "gs_set_gps_budget": (i32, [vp, u32]),
        "gs_reset_accumulation": (i32, [vp]),
        "gs_render": (i32, [vp, C.POINTER(GsCamera), vp]),
        "gs_render_host": (i32, [vp, C.POINTER(GsCamera), vp]),
        "gs_render_host_submit": (i32, [vp, C.POINTER(GsCamera), vp]),
        "gs_render_host_wait": (i32, [vp, vp]),
        "gs_read_stats": (i32, [vp, C.POINTER(GsStats)]),
        "gs_debug_read": (i32, [vp, i32, vp, u64]),
        "gs_profile_enable": (i32, [vp, i32]),
        "gs_stage_times": (i32, [vp, C.POINTER(C.c_float), C.POINTER(u32), i32, i32]),
        "gs_stage_names": (C.c_char_p, []),
        "gs_status_str": (C.c_char_p, [i32]),
        "gs_last_error": (C.c_char_p, [vp]),
        "gs_camera_uniforms": (i32, [C.POINTER(f32), f32, f32, f32, f32, f32, i32, f32, f32, i32, i32, i32,
                                     C.POINTER(GsCamera)]),
        "gs_load_ply": (C.c_int64, [C.c_char_p, vp, u64]),
        "gs_pack_raw": (i32, [vp, u64, vp]),
        "gs_sort_pairs_scratch_bytes": (C.c_size_t, [u32]),
        "gs_sort_pairs": (i32, [vp, vp, vp, vp, u32, i32, i32, vp, C.c_size_t, vp]),
        "gs_sort_pairs_noalloc": (i32, [vp, vp, vp, vp, u32, i32, i32, vp]),
        "gs_set_display_lut": (i32, [vp, vp, u32, C.c_float, C.c_float]),
        "gs_display": (i32, [vp, vp, vp, i32, i32, C.c_float]),
        "gs_debug_wait_probe": (i32, [vp, i32, u32]),
        "gs_pack_raw_device": (i32, [vp, u64, vp, vp]),
        "gs_upload_anim": (i32, [vp, vp, u32, vp]),
        "gs_set_anim_state": (i32, [vp, i32, i32, f32]),
        "gs_gsanim_load": (i32, [C.c_char_p, C.POINTER(vp)]),
        "gs_gsanim_free": (None, [vp]),
        "gs_gsanim_get_info": (i32, [vp, C.POINTER(GsGsanimInfo)]),
        "gs_gsanim_rows": (i32, [vp, vp]),
        "gs_gsanim_deltas": (i32, [vp, vp, vp]),
        "gs_gsanim_layer_data": (i32, [vp, vp]),
        "gs_gsanim_display_lut": (i32, [vp, vp]),
        "gs_gsanim_layer_name": (C.c_int64, [vp, u32, vp, u64]),
        "gs_gsanim_sample": (i32, [vp, C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_float)]),
        "gs_gsanim_layer_weights": (i32, [vp, C.c_double, vp]),
        "gs_webp_decode_rgba": (i32, [C.c_char_p, u64, C.POINTER(C.c_int32), C.POINTER(C.c_int32), vp, u64]),
        "gs_load_sog": (C.c_int64, [C.c_char_p, vp, u64]),
        "gs_upload_layers": (i32, [vp, vp, u32]),
        "gs_set_layer_weights": (i32, [vp, vp, u32]),
        "gs_debug_fail_alloc": (i32, [C.c_int64]),
        "gs_load_scene": (C.c_int64, [C.c_char_p, vp, u64]),
        "gs_scene_device_bytes": (u64, [u64, C.c_uint32]),
        "gs_denoiser_param_count": (u64, []),
        "gs_denoiser_create": (i32, [C.POINTER(vp), i32, vp]),
        "gs_denoiser_destroy": (None, [vp]),
        "gs_denoiser_init_params": (i32, [vp, u64]),
        "gs_denoiser_set_params": (i32, [vp, vp, u64]),
        "gs_denoiser_get_params": (i32, [vp, vp, u64]),
        "gs_denoiser_get_grads": (i32, [vp, vp, u64]),
        "gs_denoiser_forward": (i32, [vp, vp, i32, i32, i32, vp]),
        "gs_denoiser_backward": (i32, [vp, vp, vp, i32, i32, i32]),
        "gs_denoiser_loss": (i32, [vp, vp, vp, vp, i32, i32, i32, f32, f32, vp, vp]),
        "gs_denoiser_adam": (i32, [vp, f32]),
        "gs_denoiser_train_step": (i32, [vp, vp, vp, i32, i32, i32, f32, vp]),
        "gs_denoiser_status": (i32, [vp]),
        "gs_conv3x3_scratch_bytes": (C.c_size_t, [i32, i32]),
        "gs_set_denoiser": (i32, [vp, vp]),
        "gs_set_row_format": (i32, [vp, i32]),
        "gs_render_batch": (i32, [vp, vp, u32, vp]),
        "gs_set_tile_shape": (i32, [vp, i32, i32]),
        "gs_set_batch_depth": (i32, [vp, u32]),
        "gs_autotune_batch": (i32, [vp, vp, u32, vp, C.POINTER(GsTuneResult)]),
        "gs_render_anim_batch": (i32, [vp, vp, vp, vp, vp, u32, vp]),
        "gs_set_denoise_budget": (i32, [vp, f32, i32]),
        "gs_render_features": (i32, [vp, C.POINTER(GsCamera), vp]),
        "gs_conv3x3_bf16": (i32, [vp, vp, i32, i32, i32, i32, i32, vp, vp, i32, i32, vp, vp, vp, vp, vp, vp]),
        "gs_conv3x3_wgrad_bf16": (i32, [vp, vp, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def status_str(status: int) -> str:
    try:
        return lib().gs_status_str(status).decode()
    except Exception:  # pragma: no cover - only when the library cannot load
        return "unknown"


def check(status: int, where: str, ctx=None) -> None:
    if status != GS_OK:
        detail = ""
        if ctx:
            detail = lib().gs_last_error(ctx).decode()
        raise GsError(status, where, detail)
