"""ctypes wrapper around the CPU oracle (liboracle.so), the reference's own
CPU code (_ref/libgsref.so) and the reference's shader stages run on the CPU
(_ref/libglslref.so: shaders/*.glsl translated by glsl/extract.py and run by
glsl/harness.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The product package
(gamesplat_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SENTINEL = 0xFFFFFFFF

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OcCamera(C.Structure):
    """Byte-for-byte CameraUniforms (src/camera.h:23-38)."""

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


def camera_struct(cam: np.ndarray) -> OcCamera:
    """40-float CameraUniforms array -> OcCamera."""
    cam = np.ascontiguousarray(cam, dtype=np.float32)
    assert cam.shape == (40,)
    s = OcCamera()
    C.memmove(C.addressof(s), cam.ctypes.data, 160)
    return s


_lib = None
_ref = None
_glsl = None


def reference_dir():
    """The reference checkout whose sources oracle/_ref is compiled from:
    $GS_REFERENCE_DIR, else a directory named `reference` beside this
    repository; None when neither holds the reference sources."""
    for cand in (os.environ.get("GS_REFERENCE_DIR"), str(HERE.parent.parent / "reference")):
        if cand and (Path(cand) / "src" / "gaussian.cpp").exists():
            return str(Path(cand).resolve())
    return None


def build() -> None:
    """Compile liboracle.so (and _ref/libgsref.so when the reference tree is present)."""
    import subprocess

    cmd = ["make", "-s", "-C", str(HERE)]
    ref_dir = reference_dir()
    if ref_dir:
        cmd.append(f"REF={ref_dir}")
    subprocess.run(cmd, check=True)


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.oc_logf.restype = C.c_float
        L.oc_logf.argtypes = [C.c_float]
        L.oc_expf.restype = C.c_float
        L.oc_expf.argtypes = [C.c_float]
        L.oc_sincosf.restype = None
        L.oc_sincosf.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.oc_dilog.restype = C.c_float
        L.oc_dilog.argtypes = [C.c_float]
        L.oc_inv_dilog.restype = C.c_float
        L.oc_inv_dilog.argtypes = [C.c_float]
        L.oc_cull.restype = None
        L.oc_cull.argtypes = [_f32p, C.c_uint32, C.POINTER(OcCamera), C.c_int, C.c_float, C.c_int,
                              _u32p, _u32p, _f32p, C.POINTER(C.c_uint32), _u32p]
        L.oc_cull_anim.restype = None
        L.oc_cull_anim.argtypes = [_f32p, C.c_uint32, C.POINTER(OcCamera), C.c_int, C.c_float, C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float,
                                   _u32p, _u32p, _f32p, C.POINTER(C.c_uint32), _u32p]
        L.oc_sort_pairs.restype = None
        L.oc_sort_pairs.argtypes = [_u32p, _u32p, C.c_uint32, _u32p, _u32p]
        L.oc_quad_rect.restype = C.c_int
        L.oc_quad_rect.argtypes = [_f32p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                   C.c_int, C.c_int, _i32p]
        L.oc_composite_alpha.restype = C.c_uint64
        L.oc_composite_alpha.argtypes = [_u32p, C.c_uint32, _f32p, C.c_int, C.c_int, C.c_float, C.c_float,
                                         C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, _f32p]
        L.oc_stochastic_sample.restype = C.c_uint64
        L.oc_stochastic_sample.argtypes = [_u32p, C.c_uint32, _f32p, C.c_int, C.c_int, C.c_float, C.c_float,
                                           C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                           _f32p, _f32p]
        L.oc_gps_frame.restype = None
        L.oc_gps_frame.argtypes = [_u32p, C.c_uint32, _f32p, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                   C.c_float, C.c_int, C.c_float, C.c_float, _f32p, _f32p, _u32p]
        L.oc_accum.restype = None
        L.oc_accum.argtypes = [_f32p, _f32p, C.c_float, C.c_uint64, _f32p]
        L.oc_taa.restype = None
        L.oc_taa.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p,
                             _f32p, _f32p, C.c_float, C.c_float, _f32p, _f32p]
        L.oc_mat4_inverse.restype = C.c_int
        L.oc_mat4_inverse.argtypes = [_f32p, _f32p]
        L.oc_halton.restype = C.c_float
        L.oc_halton.argtypes = [C.c_uint32, C.c_uint32]
        L.oc_display.restype = None
        L.oc_display.argtypes = [_u16p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_float,
                                 _f32p]
        L.oc_cull_layers.restype = None
        L.oc_cull_layers.argtypes = [_f32p, C.c_uint32, C.POINTER(OcCamera), C.c_int, C.c_float, C.c_int, C.c_void_p,
                                     C.c_int, C.c_void_p, _u32p, _u32p, _f32p, C.POINTER(C.c_uint32), _u32p]
        L.oc_half_to_float.restype = C.c_float
        L.oc_half_to_float.argtypes = [C.c_uint16]
        _lib = L
    return _lib


def ref_available() -> bool:
    return (HERE / "_ref" / "libgsref.so").exists()


def ref():
    """The reference's own CPU code (compiled from the reference sources)."""
    global _ref
    if _ref is None:
        path = HERE / "_ref" / "libgsref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (needs the reference sources)")
        R = C.CDLL(str(path))
        R.ref_load_ply_rows.restype = C.c_uint32
        R.ref_load_ply_rows.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32]
        R.ref_cull_sort_ply.restype = C.c_uint32
        R.ref_cull_sort_ply.argtypes = [C.c_char_p, _f32p, _f32p, C.c_float, _u32p, _f32p, _u32p]
        R.ref_camera_matrices.restype = None
        R.ref_camera_matrices.argtypes = [_f32p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                          C.c_int, C.c_float, C.c_float, C.c_float, _f32p, _f32p]
        R.ref_camera_uniforms.restype = None
        R.ref_camera_uniforms.argtypes = [_f32p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                                          C.c_int, C.c_int, _f32p]
        vp = C.c_void_p
        R.ref_gsanim_open.restype = vp
        R.ref_gsanim_open.argtypes = [C.c_char_p]
        R.ref_gsanim_close.restype = None
        R.ref_gsanim_close.argtypes = [vp]
        R.ref_gsanim_info.restype = None
        R.ref_gsanim_info.argtypes = [vp, _u32p, _f32p, C.POINTER(C.c_double)]
        for name in ("ref_gsanim_rows", "ref_gsanim_layer_data", "ref_gsanim_display_lut"):
            getattr(R, name).restype = None
            getattr(R, name).argtypes = [vp, vp]
        R.ref_gsanim_deltas.restype = None
        R.ref_gsanim_deltas.argtypes = [vp, vp, vp]
        R.ref_gsanim_layer_name.restype = C.c_uint32
        R.ref_gsanim_layer_name.argtypes = [vp, C.c_uint32, C.c_char_p, C.c_uint32]
        R.ref_gsanim_sample.restype = None
        R.ref_gsanim_sample.argtypes = [vp, C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_float)]
        R.ref_gsanim_layer_weights.restype = C.c_uint32
        R.ref_gsanim_layer_weights.argtypes = [vp, C.c_double, vp]
        R.ref_cull_rows.restype = C.c_uint32
        R.ref_cull_rows.argtypes = [_f32p, C.c_uint32, _f32p, _f32p, C.c_float, _u32p, _f32p]
        R.ref_cull_sort_rows.restype = C.c_uint32
        R.ref_cull_sort_rows.argtypes = [_f32p, C.c_uint32, _f32p, _f32p, C.c_float, _u32p]
        R.ref_time_cull_sort_rows.restype = C.c_double
        R.ref_time_cull_sort_rows.argtypes = [_f32p, C.c_uint32, _f32p, _f32p, C.c_float, C.POINTER(C.c_uint32)]
        R.ref_sog_rows.restype = C.c_uint32
        R.ref_sog_rows.argtypes = [C.c_char_p, vp, C.c_uint32]
        R.ref_webp_decode.restype = C.c_int
        R.ref_webp_decode.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int), vp, C.c_size_t]
        _ref = R
    return _ref


def glsl_available() -> bool:
    return (HERE / "_ref" / "libglslref.so").exists()


def glsl():
    """The reference's shader stages (shaders/cull.glsl, sort.glsl, splat.glsl,
    gps.glsl, accum.glsl) compiled from their own source for the CPU; entry
    points mirror the oracle's oc_cull, oc_sort_pairs, oc_composite_alpha,
    oc_stochastic_sample, oc_gps_frame, oc_accum and oc_taa."""
    global _glsl
    if _glsl is None:
        path = HERE / "_ref" / "libglslref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (needs the reference sources)")
        G = C.CDLL(str(path))
        vp = C.c_void_p
        G.glsl_cull.restype = None
        G.glsl_cull.argtypes = [_f32p, C.c_uint32, _f32p, C.c_int, C.c_float, C.c_int, vp, C.c_int, C.c_int,
                                C.c_int, C.c_float, vp, C.c_int, vp, _u32p, _u32p, _f32p, _u32p, _u32p]
        G.ref_mat4_inverse.restype = C.c_int
        G.ref_mat4_inverse.argtypes = [_f32p, _f32p]
        G.glsl_display.restype = None
        G.glsl_display.argtypes = [_u16p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_float,
                                   _f32p]
        G.glsl_sort_pairs.restype = None
        G.glsl_sort_pairs.argtypes = [_u32p, _u32p, C.c_uint32, _u32p, _u32p]
        G.glsl_composite_alpha.restype = C.c_uint64
        G.glsl_composite_alpha.argtypes = [_u32p, C.c_uint32, _f32p, C.c_int, C.c_int, C.c_float, C.c_float,
                                           C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
        G.glsl_stochastic_sample.restype = C.c_uint64
        G.glsl_stochastic_sample.argtypes = [_u32p, C.c_uint32, _f32p, C.c_int, C.c_int, C.c_float, C.c_float,
                                             C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                             _f32p, _f32p]
        G.glsl_gps_frame.restype = None
        G.glsl_gps_frame.argtypes = [_u32p, C.c_uint32, _f32p, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                     C.c_float, C.c_int, C.c_float, C.c_float, _f32p, _f32p, _u32p]
        G.glsl_accum.restype = None
        G.glsl_accum.argtypes = [_f32p, _f32p, C.c_float, C.c_int, C.c_int, _f32p]
        G.glsl_taa.restype = None
        G.glsl_taa.argtypes = [_f32p, _f32p, _f32p, _f32p, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p,
                               _f32p, _f32p, C.c_float, C.c_float, _f32p, _f32p]
        _glsl = G
    return _glsl


def ref_cull_sort_seconds(rows: np.ndarray, cam: np.ndarray):
    """(seconds, visible count) of the reference's single-threaded CPU
    cull_gaussians + sort_gaussians (src/gaussian.cpp:77-181) on `rows`."""
    rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 64)
    cam = np.asarray(cam, dtype=np.float32).reshape(-1)
    vis = C.c_uint32(0)
    sec = ref().ref_time_cull_sort_rows(rows.reshape(-1), rows.shape[0], np.ascontiguousarray(cam[0:16]),
                                        np.ascontiguousarray(cam[16:32]), float(cam[34]), C.byref(vis))
    return float(sec), int(vis.value)


def ref_camera_uniforms(position, yaw: float, pitch: float, width: int, height: int,
                        fov_y: float = np.pi / 3, near_plane: float = 0.1, far_plane: float = 100.0) -> np.ndarray:
    """CameraUniforms (40 float32) of the reference fly camera, built by the
    reference's own camera code (src/camera.cpp:137-245) and its frame setup
    (src/main.cpp:1264-1281, GL branch)."""
    out = np.zeros(40, np.float32)
    pos = np.asarray(position, np.float32).reshape(3)
    ref().ref_camera_uniforms(pos, float(yaw), float(pitch), float(fov_y), float(near_plane), float(far_plane),
                              int(width), int(height), out)
    return out


def ref_rows_from_raw(raw: np.ndarray, tmpdir=None) -> np.ndarray:
    """GpuGaussian rows of raw 3DGS attributes (N x 59, PLY property order)
    through the reference's own PLY loader and pack_gpu_gaussians
    (src/gaussian_loader_ply.cpp:14-228, src/gaussian.cpp:53-73): the
    attributes are written as a binary PLY file and loaded back."""
    import tempfile

    raw = np.ascontiguousarray(raw, dtype="<f4")
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{k}" for k in range(45)] + \
            ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    header = "ply\nformat binary_little_endian 1.0\n" + f"element vertex {raw.shape[0]}\n" + \
             "".join(f"property float {nm}\n" for nm in names) + "end_header\n"
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        path = os.path.join(d, "scene.ply")
        with open(path, "wb") as f:
            f.write(header.encode())
            f.write(raw.tobytes())
        R = ref()
        n = raw.shape[0]
        rows = np.empty((n, 64), np.float32)
        got = R.ref_load_ply_rows(path.encode(), rows.ctypes.data, n)
    if got != n:
        raise RuntimeError(f"reference PLY loader returned {got} rows for {n}")
    return rows


def ref_sog_rows(path):
    """GpuGaussian rows of a SOG archive through the reference loader
    (gaussian_load_sog + pack_gpu_gaussians), or None when it rejects the file."""
    R = ref()
    n = R.ref_sog_rows(str(path).encode(), None, 0)
    if n == 0:
        return None
    rows = np.zeros((n, 64), np.float32)
    R.ref_sog_rows(str(path).encode(), rows.ctypes.data, n)
    return rows


def ref_webp_decode(data: bytes):
    """H x W x 4 RGBA8 through WebPGetInfo + WebPDecodeRGBA, or None."""
    R = ref()
    w, h = C.c_int(), C.c_int()
    if not R.ref_webp_decode(data, len(data), C.byref(w), C.byref(h), None, 0):
        return None
    out = np.zeros((h.value, w.value, 4), np.uint8)
    R.ref_webp_decode(data, len(data), C.byref(w), C.byref(h), out.ctypes.data, out.size)
    return out


def ref_gsanim(path, times=()):
    """The reference loader's view of a gsanim archive (gaussian_load_gsanim,
    src/gaussian_loader_gsanim.cpp:386-495), or None when it rejects the file:
    a dict of the decoded arrays, plus gsanim_sample and gsanim_layer_weights
    at each of `times`."""
    R = ref()
    h = R.ref_gsanim_open(str(path).encode())
    if not h:
        return None
    try:
        ints = np.zeros(7, np.uint32)
        floats = np.zeros(2, np.float32)
        dur = C.c_double()
        R.ref_gsanim_info(h, ints, floats, C.byref(dur))
        version, n, states, layers, keys, lut, linear = (int(v) for v in ints)
        rows = np.zeros((n, 64), np.float32)
        R.ref_gsanim_rows(h, rows.ctypes.data)
        deltas = np.zeros((max(states - 1, 0), n, 48), np.int8)
        scales = np.zeros(48, np.float32)
        R.ref_gsanim_deltas(h, deltas.ctypes.data, scales.ctypes.data)
        layer_data = np.zeros((layers, n, 48), np.uint16)
        R.ref_gsanim_layer_data(h, layer_data.ctypes.data)
        display_lut = np.zeros((lut ** 3, 3), np.uint16)
        R.ref_gsanim_display_lut(h, display_lut.ctypes.data)
        names = []
        for i in range(layers):
            length = R.ref_gsanim_layer_name(h, i, None, 0)
            buf = C.create_string_buffer(max(int(length), 1))
            R.ref_gsanim_layer_name(h, i, buf, length)
            names.append(buf.raw[:length])
        samples, weights = [], []
        for t in times:
            a, b, w = C.c_int32(), C.c_int32(), C.c_float()
            R.ref_gsanim_sample(h, float(t), C.byref(a), C.byref(b), C.byref(w))
            samples.append((a.value, b.value, w.value))
            out = np.zeros((max(layers, 1), 3), np.float32)
            k = R.ref_gsanim_layer_weights(h, float(t), out.ctypes.data)
            weights.append(out[:k])
        return dict(version=version, gaussian_count=n, state_count=states, layer_count=layers, key_count=keys,
                    lut_size=lut, linear=bool(linear), log2_min=float(floats[0]), log2_max=float(floats[1]),
                    duration=dur.value, rows=rows, deltas=deltas, scales=scales, layer_data=layer_data,
                    display_lut=display_lut, layer_names=names, samples=samples, layer_weights=weights)
    finally:
        R.ref_gsanim_close(h)


# --------------------------------------------------------------------------
# numpy-level helpers
# --------------------------------------------------------------------------
def cull(rows: np.ndarray, cam: np.ndarray, sh_degree: int = 3, sh_lod_distance: float = 0.0,
         collect_stats: bool = True):
    rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 64)
    n = rows.shape[0]
    ids = np.empty(n, np.uint32)
    keys = np.empty(n, np.uint32)
    proj = np.empty((n, 16), np.float32)
    vc = C.c_uint32(0)
    diag = np.zeros(8, np.uint32)
    cs = camera_struct(cam)
    lib().oc_cull(rows.reshape(-1), n, C.byref(cs), int(sh_degree), float(sh_lod_distance),
                  int(bool(collect_stats)), ids, keys, proj.reshape(-1), C.byref(vc), diag)
    return ids, keys, proj, int(vc.value), diag


def cull_layers(rows: np.ndarray, cam: np.ndarray, halves: np.ndarray, weights: np.ndarray, sh_degree: int = 3,
                sh_lod_distance: float = 0.0):
    """oc_cull with gsanim 0.3 layers (halves: (layers, N, 48) uint16 half bits, weights: (layers, 3) float32)."""
    rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 64)
    n = rows.shape[0]
    halves = np.ascontiguousarray(halves, dtype=np.uint16)
    weights = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1, 3)
    ids = np.empty(n, np.uint32)
    keys = np.empty(n, np.uint32)
    proj = np.empty((n, 16), np.float32)
    vc = C.c_uint32(0)
    diag = np.zeros(8, np.uint32)
    cs = camera_struct(cam)
    lib().oc_cull_layers(rows.reshape(-1), n, C.byref(cs), int(sh_degree), float(sh_lod_distance), 1,
                         halves.ctypes.data, int(weights.shape[0]), weights.ctypes.data, ids, keys,
                         proj.reshape(-1), C.byref(vc), diag)
    return ids, keys, proj, int(vc.value), diag


def cull_anim(rows: np.ndarray, cam: np.ndarray, deltas: np.ndarray, scales: np.ndarray, state_a: int,
              state_b: int = 0, weight: float = 0.0, sh_degree: int = 3):
    """oc_cull with gsanim int8 deltas (deltas: (states, N, 48) int8, scales: 48 float32)."""
    rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 64)
    n = rows.shape[0]
    deltas = np.ascontiguousarray(deltas, dtype=np.int8)
    scales = np.ascontiguousarray(scales, dtype=np.float32)
    ids = np.empty(n, np.uint32)
    keys = np.empty(n, np.uint32)
    proj = np.empty((n, 16), np.float32)
    vc = C.c_uint32(0)
    diag = np.zeros(8, np.uint32)
    cs = camera_struct(cam)
    lib().oc_cull_anim(rows.reshape(-1), n, C.byref(cs), int(sh_degree), 0.0, 1, deltas.ctypes.data,
                       scales.ctypes.data, int(state_a), int(state_b), float(weight), ids, keys, proj.reshape(-1),
                       C.byref(vc), diag)
    return ids, keys, proj, int(vc.value), diag


def sort_pairs(keys: np.ndarray, ids: np.ndarray):
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    ko = np.empty_like(keys)
    io = np.empty_like(ids)
    lib().oc_sort_pairs(keys, ids, keys.size, ko, io)
    return ko, io


def composite_alpha(sorted_ids: np.ndarray, projected: np.ndarray, width: int, height: int,
                    cam: np.ndarray | None = None, bg: float = 0.0, jitter=(0.0, 0.0),
                    fp16_per_blend: bool = False):
    vp_w, vp_h, ysign = _vp(cam, width, height)
    out = np.empty((height, width, 4), np.float32)
    sorted_ids = np.ascontiguousarray(sorted_ids, dtype=np.uint32)
    frags = lib().oc_composite_alpha(sorted_ids, sorted_ids.size, np.ascontiguousarray(projected, np.float32).reshape(-1),
                                     width, height, vp_w, vp_h, ysign, float(bg), float(jitter[0]),
                                     float(jitter[1]), int(bool(fp16_per_blend)), out.reshape(-1))
    return out, int(frags)


def sh_to_fp16(rows: np.ndarray) -> np.ndarray:
    """The rows with their SH coefficients (DC at [12:15], the 45 others at
    [16:61]) rounded to IEEE half and back: what a row layout that stores SH
    in FP16 hands the cull, whose arithmetic stays FP32."""
    r = np.array(rows, dtype=np.float32, copy=True).reshape(-1, 64)
    r[:, 12:15] = r[:, 12:15].astype(np.float16).astype(np.float32)
    r[:, 16:61] = r[:, 16:61].astype(np.float16).astype(np.float32)
    return r


def conic_to_fp16(projected: np.ndarray) -> np.ndarray:
    """Projected records with the conic (record floats [8:11]) rounded to IEEE
    half and back: FP16 conic storage between the cull and the compositor."""
    p = np.array(projected, dtype=np.float32, copy=True).reshape(-1, 16)
    p[:, 8:11] = p[:, 8:11].astype(np.float16).astype(np.float32)
    return p


def stochastic_sample(ids: np.ndarray, projected: np.ndarray, width: int, height: int, frame_seed: float,
                      cam: np.ndarray | None = None, bg: float = 0.0, jitter=(0.0, 0.0), rgba8: bool = True):
    vp_w, vp_h, ysign = _vp(cam, width, height)
    out = np.empty((height, width, 4), np.float32)
    depth = np.empty((height, width), np.float32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    kept = lib().oc_stochastic_sample(ids, ids.size, np.ascontiguousarray(projected, np.float32).reshape(-1),
                                      width, height, vp_w, vp_h, ysign, float(bg), float(jitter[0]),
                                      float(jitter[1]), float(frame_seed), int(bool(rgba8)),
                                      out.reshape(-1), depth.reshape(-1))
    return out, depth, int(kept)


def gps_frame(ids: np.ndarray, projected: np.ndarray, width: int, height: int, supersample: int,
              max_work_items: int, frame_seed: float, clip_z_01: float = 0.0, linear_color: bool = False,
              bg: float = 0.0):
    out = np.empty((height, width, 4), np.float32)
    depth = np.empty((height, width), np.float32)
    stats = np.zeros(2, np.uint32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    lib().oc_gps_frame(ids, ids.size, np.ascontiguousarray(projected, np.float32).reshape(-1), width, height,
                       int(supersample), int(max_work_items), float(clip_z_01), int(bool(linear_color)),
                       float(frame_seed), float(bg), out.reshape(-1), depth.reshape(-1), stats)
    return out, depth, int(stats[0]), int(stats[1])


def display(img_half: np.ndarray, lut, log2_min: float, log2_max: float, exposure_ev: float) -> np.ndarray:
    """Display transform (shaders/accum.glsl:201-240, or the blit when lut is None) of an
    (H, W, 4) float16 frame; lut is (n, n, n, 3) uint16 indexed [z, y, x, rgb].  -> (H, W, 4) float32."""
    img = np.ascontiguousarray(img_half, np.float16)
    h, w = img.shape[:2]
    out = np.empty((h, w, 4), np.float32)
    if lut is None:
        lp, n = None, 0
    else:
        lut = np.ascontiguousarray(lut, np.uint16)
        lp, n = lut.ctypes.data, lut.shape[0]
    lib().oc_display(img.view(np.uint16).reshape(-1), w, h, lp, n, float(log2_min), float(log2_max),
                     float(exposure_ev), out.reshape(-1))
    return out


def accum(sample: np.ndarray, history: np.ndarray, n: float):
    sample = np.ascontiguousarray(sample, np.float32)
    history = np.ascontiguousarray(history, np.float32)
    out = np.empty_like(sample)
    lib().oc_accum(sample.reshape(-1), history.reshape(-1), float(n), sample.size, out.reshape(-1))
    return out


def taa(cur_color, cur_depth, hist_color, hist_xyz, inv_view, prev_view, viewport_ortho, focal_clip,
        prev_focal_clip, proj_z, history_valid: float, view_changed: float):
    h, w = cur_depth.shape
    oc = np.empty((h, w, 4), np.float32)
    ox = np.empty((h, w, 4), np.float32)
    f = lambda a: np.ascontiguousarray(a, np.float32).reshape(-1)  # noqa: E731
    lib().oc_taa(f(cur_color), f(cur_depth), f(hist_color), f(hist_xyz), w, h, f(inv_view), f(prev_view),
                 f(viewport_ortho), f(focal_clip), f(prev_focal_clip), f(proj_z), float(history_valid),
                 float(view_changed), oc.reshape(-1), ox.reshape(-1))
    return oc, ox


def mat4_inverse(m: np.ndarray):
    """(ok, inverse) of a column-major 4x4 float32 matrix, as the reference's
    TAA computes its inverse view (src/renderer.cpp:86-206)."""
    m = np.ascontiguousarray(m, np.float32).reshape(16)
    out = np.zeros(16, np.float32)
    ok = lib().oc_mat4_inverse(m, out)
    return bool(ok), out


def ref_mat4_inverse(m: np.ndarray):
    """The reference's own mat4_inverse (cut from src/renderer.cpp at build
    time into oracle/_ref/libglslref.so): (ok, inverse)."""
    m = np.ascontiguousarray(m, np.float32).reshape(16)
    out = np.zeros(16, np.float32)
    ok = glsl().ref_mat4_inverse(m, out)
    return bool(ok), out


def quad_rect(projected16: np.ndarray, width: int, height: int, cam=None, jitter=(0.0, 0.0)):
    vp_w, vp_h, ysign = _vp(cam, width, height)
    rect = np.zeros(4, np.int32)
    ok = lib().oc_quad_rect(np.ascontiguousarray(projected16, np.float32), float(jitter[0]), float(jitter[1]),
                            vp_w, vp_h, ysign, width, height, rect)
    return bool(ok), rect


def _vp(cam, width, height):
    if cam is None:
        return float(width), float(height), 1.0
    cam = np.asarray(cam, np.float32)
    return float(cam[32]), float(cam[33]), float(cam[37])


def to_f16(img: np.ndarray) -> np.ndarray:
    """Round an FP32 image to RGBA16F (round-to-nearest-even), once."""
    return img.astype(np.float16)


# --------------------------------------------------------------------------
# the reference's shader stages on the CPU (libglslref.so), same calls and
# outputs as the oracle helpers above
# --------------------------------------------------------------------------
def glsl_cull(rows: np.ndarray, cam: np.ndarray, sh_degree: int = 3, sh_lod_distance: float = 0.0,
              collect_stats: bool = True, deltas=None, scales=None, state_a: int = 0, state_b: int = 0,
              weight: float = 0.0, halves=None, layer_weights=None):
    """cull_reset_cs + cull_cs; deltas: (states, N, 48) int8 with 48 scales, or
    halves: (layers, N, 48) uint16 half bits with (layers, 3) weights."""
    rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 64)
    n = rows.shape[0]
    ids = np.empty(n, np.uint32)
    keys = np.empty(n, np.uint32)
    proj = np.empty((n, 16), np.float32)
    vc = np.zeros(1, np.uint32)
    diag = np.zeros(8, np.uint32)
    cam = np.ascontiguousarray(cam, np.float32)
    words, states, layers, sc, lw = None, 0, 0, None, None
    if halves is not None:
        words = np.ascontiguousarray(halves, np.uint16).reshape(-1)
        if words.size % 2:
            words = np.concatenate([words, np.zeros(1, np.uint16)])
        words = words.view(np.uint32)
        lw = np.ascontiguousarray(layer_weights, np.float32).reshape(-1)
        layers = int(np.asarray(halves).shape[0])
    elif deltas is not None:
        d = np.ascontiguousarray(deltas, np.int8).reshape(-1)
        pad = (-d.size) % 4
        if pad:
            d = np.concatenate([d, np.zeros(pad, np.int8)])
        words = d.view(np.uint32)
        states = int(np.asarray(deltas).shape[0])
        sc = np.ascontiguousarray(scales, np.float32).reshape(48)
    ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    glsl().glsl_cull(rows.reshape(-1), n, cam, int(sh_degree), float(sh_lod_distance), int(bool(collect_stats)),
                     ptr(words), states, int(state_a), int(state_b), float(weight), ptr(sc), layers, ptr(lw),
                     ids, keys, proj.reshape(-1), vc, diag)
    return ids, keys, proj, int(vc[0]), diag


def glsl_sort_pairs(keys: np.ndarray, ids: np.ndarray):
    """radix_hist_cs, radix_prefix_cs and radix_scatter_cs over four 8-bit passes."""
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    ko = np.empty_like(keys)
    io = np.empty_like(ids)
    glsl().glsl_sort_pairs(keys, ids, keys.size, ko, io)
    return ko, io


def glsl_composite_alpha(sorted_ids: np.ndarray, projected: np.ndarray, width: int, height: int,
                         cam: np.ndarray | None = None, bg: float = 0.0, jitter=(0.0, 0.0)):
    vp_w, vp_h, ysign = _vp(cam, width, height)
    out = np.empty((height, width, 4), np.float32)
    sorted_ids = np.ascontiguousarray(sorted_ids, dtype=np.uint32)
    frags = glsl().glsl_composite_alpha(sorted_ids, sorted_ids.size,
                                        np.ascontiguousarray(projected, np.float32).reshape(-1), width, height,
                                        vp_w, vp_h, ysign, float(bg), float(jitter[0]), float(jitter[1]),
                                        out.reshape(-1))
    return out, int(frags)


def glsl_stochastic_sample(ids: np.ndarray, projected: np.ndarray, width: int, height: int, frame_seed: float,
                           cam: np.ndarray | None = None, bg: float = 0.0, jitter=(0.0, 0.0), rgba8: bool = True):
    vp_w, vp_h, ysign = _vp(cam, width, height)
    out = np.empty((height, width, 4), np.float32)
    depth = np.empty((height, width), np.float32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    kept = glsl().glsl_stochastic_sample(ids, ids.size, np.ascontiguousarray(projected, np.float32).reshape(-1),
                                         width, height, vp_w, vp_h, ysign, float(bg), float(jitter[0]),
                                         float(jitter[1]), float(frame_seed), int(bool(rgba8)), out.reshape(-1),
                                         depth.reshape(-1))
    return out, depth, int(kept)


def glsl_gps_frame(ids: np.ndarray, projected: np.ndarray, width: int, height: int, supersample: int,
                   max_work_items: int, frame_seed: float, clip_z_01: float = 0.0, linear_color: bool = False,
                   bg: float = 0.0):
    out = np.empty((height, width, 4), np.float32)
    depth = np.empty((height, width), np.float32)
    stats = np.zeros(2, np.uint32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    glsl().glsl_gps_frame(ids, ids.size, np.ascontiguousarray(projected, np.float32).reshape(-1), width, height,
                          int(supersample), int(max_work_items), float(clip_z_01), int(bool(linear_color)),
                          float(frame_seed), float(bg), out.reshape(-1), depth.reshape(-1), stats)
    return out, depth, int(stats[0]), int(stats[1])


def glsl_accum(sample: np.ndarray, history: np.ndarray, n: float):
    """accum_fs over an (H, W, 4) frame."""
    sample = np.ascontiguousarray(sample, np.float32)
    history = np.ascontiguousarray(history, np.float32)
    h, w = sample.shape[:2]
    out = np.empty_like(sample)
    glsl().glsl_accum(sample.reshape(-1), history.reshape(-1), float(n), w, h, out.reshape(-1))
    return out


def glsl_taa(cur_color, cur_depth, hist_color, hist_xyz, inv_view, prev_view, viewport_ortho, focal_clip,
             prev_focal_clip, proj_z, history_valid: float, view_changed: float):
    h, w = cur_depth.shape
    oc = np.empty((h, w, 4), np.float32)
    ox = np.empty((h, w, 4), np.float32)
    f = lambda a: np.ascontiguousarray(a, np.float32).reshape(-1)  # noqa: E731
    glsl().glsl_taa(f(cur_color), f(cur_depth), f(hist_color), f(hist_xyz), w, h, f(inv_view), f(prev_view),
                    f(viewport_ortho), f(focal_clip), f(prev_focal_clip), f(proj_z), float(history_valid),
                    float(view_changed), oc.reshape(-1), ox.reshape(-1))
    return oc, ox


def glsl_display(img_half: np.ndarray, lut, log2_min: float, log2_max: float, exposure_ev: float) -> np.ndarray:
    """blit_fs / layers_display_fs over an (H, W, 4) float16 frame, as display()."""
    img = np.ascontiguousarray(img_half, np.float16)
    h, w = img.shape[:2]
    out = np.empty((h, w, 4), np.float32)
    if lut is None:
        lp, n = None, 0
    else:
        lut = np.ascontiguousarray(lut, np.uint16)
        lp, n = lut.ctypes.data, lut.shape[0]
    glsl().glsl_display(img.view(np.uint16).reshape(-1), w, h, lp, n, float(log2_min), float(log2_max),
                        float(exposure_ev), out.reshape(-1))
    return out
