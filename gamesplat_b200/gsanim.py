"""gsanim assets (the reference's GSAnim, src/gsanim.h) through the C ABI.

``load_gsanim(path)`` mirrors ``gaussian_load_gsanim``
(src/gaussian_loader_gsanim.cpp:386-495): it raises ``GsError`` with
``GS_ERR_FORMAT`` for every file the reference loader rejects.  The result
carries the arrays the renderer uploads (``rows`` for ``upload_gaussians``,
``deltas`` / ``scales`` for ``upload_anim``, ``display_lut`` for
``set_display_lut``) and the playback functions ``sample``
(``gsanim_sample``) and ``layer_weights`` (``gsanim_layer_weights``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class GSAnim:
    version: int                   # 1, 2, 3 for manifest "0.1", "0.2", "0.3"
    gaussian_count: int
    state_count: int               # incl. the base state 0 (0.1 / 0.2); 0 for 0.3
    duration: float
    linear: bool                   # manifest interpolation (0.1 / 0.2)
    key_count: int
    rows: np.ndarray               # gaussian_count x 64 float32 GpuGaussian rows
    deltas: np.ndarray             # (state_count - 1) x gaussian_count x 48 int8
    scales: np.ndarray             # 48 float32
    layer_names: list[bytes] = field(default_factory=list)
    layer_data: np.ndarray | None = None     # layers x gaussian_count x 48 uint16 (half bits)
    display_lut: np.ndarray | None = None    # lut_size^3 x 3 uint16, red fastest
    lut_size: int = 0
    log2_min: float = 0.0
    log2_max: float = 0.0
    _handle: int | None = None

    def sample(self, seconds: float) -> tuple[int, int, float]:
        """(state_a, state_b, weight) at `seconds` (gsanim_sample)."""
        a, b, w = C.c_int32(), C.c_int32(), C.c_float()
        L.check(L.lib().gs_gsanim_sample(self._handle, float(seconds), C.byref(a), C.byref(b), C.byref(w)),
                "gs_gsanim_sample")
        return a.value, b.value, w.value

    def layer_weights(self, seconds: float) -> np.ndarray:
        """layers x 3 float32 weights at `seconds`; empty for 0.1 / 0.2 or non-finite times."""
        out = np.zeros((max(len(self.layer_names), 1), 3), np.float32)
        n = L.lib().gs_gsanim_layer_weights(self._handle, float(seconds), out.ctypes.data)
        if n < 0:
            raise L.GsError(int(n), "gs_gsanim_layer_weights")
        return out[:n]

    def close(self) -> None:
        if self._handle:
            L.lib().gs_gsanim_free(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass


def load_gsanim(path) -> GSAnim:
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.gs_gsanim_load(str(path).encode(), C.byref(h)), f"gs_gsanim_load({path})")
    info = L.GsGsanimInfo()
    L.check(lib.gs_gsanim_get_info(h, C.byref(info)), "gs_gsanim_get_info")
    n = info.gaussian_count
    rows = np.empty((n, 64), np.float32)
    L.check(lib.gs_gsanim_rows(h, rows.ctypes.data), "gs_gsanim_rows")
    states = max(int(info.state_count) - 1, 0)
    deltas = np.empty((states, n, 48), np.int8)
    scales = np.empty(48, np.float32)
    L.check(lib.gs_gsanim_deltas(h, deltas.ctypes.data if deltas.size else None, scales.ctypes.data),
            "gs_gsanim_deltas")
    names = []
    for i in range(info.layer_count):
        length = lib.gs_gsanim_layer_name(h, i, None, 0)
        buf = C.create_string_buffer(max(int(length), 1))
        lib.gs_gsanim_layer_name(h, i, buf, length)
        names.append(buf.raw[:length])
    layer_data = display_lut = None
    if info.version == 3:
        layer_data = np.empty((info.layer_count, n, 48), np.uint16)
        L.check(lib.gs_gsanim_layer_data(h, layer_data.ctypes.data), "gs_gsanim_layer_data")
        display_lut = np.empty((info.lut_size ** 3, 3), np.uint16)
        L.check(lib.gs_gsanim_display_lut(h, display_lut.ctypes.data), "gs_gsanim_display_lut")
    return GSAnim(version=info.version, gaussian_count=n, state_count=info.state_count,
                  duration=info.duration_seconds, linear=bool(info.linear), key_count=info.key_count, rows=rows,
                  deltas=deltas, scales=scales, layer_names=names, layer_data=layer_data, display_lut=display_lut,
                  lut_size=info.lut_size, log2_min=info.log2_min, log2_max=info.log2_max, _handle=h.value)
