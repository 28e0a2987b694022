"""Python face of the stochastic-splat denoiser (gs_denoiser_* in
include/gs_api.h): a 5-layer, 32-channel convolutional network with a U-Net
skip whose convolutions run on the tensor cores, trained with hand-written
forward, backward and Adam kernels.  Tensors are passed as device pointers
(for example torch tensors' data_ptr()); parameters come and go as numpy
float32 arrays."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

IN_CHANNELS = 16
OUT_CHANNELS = 16
# conv1 .. conv5: (cin, cout)
LAYERS = ((16, 32), (32, 32), (32, 32), (32, 32), (32, 16))


def param_count() -> int:
    return int(L.lib().gs_denoiser_param_count())


def split_params(flat: np.ndarray):
    """[(W[3,3,cin,cout], b[cout])] per layer from the flat parameter vector."""
    out, o = [], 0
    for cin, cout in LAYERS:
        w = flat[o:o + 9 * cin * cout].reshape(3, 3, cin, cout)
        o += 9 * cin * cout
        b = flat[o:o + cout]
        o += cout
        out.append((w, b))
    return out


class Denoiser:
    def __init__(self, device: int = 0, stream: int | None = None):
        self._d = C.c_void_p()
        L.check(L.lib().gs_denoiser_create(C.byref(self._d), int(device), C.c_void_p(stream or 0)),
                "gs_denoiser_create")

    def close(self):
        if self._d:
            L.lib().gs_denoiser_destroy(self._d)
            self._d = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._d

    def init_params(self, seed: int) -> None:
        L.check(L.lib().gs_denoiser_init_params(self._d, int(seed)), "gs_denoiser_init_params")

    def params(self) -> np.ndarray:
        out = np.empty(param_count(), np.float32)
        L.check(L.lib().gs_denoiser_get_params(self._d, out.ctypes.data, out.size), "gs_denoiser_get_params")
        return out

    def set_params(self, flat: np.ndarray) -> None:
        flat = np.ascontiguousarray(flat, np.float32)
        L.check(L.lib().gs_denoiser_set_params(self._d, flat.ctypes.data, flat.size), "gs_denoiser_set_params")

    def grads(self) -> np.ndarray:
        out = np.empty(param_count(), np.float32)
        L.check(L.lib().gs_denoiser_get_grads(self._d, out.ctypes.data, out.size), "gs_denoiser_get_grads")
        return out

    def forward(self, x_ptr: int, n: int, h: int, w: int, out_ptr: int) -> None:
        L.check(L.lib().gs_denoiser_forward(self._d, C.c_void_p(x_ptr), n, h, w, C.c_void_p(out_ptr)),
                "gs_denoiser_forward")

    def backward(self, x_ptr: int, dout_ptr: int, n: int, h: int, w: int) -> None:
        L.check(L.lib().gs_denoiser_backward(self._d, C.c_void_p(x_ptr), C.c_void_p(dout_ptr), n, h, w),
                "gs_denoiser_backward")

    def loss(self, x_ptr: int, out_ptr: int, target_ptr: int, n: int, h: int, w: int, dout_ptr: int,
             ssim_weight: float = 0.2, err_weight: float = 0.01) -> np.ndarray:
        parts = np.zeros(4, np.float32)
        L.check(L.lib().gs_denoiser_loss(self._d, C.c_void_p(x_ptr), C.c_void_p(out_ptr), C.c_void_p(target_ptr),
                                         n, h, w, float(ssim_weight), float(err_weight), C.c_void_p(dout_ptr),
                                         parts.ctypes.data), "gs_denoiser_loss")
        return parts

    def adam(self, lr: float) -> None:
        L.check(L.lib().gs_denoiser_adam(self._d, float(lr)), "gs_denoiser_adam")

    def train_step(self, x_ptr: int, target_ptr: int, n: int, h: int, w: int, lr: float,
                   want_loss: bool = True) -> np.ndarray | None:
        parts = np.zeros(4, np.float32) if want_loss else None
        L.check(L.lib().gs_denoiser_train_step(self._d, C.c_void_p(x_ptr), C.c_void_p(target_ptr), n, h, w,
                                               float(lr), parts.ctypes.data if want_loss else None),
                "gs_denoiser_train_step")
        return parts

    def status(self) -> None:
        L.check(L.lib().gs_denoiser_status(self._d), "gs_denoiser_status")
