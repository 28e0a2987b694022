"""Writers of small gsanim archives for the loader tests.

A gsanim asset is a ZIP archive of exactly four entries
(src/gaussian_loader_gsanim.cpp:386-488):

* 0.1 / 0.2: ``manifest.json``, ``base.ply``, ``scales.bin`` (48 little-endian
  floats) and ``deltas.bin`` (int8, state-major, original row order, 48
  coefficients per row: the three DC values, then f_rest channel-major);
* 0.3: ``manifest.json``, ``base.ply``, ``layers.bin`` (IEEE half bits,
  layer-major, 48 per row) and ``display_lut.bin`` (RGB uint16 UNORM,
  red-fastest, size^3 texels).

``base.ply`` is a binary little-endian PLY with exactly the 62 float
properties x y z nx ny nz f_dc_0..2 f_rest_0..44 opacity scale_0..2 rot_0..3
(comment lines allowed between header lines).
"""
from __future__ import annotations

import json
import warnings
import zipfile
from pathlib import Path

import numpy as np

PLY_NAMES = (["x", "y", "z", "nx", "ny", "nz"] + [f"f_dc_{i}" for i in range(3)] +
             [f"f_rest_{i}" for i in range(45)] + ["opacity"] + [f"scale_{i}" for i in range(3)] +
             [f"rot_{i}" for i in range(4)])


def write_ply(base: np.ndarray, comments: tuple[str, ...] = ()) -> bytes:
    """base: (N, 62) float32 in PLY_NAMES order."""
    base = np.ascontiguousarray(base, dtype="<f4")
    lines = ["ply", "format binary_little_endian 1.0", *[f"comment {c}" for c in comments],
             f"element vertex {base.shape[0]}", *[f"property float {n}" for n in PLY_NAMES], "end_header"]
    return ("\n".join(lines) + "\n").encode() + base.tobytes()


def base_rows(n: int, seed: int, appearance: bool = True) -> np.ndarray:
    """Seeded (n, 62) base attributes; appearance=False zeroes f_dc/f_rest (0.3 assets)."""
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 62), np.float32)
    b[:, 0:3] = rng.uniform(-3, 3, (n, 3))
    b[:, 3:6] = rng.normal(0, 1, (n, 3))
    if appearance:
        b[:, 6:54] = rng.normal(0, 0.4, (n, 48))
    b[:, 54] = rng.normal(0.5, 2, n)
    b[:, 55:58] = rng.normal(-3.5, 0.8, (n, 3))
    b[:, 58:62] = rng.normal(0, 1, (n, 4))
    return b


def manifest_v01(n: int, states: int, keys, duration=8.0, interpolation="step", version="0.1") -> dict:
    return dict(format="gsanim", version=version, sh_degree=3, gaussian_count=n, state_count=states,
                coordinate_system="blender_world_z_up_meters", color_encoding="display_referred_agx_baked",
                duration_seconds=duration, interpolation=interpolation, keys=list(keys))


def manifest_v03(n: int, layers, lut_size: int, log2_min=-2.0, log2_max=3.0, duration=2.0) -> dict:
    return dict(format="gsanim", version="0.3", sh_degree=3, gaussian_count=n,
                coordinate_system="blender_world_z_up_meters", color_encoding="scene_linear_rec709",
                duration_seconds=duration, layers=list(layers),
                display_transform=dict(type="lut3d_log2", encoding="uint16_unorm_rgb", layout="r_fastest",
                                       size=lut_size, log2_min=log2_min, log2_max=log2_max))


def entries_v01(manifest: dict, base: np.ndarray, scales: np.ndarray, deltas: np.ndarray) -> dict:
    return {"manifest.json": json.dumps(manifest).encode(), "base.ply": write_ply(base),
            "scales.bin": np.asarray(scales, "<f4").tobytes(), "deltas.bin": np.asarray(deltas, "i1").tobytes()}


def entries_v03(manifest: dict, base: np.ndarray, layer_halves: np.ndarray, lut: np.ndarray) -> dict:
    return {"manifest.json": json.dumps(manifest).encode(), "base.ply": write_ply(base),
            "layers.bin": np.asarray(layer_halves, "<u2").tobytes(),
            "display_lut.bin": np.asarray(lut, "<u2").tobytes()}


def pack(path: Path, entries, compression=zipfile.ZIP_STORED) -> Path:
    """Write entries (a dict or a list of (name, bytes), duplicates allowed) as a ZIP archive."""
    items = entries.items() if isinstance(entries, dict) else entries
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)   # duplicate names on purpose
        with zipfile.ZipFile(path, "w", compression=compression) as z:
            for name, value in items:
                z.writestr(name, value)
    return path


def v01_asset(n=5, states=3, seed=0, version="0.1", interpolation="step"):
    """A small valid 0.1 / 0.2 asset: (manifest, base, scales, deltas)."""
    rng = np.random.default_rng(seed + 100)
    base = base_rows(n, seed)
    scales = np.linspace(0.001, 0.07, 48).astype(np.float32)
    deltas = rng.integers(-127, 128, (states - 1, n, 48)).astype(np.int8)
    keys = [dict(time_seconds=0, state=2 % states), dict(time_seconds=2, state=0),
            dict(time_seconds=5, state=1 % states)]
    if version == "0.2":
        for k, mode in zip(keys, ["linear", "step", "linear"]):
            k["interpolation"] = mode
    return manifest_v01(n, states, keys, interpolation=interpolation, version=version), base, scales, deltas


def v03_asset(n=4, seed=0, lut_size=3):
    """A small valid 0.3 asset: (manifest, base, layer halves, lut)."""
    rng = np.random.default_rng(seed + 200)
    base = base_rows(n, seed, appearance=False)
    layers = [dict(name="steady", keys=[dict(time_seconds=0, weight=[1, 1, 1], interpolation="step")]),
              dict(name="lamp", keys=[dict(time_seconds=0, weight=[0, 0, 0], interpolation="linear"),
                                      dict(time_seconds=1, weight=[2, 1.5, 1], interpolation="linear"),
                                      dict(time_seconds=1.5, weight=[0.5, 0.25, 0], interpolation="step")])]
    halves = rng.normal(0, 0.5, (len(layers), n, 48)).astype(np.float16).view(np.uint16)
    lut = rng.integers(0, 65536, (lut_size ** 3, 3)).astype(np.uint16)
    return manifest_v03(n, layers, lut_size), base, halves, lut
