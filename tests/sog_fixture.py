"""Writers of small SOG (version 2) archives for the loader tests.

A SOG archive is a ZIP of ``meta.json`` and lossless WebP images, one RGBA8
pixel per Gaussian in row-major order (src/gaussian_loader_sog.cpp:126-551):

* ``means_l`` / ``means_u``: low / high bytes of a 16-bit value per axis (RGB)
  that lerps between ``means.mins`` and ``means.maxs`` into log space;
* ``scales``: per-axis labels (RGB) into ``scales.codebook`` (log scales);
* ``quats``: three stored quaternion components (RGB) and 252 + the index of
  the omitted one (A);
* ``sh0``: per-channel labels (RGB) into ``sh0.codebook`` and opacity (A);
* optional ``shN``: a label image (R + 256 G per Gaussian) into a centroid
  image of 64 centroids per row, ``coeffs`` pixels per centroid (RGB labels
  into ``shN.codebook``), coeffs = 3 / 8 / 15 for 1 / 2 / 3 bands.
"""
from __future__ import annotations

import io
import json
import warnings
import zipfile
from pathlib import Path

import numpy as np
from PIL import Image


def webp(pixels: np.ndarray, **kw) -> bytes:
    """Lossless WebP of an H x W x 4 uint8 image; exact keeps RGB under alpha 0."""
    b = io.BytesIO()
    Image.fromarray(np.ascontiguousarray(pixels, np.uint8), "RGBA").save(b, "WEBP", lossless=True, exact=True, **kw)
    return b.getvalue()


def grid(n: int) -> tuple[int, int]:
    w = max(1, int(np.ceil(np.sqrt(n))))
    return w, (n + w - 1) // w


def sog_asset(n: int, seed: int, bands: int = 0, shn_count: int = 37):
    """(meta dict, {file name: H x W x 4 uint8 image}) of a seeded asset."""
    rng = np.random.default_rng(seed)
    w, h = grid(n)

    def img():
        return rng.integers(0, 256, (h, w, 4)).astype(np.uint8)

    means_l, means_u, scales, quats, sh0 = img(), img(), img(), img(), img()
    for im in (means_l, means_u, scales):
        im[..., 3] = 255
    quats[..., 3] = 252 + rng.integers(0, 4, (h, w)).astype(np.uint8)
    images = {"means_l.webp": means_l, "means_u.webp": means_u, "scales.webp": scales, "quats.webp": quats,
              "sh0.webp": sh0}
    f32 = lambda a: [float(v) for v in np.asarray(a, np.float32)]   # noqa: E731
    meta = {
        "version": 2, "count": n, "antialias": False,
        "means": {"mins": f32(rng.uniform(-3, -0.5, 3)), "maxs": f32(rng.uniform(0.5, 3, 3)),
                  "files": ["means_l.webp", "means_u.webp"]},
        "scales": {"codebook": f32(np.sort(rng.uniform(-8, 0, 256))), "files": ["scales.webp"]},
        "quats": {"files": ["quats.webp"]},
        "sh0": {"codebook": f32(np.sort(rng.uniform(-2, 2, 256))), "files": ["sh0.webp"]},
    }
    if bands:
        coeffs = {1: 3, 2: 8, 3: 15}[bands]
        centroids = rng.integers(0, 256, ((shn_count + 63) // 64, 64 * coeffs, 4)).astype(np.uint8)
        centroids[..., 3] = 255
        labels = np.zeros((h, w, 4), np.uint8)
        lab = rng.integers(0, shn_count, (h, w))
        labels[..., 0] = lab & 255
        labels[..., 1] = lab >> 8
        labels[..., 3] = 255
        images["shN_centroids.webp"] = centroids
        images["shN_labels.webp"] = labels
        meta["shN"] = {"count": shn_count, "bands": bands, "codebook": f32(np.sort(rng.uniform(-1, 1, 256))),
                       "files": ["shN_centroids.webp", "shN_labels.webp"]}
    return meta, images


def entries(meta: dict, images: dict) -> dict:
    out = {"meta.json": json.dumps(meta).encode()}
    out.update({name: webp(px) for name, px in images.items()})
    return out


def pack(path: Path, items, compression=zipfile.ZIP_STORED) -> Path:
    """Write items (a dict or a list of (name, bytes), duplicates allowed) as a ZIP archive."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)   # duplicate names on purpose
        with zipfile.ZipFile(path, "w", compression=compression) as z:
            for name, value in (items.items() if isinstance(items, dict) else items):
                z.writestr(name, value)
    return path
