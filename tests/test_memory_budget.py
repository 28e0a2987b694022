"""gs_scene_device_bytes, the device-memory figure the uploads check against
the budget (the counterpart of renderer_scene_buffer_bytes,
src/renderer.cpp:705-709), restated here from the buffer layout: per
Gaussian the 256-byte row, 16-byte head, 64-byte projected record, 16 bytes
of sort pairs, 64-byte raster record, 16 bytes of binning state and the
48-byte GPS prepared record; look-back words per 2048-row cull tile, per
4096-pair sort tile (256 words of 8 bytes for each of 4 passes) and per
1024-splat binning tile; tile entries at their initial capacity
max(8N, 2^20) (16 bytes each, a 4-byte owner per 1024-entry chunk, sort
look-back words); 8 bytes per GPS work item.  Host only (no GPU)."""
from __future__ import annotations

import pytest

from gamesplat_b200 import _lib as L


def cdiv(a, b):
    return (a + b - 1) // b


def expected(n, work):
    work = max(work, 1)
    cap = min(max(8 * n, 1 << 20), (1 << 30) - 1)
    sort_words = lambda m: max(1, cdiv(m, 4096)) * 256   # noqa: E731
    return (8 * work + n * 480 + cdiv(n, 2048) * 8 + sort_words(n) * 4 * 8 + cdiv(n, 1024) * 8 +
            cap * 16 + (cap // 1024 + 2) * 4 + sort_words(cap) * 4 * 8)


@pytest.mark.parametrize("n", [1, 1000, 131_071, 131_072, 131_073, 3_000_000, (1 << 30) - 1])
@pytest.mark.parametrize("work", [0, 1, 16 << 20, (250 << 20)])
def test_scene_device_bytes(n, work):
    assert L.lib().gs_scene_device_bytes(n, work) == expected(n, work)


def test_out_of_range_counts():
    assert L.lib().gs_scene_device_bytes(0, 1 << 20) == 0
    assert L.lib().gs_scene_device_bytes(1 << 30, 1 << 20) == 0
    assert L.lib().gs_scene_device_bytes((1 << 64) - 1, 1 << 20) == 0


def test_benchmark_scene_figure():
    """3M Gaussians with the default 16 Mi GPS work items: ~2.0 GB (1.44 GB
    per-Gaussian buffers, 0.38 GB of tile entries, 0.13 GB of GPS work)."""
    b = L.lib().gs_scene_device_bytes(3_000_000, 16 << 20)
    assert 1.95e9 < b < 2.05e9


def test_knob_field_layout():
    assert L.GsKnobs.gpu_budget_mb.offset == 48 and L.GsKnobs.reserved.offset == 52
