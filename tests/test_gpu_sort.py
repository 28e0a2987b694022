"""GPU tests of the stage-level radix sort entry point gs_sort_pairs
(stable ascending, bit-exact against numpy's stable sort)."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import _lib as L
from gamesplat_b200 import renderer as RR

pytestmark = pytest.mark.gpu


def _run(keys: np.ndarray, vals: np.ndarray, begin=0, end=32):
    import torch

    n = keys.size
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    ok = torch.empty_like(dk)
    ov = torch.empty_like(dv)
    nbytes = RR.sort_pairs_scratch_bytes(n)
    scratch = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    RR.sort_pairs(dk.data_ptr(), dv.data_ptr(), ok.data_ptr(), ov.data_ptr(), n, scratch.data_ptr(), nbytes,
                  begin, end, stream)
    torch.cuda.synchronize()
    return ok.cpu().numpy().view(np.uint32), ov.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 5, 4095, 4096, 4097, 100_003, 3_000_000])
def test_sort_pairs_random(n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = _run(keys, vals)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])


def test_sort_pairs_many_ties_and_constant_digits():
    rng = np.random.default_rng(1)
    n = 250_000
    keys = (rng.integers(0, 50, size=n).astype(np.uint32) << 8) | np.uint32(0x3F000000)
    vals = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    k, v = _run(keys, vals)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])
    # every digit constant: all passes skipped, result copied
    same = np.full(10_000, 0xABCDEF01, np.uint32)
    k, v = _run(same, np.arange(10_000, dtype=np.uint32))
    assert np.array_equal(k, same) and np.array_equal(v, np.arange(10_000, dtype=np.uint32))


def test_sort_pairs_bit_range():
    rng = np.random.default_rng(2)
    n = 77_777
    keys = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = _run(keys, vals, 4, 17)
    sub = (keys >> 4) & ((1 << 13) - 1)
    order = np.argsort(sub, kind="stable")
    assert np.array_equal(v, vals[order]) and np.array_equal(k, keys[order])


def test_sort_pairs_rejects_bad_arguments():
    import torch

    buf = torch.empty(1024, dtype=torch.int32, device="cuda")
    scratch = torch.empty(RR.sort_pairs_scratch_bytes(256), dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    with pytest.raises(L.GsError):   # in place
        RR.sort_pairs(p, p + 1024, p, p + 2048, 256, scratch.data_ptr(), scratch.numel())
    with pytest.raises(L.GsError):   # scratch too small
        RR.sort_pairs(p, p + 1024, p + 2048, p + 3072, 256, scratch.data_ptr(), 16)
    with pytest.raises(L.GsError):   # bad bit range
        RR.sort_pairs(p, p + 1024, p + 2048, p + 3072, 256, scratch.data_ptr(), scratch.numel(), 8, 8)
    RR.sort_pairs(p, p + 1024, p + 2048, p + 3072, 0, 0, 0)   # n = 0 is a no-op
