"""GPU test of gs_sort_pairs_noalloc, the radix-sort entry point that
allocates nothing.

It serves callers that cannot allocate device memory through the library (a
render loop where cudaMalloc would synchronise the device mid-frame, or an
engine whose memory manager owns every device allocation); its scratch is a
fixed array in the library's device memory.  The test calls it through the C
ABI twice in a row and checks each result against gs_sort_pairs (the
allocating entry point, given scratch from torch): an integer sort, so the
tolerance is exact equality.  The file name makes pytest collect it last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gamesplat_b200 import _lib as L
from gamesplat_b200 import renderer as RR

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _device(a: np.ndarray):
    import torch

    return torch.from_numpy(a.view(np.int32)).cuda()


def test_noalloc_sort_matches_allocating_sort_on_two_calls():
    import torch

    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(MAX_PAIRS, 0, 32, 11), (300_001, 3, 29, 12)]
    for n, b0, b1, seed in cases:
        rng = np.random.default_rng(seed)
        keys = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
        keys[::7] = keys[0]   # plenty of equal keys: stability matters
        vals = np.arange(n, dtype=np.uint32)
        dk, dv = _device(keys), _device(vals)
        ko_a, vo_a = torch.empty_like(dk), torch.empty_like(dv)
        ko_b, vo_b = torch.empty_like(dk), torch.empty_like(dv)
        st = lib.gs_sort_pairs_noalloc(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()),
                                       C.c_void_p(ko_a.data_ptr()), C.c_void_p(vo_a.data_ptr()), n, b0, b1,
                                       C.c_void_p(stream))
        assert st == L.GS_OK, L.status_str(st)
        nbytes = RR.sort_pairs_scratch_bytes(n)
        scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        RR.sort_pairs(dk.data_ptr(), dv.data_ptr(), ko_b.data_ptr(), vo_b.data_ptr(), n, scratch.data_ptr(),
                      nbytes, b0, b1, stream)
        torch.cuda.synchronize()
        assert torch.equal(ko_a, ko_b) and torch.equal(vo_a, vo_b)
        sub = (keys >> np.uint32(b0)) & np.uint32((1 << (b1 - b0)) - 1) if b1 - b0 < 32 else keys
        order = np.argsort(sub, kind="stable")
        assert np.array_equal(vo_a.cpu().numpy().view(np.uint32), vals[order])


def test_noalloc_sort_rejects_more_than_its_limit():
    st = L.lib().gs_sort_pairs_noalloc(None, None, None, None, MAX_PAIRS + 1, 0, 32, None)
    assert st == L.GS_ERR_TOO_LARGE
