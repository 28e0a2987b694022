"""Seeded mutation fuzz of the host loaders (PLY, SOG, gsanim, WebP, raw
archive bytes) against a build of them given as the first argument; run by
tests/test_loader_sanitizers.py with AddressSanitizer and UBSan preloaded.
Usage: loader_fuzz.py LIB SEED TRIALS.  Prints the accepted counts."""
import ctypes as C
import sys
import tempfile
import zipfile
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
from tests import gsanim_fixture as F
from tests import sog_fixture as S
from tests.test_ply_loader import ply

lib = C.CDLL(sys.argv[1])
lib.gs_load_ply.restype = C.c_int64
lib.gs_load_ply.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64]
lib.gs_load_sog.restype = C.c_int64
lib.gs_load_sog.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64]
lib.gs_load_scene.restype = C.c_int64
lib.gs_load_scene.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64]
lib.gs_gsanim_load.restype = C.c_int
lib.gs_gsanim_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
lib.gs_gsanim_free.argtypes = [C.c_void_p]
lib.gs_webp_decode_rgba.restype = C.c_int
lib.gs_webp_decode_rgba.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                                    C.c_uint64]

_tmpdir = tempfile.TemporaryDirectory()
tmp = Path(_tmpdir.name)
rng = np.random.default_rng(int(sys.argv[2]))
trials = int(sys.argv[3])


def mutate(b: bytes) -> bytes:
    blob = bytearray(b)
    for _ in range(int(rng.integers(1, 6))):
        if not blob:
            break
        pos = int(rng.integers(0, len(blob)))
        k = int(rng.integers(0, 5))
        if k == 0:
            blob[pos] ^= 1 << int(rng.integers(0, 8))
        elif k == 1:
            blob[pos] = int(rng.integers(0, 256))
        elif k == 2:
            del blob[pos]
        elif k == 3:
            blob.insert(pos, int(rng.integers(0, 256)))
        else:
            del blob[pos:]
    return bytes(blob)


def load_rows(fn, path):
    n = fn(str(path).encode(), None, 0)
    if n > 0 and n < 1 << 20:
        rows = np.zeros((n, 64), np.float32)
        fn(str(path).encode(), rows.ctypes.data, n)
    return n


plys = [ply(n=5, seed=s) for s in range(3)]
sog_assets = [S.sog_asset(25, seed=9, bands=1, shn_count=20), S.sog_asset(17, seed=11),
              S.sog_asset(30, seed=12, bands=3, shn_count=70)]
sog_entries = [S.entries(m, i) for m, i in sog_assets]
gsa = []
m, base, scales, deltas = F.v01_asset(n=5, states=3, seed=1)
gsa.append(F.entries_v01(m, base, scales, deltas))
m, base, halves, lut = F.v03_asset(n=4, seed=2)
gsa.append(F.entries_v03(m, base, halves, lut))

counts = dict(ply=0, sog=0, gsanim=0, webp=0, zipraw=0)
for t in range(trials):
    kind = t % 5
    if kind == 0:
        p = tmp / 'a.ply'
        p.write_bytes(mutate(plys[t % 3]))
        counts['ply'] += load_rows(lib.gs_load_ply, p) > 0
    elif kind == 1:
        e = sog_entries[t % 3]
        name = list(e)[int(rng.integers(0, len(e)))]
        p = S.pack(tmp / 'a.sog', {**e, name: mutate(e[name])},
                   zipfile.ZIP_DEFLATED if t % 2 else zipfile.ZIP_STORED)
        counts['sog'] += load_rows(lib.gs_load_sog, p) > 0
    elif kind == 2:
        e = gsa[t % 2]
        name = list(e)[int(rng.integers(0, len(e)))]
        p = F.pack(tmp / 'a.gsanim', {**e, name: mutate(e[name])},
                   zipfile.ZIP_DEFLATED if t % 2 else zipfile.ZIP_STORED)
        h = C.c_void_p()
        if lib.gs_gsanim_load(str(p).encode(), C.byref(h)) == 0:
            counts['gsanim'] += 1
            lib.gs_gsanim_free(h)
        load_rows(lib.gs_load_scene, p)
    elif kind == 3:
        e = sog_entries[t % 3]
        webps = [k for k in e if k.endswith('.webp')]
        data = mutate(e[webps[int(rng.integers(0, len(webps)))]])
        w, h = C.c_int(), C.c_int()
        st = lib.gs_webp_decode_rgba(data, len(data), C.byref(w), C.byref(h), None, 0)
        if st == 0 and w.value * h.value < 1 << 22:
            out = np.zeros(w.value * h.value * 4, np.uint8)
            lib.gs_webp_decode_rgba(data, len(data), C.byref(w), C.byref(h), out.ctypes.data, out.nbytes)
            counts['webp'] += 1
    else:
        # mutate the archive bytes themselves (central directory, local headers)
        e = gsa[t % 2] if t % 2 else sog_entries[t % 3]
        src = F.pack(tmp / 'z.zip', e, zipfile.ZIP_DEFLATED if (t // 2) % 2 else zipfile.ZIP_STORED)
        p = tmp / ('z.gsanim' if t % 2 else 'z.sog')
        p.write_bytes(mutate(src.read_bytes()))
        counts['zipraw'] += load_rows(lib.gs_load_scene, p) > 0
print('accepted', counts)
