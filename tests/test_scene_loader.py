"""gs_load_scene against the reference's scene dispatch compiled from its
sources (load_gaussian_scene, src/gaussian.cpp:15-40): the format by the
file name's extension, compared case-insensitively, for PLY, SOG and gsanim
files; any other name is refused.  Rows are compared bit for bit with the
reference's pack_gpu_gaussians output and with the per-format loaders.
CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import _lib as L
from gamesplat_b200 import renderer as R
from gamesplat_b200.gsanim import load_gsanim
from oracle import oracle as O
from tests import gsanim_fixture as F
from tests.test_ply_loader import ply

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference CPU build (oracle/_ref) not present")


def ours(path, capacity=None):
    lib = L.lib()
    n = lib.gs_load_scene(str(path).encode(), None, 0)
    if n < 0:
        return int(n)
    cap = n if capacity is None else capacity
    rows = np.full((max(cap, 1), 64), np.nan, np.float32)
    got = lib.gs_load_scene(str(path).encode(), rows.ctypes.data, cap)
    assert got == n
    return rows[:cap]


def reference(path):
    Rf = O.ref()
    n = Rf.ref_load_ply_rows(str(path).encode(), None, 0)
    if n == 0:
        return None
    rows = np.zeros((n, 64), np.float32)
    Rf.ref_load_ply_rows(str(path).encode(), rows.ctypes.data, n)
    return rows


def ply_bytes(seed=0, n=7):
    return ply(n=n, seed=seed)


def sog_bytes(tmp_path, seed=0, n=11):
    pytest.importorskip("PIL")
    from tests import sog_fixture as S
    meta, images = S.sog_asset(n, seed, bands=1)
    return S.pack(tmp_path / f"src{seed}.zip", S.entries(meta, images)).read_bytes()


def gsanim_bytes(tmp_path, seed=0):
    manifest, base, scales, deltas = F.v01_asset(n=6, states=3, seed=seed)
    return F.pack(tmp_path / f"src{seed}.zip", F.entries_v01(manifest, base, scales, deltas)).read_bytes()


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("fmt,suffixes", [
    ("ply", [".ply", ".PLY", ".Ply"]),
    ("sog", [".sog", ".SOG", ".sOg"]),
    ("gsanim", [".gsanim", ".GSANIM", ".GsAnim"]),
])
def test_dispatch_by_extension_matches_reference(tmp_path, fmt, suffixes):
    data = {"ply": lambda: ply_bytes(3), "sog": lambda: sog_bytes(tmp_path, 3),
            "gsanim": lambda: gsanim_bytes(tmp_path, 3)}[fmt]()
    direct = {"ply": R.load_ply, "sog": R.load_sog, "gsanim": lambda p: load_gsanim(p).rows}[fmt]
    for k, suffix in enumerate(suffixes):
        path = tmp_path / f"scene{k}{suffix}"
        path.write_bytes(data)
        got, want = ours(path), reference(path)
        assert want is not None and not isinstance(got, int), (fmt, suffix, got)
        assert same(got, want), (fmt, suffix)
        assert same(np.asarray(direct(path), np.float32), got), (fmt, suffix)
        assert same(R.load_scene(path), want)


@pytest.mark.parametrize("name", ["scene.splat", "scene.txt", "scene", "ply", "scene.ply.bak", "scene.plyx",
                                  "scene.so", "scene.gsani", ".ply_", "scene.sog "])
def test_other_names_are_refused(tmp_path, name):
    path = tmp_path / name
    path.write_bytes(ply_bytes(1))
    assert reference(path) is None
    assert ours(path) == L.GS_ERR_FORMAT
    with pytest.raises(L.GsError):
        R.load_scene(path)


def test_bare_extension_names(tmp_path):
    """A name that is only the extension still ends with it."""
    (tmp_path / "d").mkdir()
    path = tmp_path / "d" / ".ply"
    path.write_bytes(ply_bytes(2))
    want = reference(path)
    assert want is not None and same(ours(path), want)


def test_content_of_another_format(tmp_path):
    """The extension alone picks the loader.  A stored (uncompressed) gsanim
    archive named .ply loads as its base PLY in both, since the PLY header
    scan takes no magic from the first line and the stored base.ply's header
    and body lie in the archive as they are; the other mixes are refused."""
    cases = {"a.sog": ply_bytes(4), "b.ply": gsanim_bytes(tmp_path, 4), "c.gsanim": ply_bytes(5),
             "d.ply": sog_bytes(tmp_path, 5)}
    loaded = set()
    for name, data in cases.items():
        path = tmp_path / name
        path.write_bytes(data)
        want, got = reference(path), ours(path)
        if want is None:
            assert isinstance(got, int) and got < 0, name
        else:
            assert not isinstance(got, int) and same(got, want), name
            loaded.add(name)
    assert loaded == {"b.ply"}


def test_missing_file(tmp_path):
    for name in ("none.ply", "none.sog", "none.gsanim"):
        assert reference(tmp_path / name) is None
        got = ours(tmp_path / name)
        assert isinstance(got, int) and got < 0


def test_capacity_below_count_fills_a_prefix(tmp_path):
    for name, data in (("p.ply", ply_bytes(6, n=9)), ("s.sog", sog_bytes(tmp_path, 6)),
                       ("g.gsanim", gsanim_bytes(tmp_path, 6))):
        path = tmp_path / name
        path.write_bytes(data)
        want = reference(path)
        for cap in (0, 1, len(want) - 1):
            got = ours(path, capacity=cap)
            assert same(got, want[:cap]), (name, cap)


def test_null_path():
    assert L.lib().gs_load_scene(None, None, 0) == L.GS_ERR_BAD_ARG
