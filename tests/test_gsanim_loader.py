"""gsanim archive loading (gs_gsanim_load and friends) against the reference
loader compiled from its own sources (gaussian_load_gsanim, gsanim_sample,
gsanim_layer_weights; src/gaussian_loader_gsanim.cpp:386-531).

Every case asserts the same verdict from both loaders, and for accepted
assets identical outputs: the GpuGaussian rows bit for bit, the deltas,
scales, half layers, display LUT and layer names byte for byte, and the
playback samples and layer weights at a set of times, bit for bit.  The
cases follow the reference's own conformance tests (tests/test_gsanim.py):
valid 0.1 / 0.2 / 0.3 assets, stored and deflated archives, every manifest
field missing, mistyped or out of range, broken payloads, archive damage and
JSON text edge cases.  CPU only.
"""
from __future__ import annotations

import copy
import json
import struct
import zipfile

import numpy as np
import pytest

from gamesplat_b200 import GsError, load_gsanim
from gamesplat_b200 import _lib as L
from oracle import oracle as O
from tests import gsanim_fixture as F

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference CPU build (oracle/_ref) not present")

TIMES = [0, .5, 1.0, 1.25, 1.49, 1.5, 1.75, 1.999, 2, 2.75, 4.999, 5, 6, 7.999, 8, -1, -8, 17, -0.25,
         1e300, -1e300, float("nan"), float("inf"), float("-inf")]


def ours(path, times=TIMES):
    try:
        a = load_gsanim(path)
    except GsError as e:
        assert e.status == L.GS_ERR_FORMAT, e
        return None
    try:
        return dict(version=a.version, gaussian_count=a.gaussian_count, state_count=a.state_count,
                    layer_count=len(a.layer_names), key_count=a.key_count, lut_size=a.lut_size, linear=a.linear,
                    log2_min=a.log2_min, log2_max=a.log2_max, duration=a.duration, rows=a.rows, deltas=a.deltas,
                    scales=a.scales,
                    layer_data=a.layer_data if a.layer_data is not None else np.zeros((0, a.gaussian_count, 48),
                                                                                        np.uint16),
                    display_lut=a.display_lut if a.display_lut is not None else np.zeros((0, 3), np.uint16),
                    layer_names=a.layer_names, samples=[a.sample(t) for t in times],
                    layer_weights=[a.layer_weights(t) for t in times])
    finally:
        a.close()


def bits(x):
    return np.ascontiguousarray(x).view(np.uint8)


def same(path, times=TIMES):
    """Both loaders agree on `path`; returns True if they accepted it."""
    r = O.ref_gsanim(path, times)
    o = ours(path, times)
    assert (r is None) == (o is None), f"reference {'rejects' if r is None else 'accepts'}, ours does not"
    if r is None:
        return False
    for k in ("version", "gaussian_count", "state_count", "layer_count", "key_count", "lut_size", "linear",
              "layer_names"):
        assert r[k] == o[k], k
    for k in ("log2_min", "log2_max"):
        assert np.float32(r[k]).tobytes() == np.float32(o[k]).tobytes(), k
    assert r["duration"] == o["duration"]
    for k in ("rows", "deltas", "scales", "layer_data", "display_lut"):
        assert r[k].shape == o[k].shape, k
        assert np.array_equal(bits(r[k]), bits(o[k])), k
    for t, rs, os_ in zip(times, r["samples"], o["samples"]):
        assert rs[:2] == os_[:2], t
        assert np.float32(rs[2]).tobytes() == np.float32(os_[2]).tobytes(), t
    for t, rw, ow in zip(times, r["layer_weights"], o["layer_weights"]):
        assert rw.shape == ow.shape and np.array_equal(bits(rw), bits(ow)), t
    return True


@pytest.fixture
def tmp_asset(tmp_path):
    return tmp_path / "fixture.gsanim"


def v01_entries(**kw):
    m, b, s, d = F.v01_asset(**kw)
    return m, F.entries_v01(m, b, s, d)


def v03_entries(**kw):
    m, b, h, lut = F.v03_asset(**kw)
    return m, F.entries_v03(m, b, h, lut)


def with_manifest(entries, m):
    return {**entries, "manifest.json": json.dumps(m).encode()}


# ---- valid assets --------------------------------------------------------------

@pytest.mark.parametrize("compression", [zipfile.ZIP_STORED, zipfile.ZIP_DEFLATED])
@pytest.mark.parametrize("interp", ["step", "linear"])
@pytest.mark.parametrize("n,states,seed", [(1, 2, 0), (5, 3, 1), (64, 9, 2)])
def test_v01_assets_match_reference(tmp_asset, compression, interp, n, states, seed):
    _, e = v01_entries(n=n, states=states, seed=seed, interpolation=interp)
    F.pack(tmp_asset, e, compression)
    assert same(tmp_asset)


@pytest.mark.parametrize("global_mode", ["step", "linear"])
def test_v02_per_key_modes_match_reference(tmp_asset, global_mode):
    _, e = v01_entries(n=6, states=3, seed=3, version="0.2", interpolation=global_mode)
    F.pack(tmp_asset, e)
    assert same(tmp_asset)
    a = load_gsanim(tmp_asset)
    assert a.sample(0.5) == (2, 0, 0.25)        # linear out of key 0 (t 0 -> 2)
    assert a.sample(2.75) == (0, 0, 0.0)        # step out of key 1
    assert a.sample(6)[:2] == (1, 2)            # linear out of the last key wraps to key 0
    a.close()


@pytest.mark.parametrize("compression", [zipfile.ZIP_STORED, zipfile.ZIP_DEFLATED])
@pytest.mark.parametrize("n,lut_size,seed", [(1, 2, 0), (4, 3, 1), (33, 5, 2)])
def test_v03_assets_match_reference(tmp_asset, compression, n, lut_size, seed):
    _, e = v03_entries(n=n, lut_size=lut_size, seed=seed)
    F.pack(tmp_asset, e, compression)
    assert same(tmp_asset)


def test_step_and_linear_samples(tmp_asset):
    """Keys (0 s: state 2, 2 s: state 0, 5 s: state 1) over an 8 s loop."""
    for mode in ("step", "linear"):
        _, e = v01_entries(n=2, states=3, seed=4, interpolation=mode)
        F.pack(tmp_asset, e, zipfile.ZIP_DEFLATED)
        assert same(tmp_asset)
        a = load_gsanim(tmp_asset)
        for t, state in [(0, 2), (2, 0), (5, 1), (8, 2), (-8, 2)]:
            assert a.sample(t)[0] == state and a.sample(t)[2] == 0
        if mode == "linear":
            assert a.sample(0.5) == (2, 0, 0.25)
            assert a.sample(2.75) == (0, 1, 0.25)
            assert a.sample(6)[:2] == (1, 2) and abs(a.sample(6)[2] - 1 / 3) < 1e-7
        a.close()
    m, e = v01_entries(n=2, states=3, seed=4, interpolation="linear")
    m["keys"] = [dict(time_seconds=0, state=1)]
    F.pack(tmp_asset, with_manifest(e, m))
    assert same(tmp_asset)
    a = load_gsanim(tmp_asset)
    assert all(a.sample(t) == (1, 1, 0.0) for t in (0, 3, 7.5, -2))
    a.close()


def test_comments_unknown_metadata_and_escaped_identifiers(tmp_asset):
    m, b, s, d = F.v01_asset(n=3, states=3, seed=5)
    m["provenance"] = {"unknown": ["✓", {"deep": True}, None]}
    m["keys"][1]["state"] = 2            # a state repeated by two keys
    e = F.entries_v01(m, b, s, d)
    e["base.ply"] = F.write_ply(b, comments=("allowed", "another one"))
    F.pack(tmp_asset, e)
    assert same(tmp_asset)
    text = e["manifest.json"].replace(b'"format"', b'"\\u0066ormat"').replace(b'"0.1"', b'"\\u0030.1"')
    F.pack(tmp_asset, {**e, "manifest.json": text})
    assert same(tmp_asset)
    # only \uXXXX escapes spell an identifier: "\/" makes the key unknown, so "format" goes missing
    F.pack(tmp_asset, {**e, "manifest.json": e["manifest.json"].replace(b'"format"', b'"form\\/at"')})
    assert not same(tmp_asset)


def test_half_boundaries_and_layer_counts(tmp_asset):
    m, e = v03_entries(n=2, lut_size=2, seed=6)
    halves = np.resize(np.array([0, 0x8000, 1, 0x8001, 0x03ff, 0x0400, 0x7bff, 0xfbff], np.uint16), 2 * 2 * 48)
    F.pack(tmp_asset, {**e, "layers.bin": halves.tobytes()})
    assert same(tmp_asset)
    for count in (256, 257):
        mm = copy.deepcopy(m)
        mm["layers"] = [dict(name=str(i), keys=[dict(time_seconds=0, weight=[1, 2, 3], interpolation="step")])
                        for i in range(count)]
        F.pack(tmp_asset, {**with_manifest(e, mm), "layers.bin": bytes(count * 2 * 48 * 2)})
        assert same(tmp_asset) == (count == 256)


def test_layer_names_utf8(tmp_asset):
    m, e = v03_entries(n=2, lut_size=2, seed=7)
    for names in (["café", "\U0001F600"], ["a\nb", "a\x00b"]):
        mm = copy.deepcopy(m)
        for layer, name in zip(mm["layers"], names):
            layer["name"] = name
        F.pack(tmp_asset, with_manifest(e, mm))
        assert same(tmp_asset)
        a = load_gsanim(tmp_asset)
        assert a.layer_names == [n.encode() for n in names]
        a.close()
    text = e["manifest.json"]
    # escaped and literal spellings of one name are the same name: duplicate layers
    for first, second in [(b"caf\\u00e9", "café".encode()), (b"\\ud83d\\ude00", "\U0001F600".encode())]:
        F.pack(tmp_asset, {**e, "manifest.json": text.replace(b'"steady"', b'"' + first + b'"')
                                                        .replace(b'"lamp"', b'"' + second + b'"')})
        assert not same(tmp_asset)
    for bad in [b"\\ud800", b"\\udc00", b"\\ud800x", b"\\ud800\\u0061", b"\xff"]:
        F.pack(tmp_asset, {**e, "manifest.json": text.replace(b'"lamp"', b'"' + bad + b'"')})
        assert not same(tmp_asset)


# ---- invalid manifests -----------------------------------------------------------

V01_BAD_FIELDS = [
    ("format", "other"), ("version", "0.4"), ("sh_degree", 2), ("coordinate_system", "other"),
    ("color_encoding", "linear"), ("color_encoding", "scene_linear_rec709"), ("gaussian_count", 0),
    ("gaussian_count", 3), ("gaussian_count", 1000001), ("gaussian_count", True), ("gaussian_count", 2.0),
    ("gaussian_count", -0), ("state_count", 1), ("state_count", 257), ("state_count", 3.5),
    ("duration_seconds", 0), ("duration_seconds", -1), ("duration_seconds", float("inf")),
    ("duration_seconds", True), ("interpolation", "cubic"), ("keys", []),
    ("keys", [dict(time_seconds=1, state=0)]), ("keys", [dict(time_seconds=0, state=3)]),
    ("keys", [dict(time_seconds=0, state=-1)]), ("keys", [dict(time_seconds=0, state=True)]),
    ("keys", [dict(time_seconds=0, state=0), dict(time_seconds=0, state=1)]),
    ("keys", [dict(time_seconds=0, state=0), dict(time_seconds=8, state=1)]),
    ("keys", [dict(time_seconds=0)]), ("keys", [dict(state=0)]), ("keys", {}), ("keys", [[0, 0]]),
]


def test_v01_invalid_fields(tmp_asset):
    m, e = v01_entries(n=2, states=3, seed=8)
    for field, value in V01_BAD_FIELDS:
        mm = copy.deepcopy(m)
        mm[field] = value
        F.pack(tmp_asset, with_manifest(e, mm))
        # gaussian_count -0 spells 0 and is rejected like 0; the rest are invalid
        assert not same(tmp_asset), (field, value)
    for field in m:
        mm = copy.deepcopy(m)
        del mm[field]
        F.pack(tmp_asset, with_manifest(e, mm))
        assert not same(tmp_asset), field


def dur(text: bytes, spelling: bytes) -> bytes:
    """The manifest text with duration_seconds written as `spelling`."""
    old = b'"duration_seconds": 8.0'
    assert old in text
    return text.replace(old, b'"duration_seconds": ' + spelling)


def test_manifest_text_edge_cases(tmp_asset):
    m, e = v01_entries(n=2, states=3, seed=9)
    text = e["manifest.json"]
    bad_texts = [
        text + b" {}", text.replace(b",", b"", 1), text[:-1] + b",}", text.replace(b'"format":', b'"format"'),
        text[:-1] + b',"state_count":3}', text.replace(b'"version": "0.1"', b'"version": "\\q"'),
        b" " * (1024 * 1024 + 1), b"[" * 40 + b"]" * 40, b"", b"\xef\xbb\xbf" + text, text.replace(b'"', b"'"),
        text.replace(b'"0.1"', b'"0.1\x01"'), text.replace(b'"step"', b'"st\xc0\xafep"'), b"{" * 1,
        dur(text, b"08"), dur(text, b"8."), dur(text, b".8"), dur(text, b"+8"), dur(text, b"8e"), dur(text, b"0x8"),
        dur(text, b"8" * 65), dur(text, b"NaN"), dur(text, b"1e999"),
    ]
    for i, bad in enumerate(bad_texts):
        F.pack(tmp_asset, {**e, "manifest.json": bad})
        assert not same(tmp_asset), i
    good_texts = [
        b"  \n\t" + text + b"\r\n ", dur(text, b"8.0e0"), dur(text, b"0.8e1"), dur(text, b"80E-1"),
        dur(text, b"8" + b"0" * 40 + b"e-40"),
        text[:-1] + b', "x": [' + b"[" * 30 + b"]" * 30 + b"]}",
        text[:-1] + b', "deep": ' + b"[" * 31 + b"]" * 31 + b"}",
        text[:-1] + b', "esc": "\\b\\f\\n\\r\\t\\"\\\\\\/ \\u00e9"}',
    ]
    for i, good in enumerate(good_texts):
        F.pack(tmp_asset, {**e, "manifest.json": good})
        assert same(tmp_asset), i
    # nesting: 32 levels below the root object still parse, 33 do not
    for depth, ok in ((31, True), (32, False), (40, False)):
        F.pack(tmp_asset, {**e, "manifest.json": text[:-1] + b', "n": ' + b"[" * depth + b"0" + b"]" * depth + b"}"})
        assert same(tmp_asset) == ok, depth


def test_v02_invalid_key_modes(tmp_asset):
    m, e = v01_entries(n=2, states=3, seed=10, version="0.2")
    for index in range(3):
        for value in (None, "cubic", True):
            mm = copy.deepcopy(m)
            if value is None:
                del mm["keys"][index]["interpolation"]
            else:
                mm["keys"][index]["interpolation"] = value
            F.pack(tmp_asset, with_manifest(e, mm))
            assert not same(tmp_asset), (index, value)


def test_v03_invalid_manifests(tmp_asset):
    m, e = v03_entries(n=2, lut_size=2, seed=11)
    mutations = []
    for field in m:
        bad = copy.deepcopy(m)
        del bad[field]
        mutations.append(bad)
    for field, values in [("layers", [[], {}, [m["layers"][0]] * 257, [m["layers"][0]] * 2]),
                          ("duration_seconds", [0, True, float("inf"), 1.5]),
                          ("color_encoding", ["display_referred_agx_baked"])]:
        for value in values:
            bad = copy.deepcopy(m)
            bad[field] = value
            mutations.append(bad)
    for field, values in [("name", ["", None, 3, "steady"]), ("keys", [[], {}])]:
        for value in values:
            bad = copy.deepcopy(m)
            bad["layers"][1][field] = value
            mutations.append(bad)
    for field, values in [("weight", [[1, -1, 1], [True, 1, 1], [1, 2], [1, 2, 3, 4], "abc", [1, float("nan"), 1],
                                      [1e300, 1, 1]]),
                          ("interpolation", [None, "cubic", True]),
                          ("time_seconds", [1, -1, True, float("inf")])]:
        for value in values:
            bad = copy.deepcopy(m)
            bad["layers"][1]["keys"][0][field] = value
            mutations.append(bad)
    for field in ("weight", "time_seconds", "interpolation"):
        bad = copy.deepcopy(m)
        del bad["layers"][1]["keys"][2][field]
        mutations.append(bad)
    for time in (0, 2):
        bad = copy.deepcopy(m)
        bad["layers"][1]["keys"][1]["time_seconds"] = time
        mutations.append(bad)
    for field, values in [("size", [1, 257, 2.0, True, 3]), ("log2_min", [3, 4, float("nan")]),
                          ("log2_max", [float("inf"), -2]), ("layout", ["b_fastest"]),
                          ("encoding", ["float16"]), ("type", ["other"])]:
        for value in values:
            bad = copy.deepcopy(m)
            bad["display_transform"][field] = value
            mutations.append(bad)
    for field in m["display_transform"]:
        bad = copy.deepcopy(m)
        del bad["display_transform"][field]
        mutations.append(bad)
    for i, bad in enumerate(mutations):
        F.pack(tmp_asset, with_manifest(e, bad))
        assert not same(tmp_asset), i
    # 0.1 fields in a 0.3 manifest are ignored metadata; 0.3 fields in 0.1 too
    ok = copy.deepcopy(m)
    ok.update(state_count="x", interpolation=7, keys="y")
    F.pack(tmp_asset, with_manifest(e, ok))
    assert same(tmp_asset)
    m1, e1 = v01_entries(n=2, states=3, seed=12)
    m1.update(layers=3, display_transform=[])
    F.pack(tmp_asset, with_manifest(e1, m1))
    assert same(tmp_asset)


# ---- payloads and archive damage -----------------------------------------------------

def test_v01_bad_payloads_and_archive(tmp_asset):
    m, b, s, d = F.v01_asset(n=2, states=3, seed=13)
    original = F.entries_v01(m, b, s, d)
    variants = []
    for name in original:
        variants.append({k: v for k, v in original.items() if k != name})
        variants.append({**original, name: original[name][:-1]})
        variants.append({**original, name: original[name] + b"X"})
    variants += [{**original, "../bad": b"x"}, {**original, "dir/": b""},
                 list(original.items()) + [("base.ply", original["base.ply"])],
                 {**original, "deltas.bin": b"\x80" + original["deltas.bin"][1:]},
                 {**{k: v for k, v in original.items() if k != "deltas.bin"}, "layers.bin": original["deltas.bin"]}]
    for value in (0.0, -1.0, float("nan"), float("inf"), 3e38):
        variants.append({**original, "scales.bin": struct.pack("<f", value) + original["scales.bin"][4:]})
    for index, value in [(0, float("nan")), (3, float("inf")), (55, 1000), (55, -1000), (58, 3e38), (56, 44.5)]:
        bb = b.copy()
        bb[0, index] = value
        variants.append({**original, "base.ply": F.write_ply(bb)})
    bb = b.copy()
    bb[1, 58:62] = 0
    variants.append({**original, "base.ply": F.write_ply(bb)})
    for old, new in [(b"float x", b"float y"), (b"float x", b"double x"), (b"element vertex 2", b"element vertex 3"),
                     (b"end_header", b"element face 1\nend_header"), (b"\n", b"\r\n"), (b"ply\n", b"comment x\nply\n")]:
        variants.append({**original, "base.ply": original["base.ply"].replace(old, new)})
    for i, entries in enumerate(variants):
        F.pack(tmp_asset, entries)
        assert not same(tmp_asset), i
    F.pack(tmp_asset, original, zipfile.ZIP_BZIP2)
    assert not same(tmp_asset)
    # each stored payload corrupted without updating its CRC
    for name in original:
        F.pack(tmp_asset, original)
        with zipfile.ZipFile(tmp_asset) as z:
            offset = z.getinfo(name).header_offset
        blob = bytearray(tmp_asset.read_bytes())
        n, extra = struct.unpack_from("<HH", blob, offset + 26)
        blob[offset + 30 + n + extra] ^= 1
        tmp_asset.write_bytes(bytes(blob))
        assert not same(tmp_asset), name
    F.pack(tmp_asset, original)
    blob = tmp_asset.read_bytes()
    tmp_asset.write_bytes(blob[:-10])
    assert not same(tmp_asset)
    tmp_asset.write_bytes(blob + b"trailing comment bytes")
    same(tmp_asset)     # whatever the verdict, both loaders agree
    tmp_asset.write_bytes(b"")
    assert not same(tmp_asset)
    assert not same(tmp_asset.parent / "missing.gsanim")


def test_v01_delta_overflow_is_rejected(tmp_asset):
    m, b, s, d = F.v01_asset(n=2, states=3, seed=14)
    s = s.copy()
    s[5] = 3e36                       # 127 * 3e36 overflows float
    d = d.copy()
    d[1, 1, 5] = 127
    F.pack(tmp_asset, F.entries_v01(m, b, s, d))
    assert not same(tmp_asset)
    bb = b.copy()
    bb[0, 6 + 7] = 3.4e38             # a finite base whose sum with a delta overflows
    s2 = np.full(48, 1e37, np.float32)
    d2 = np.full_like(d, 100)
    F.pack(tmp_asset, F.entries_v01(m, bb, s2, d2))
    assert not same(tmp_asset)


def test_v03_bad_payloads(tmp_asset):
    m, b, h, lut = F.v03_asset(n=2, lut_size=2, seed=15)
    original = F.entries_v03(m, b, h, lut)
    variants = []
    for name in original:
        variants.append({**original, name: original[name][:-1]})
        variants.append({**original, name: original[name] + b"X"})
    for half in (0x7c00, 0xfc00, 0x7e00):
        variants.append({**original, "layers.bin": struct.pack("<H", half) + original["layers.bin"][2:]})
    for index in (6, 8, 9, 53):               # appearance in a 0.3 base is invalid
        bb = b.copy()
        bb[0, index] = 1
        variants.append({**original, "base.ply": F.write_ply(bb)})
    variants += [{**original, "deltas.bin": b""}, list(original.items()) + [("layers.bin", original["layers.bin"])]]
    for i, entries in enumerate(variants):
        F.pack(tmp_asset, entries)
        assert not same(tmp_asset), i
    for name in original:
        F.pack(tmp_asset, original)
        with zipfile.ZipFile(tmp_asset) as z:
            offset = z.getinfo(name).header_offset
        blob = bytearray(tmp_asset.read_bytes())
        n, extra = struct.unpack_from("<HH", blob, offset + 26)
        blob[offset + 30 + n + extra] ^= 1
        tmp_asset.write_bytes(bytes(blob))
        assert not same(tmp_asset), name
    # normals are not appearance: any finite value is allowed
    bb = b.copy()
    bb[:, 3:6] = 5
    F.pack(tmp_asset, {**original, "base.ply": F.write_ply(bb)})
    assert same(tmp_asset)


def test_rows_are_the_ply_transforms(tmp_asset):
    """The rows are the loader's decode (exp scale, sigmoid opacity, unit
    quaternion, channel-major f_rest reordered to RGB triples) packed as
    GpuGaussian rows, the same as gs_pack_raw of the base attributes."""
    from gamesplat_b200 import pack_raw

    m, b, s, d = F.v01_asset(n=7, states=2, seed=16)
    F.pack(tmp_asset, F.entries_v01(m, b, s, d))
    a = load_gsanim(tmp_asset)
    raw = np.concatenate([b[:, 0:3], b[:, 6:62]], axis=1)
    assert np.array_equal(a.rows.view(np.uint32), pack_raw(raw).view(np.uint32))
    assert np.allclose(a.rows[:, 4:7], np.exp(b[:, 55:58]), rtol=1e-6)
    a.close()


def test_bad_arguments():
    lib = L.lib()
    import ctypes as C

    h = C.c_void_p(1)
    assert lib.gs_gsanim_load(None, C.byref(h)) == L.GS_ERR_BAD_ARG and not h.value
    assert lib.gs_gsanim_load(b"x", None) == L.GS_ERR_BAD_ARG
    assert lib.gs_gsanim_get_info(None, None) == L.GS_ERR_BAD_ARG
    assert lib.gs_gsanim_rows(None, None) == L.GS_ERR_BAD_ARG
    lib.gs_gsanim_free(None)


@pytest.mark.parametrize("target", ["manifest", "ply", "archive"])
def test_random_mutations_agree(tmp_asset, target):
    """Seeded random byte edits of a valid asset: both loaders reach the same
    verdict and, where they accept, the same outputs."""
    rng = np.random.default_rng({"manifest": 1, "ply": 2, "archive": 3}[target])
    m, e = v01_entries(n=3, states=3, seed=17, version="0.2", interpolation="linear")
    m3, e3 = v03_entries(n=3, lut_size=2, seed=18)
    accepted = 0
    for trial in range(150):
        entries = dict(e if trial % 2 == 0 else e3)
        if target == "archive":
            F.pack(tmp_asset, entries, zipfile.ZIP_DEFLATED if trial % 3 == 0 else zipfile.ZIP_STORED)
            blob = bytearray(tmp_asset.read_bytes())
        else:
            name = "manifest.json" if target == "manifest" else "base.ply"
            blob = bytearray(entries[name])
        for _ in range(int(rng.integers(1, 4))):
            pos = int(rng.integers(0, len(blob)))
            kind = int(rng.integers(0, 3))
            if kind == 0:
                blob[pos] ^= 1 << int(rng.integers(0, 8))
            elif kind == 1:
                blob[pos] = int(rng.integers(0, 256))
            else:
                del blob[pos]
        if target == "archive":
            tmp_asset.write_bytes(bytes(blob))
        else:
            entries[name] = bytes(blob)
            F.pack(tmp_asset, entries)
        accepted += same(tmp_asset)
    assert accepted < 150


def test_zip_structure_mutations_agree(tmp_asset):
    """Seeded edits of the archive's own records (central directory, local
    headers, end record), data in front of the archive, trailing data and
    comments, and +-small changes of entry sizes, offsets and disk numbers:
    both loaders reach the same verdict and the same outputs."""
    rng = np.random.default_rng(21)
    _, e = v01_entries(n=3, states=3, seed=17, version="0.2", interpolation="linear")
    accepted = 0
    for trial in range(360):
        F.pack(tmp_asset, e, zipfile.ZIP_DEFLATED if trial % 2 else zipfile.ZIP_STORED)
        blob = bytearray(tmp_asset.read_bytes())
        eocd = blob.rfind(b"PK\x05\x06")
        cd_off = struct.unpack_from("<I", blob, eocd + 16)[0]
        kind = trial % 6
        if kind == 0:
            blob[cd_off + int(rng.integers(0, eocd - cd_off))] = int(rng.integers(0, 256))
        elif kind == 1:
            blob[eocd + int(rng.integers(4, 22))] = int(rng.integers(0, 256))
        elif kind == 2:
            with zipfile.ZipFile(tmp_asset) as z:
                local = z.infolist()[int(rng.integers(0, 4))].header_offset
            blob[local + int(rng.integers(4, 30))] = int(rng.integers(0, 256))
        elif kind == 3:
            blob = bytearray(rng.integers(0, 256, int(rng.integers(1, 300)), dtype=np.uint8).tobytes()) + blob
        elif kind == 4:
            tail = rng.integers(0, 256, int(rng.integers(1, 300)), dtype=np.uint8).tobytes()
            if rng.integers(0, 2):
                struct.pack_into("<H", blob, eocd + 20, len(tail))     # a declared comment
            blob += tail
        else:
            h = cd_off
            for _ in range(int(rng.integers(0, 4))):
                nl, el, cl = struct.unpack_from("<HHH", blob, h + 28)
                h += 46 + nl + el + cl
            off = [20, 24, 42, 34][int(rng.integers(0, 4))]     # compressed / uncompressed size, offset, disk
            fmt, bits_ = ("<H", 16) if off == 34 else ("<I", 32)
            v = struct.unpack_from(fmt, blob, h + off)[0]
            struct.pack_into(fmt, blob, h + off, (v + int(rng.choice([-2, -1, 1, 2, 100]))) % (1 << bits_))
        tmp_asset.write_bytes(bytes(blob))
        accepted += same(tmp_asset)
    assert 0 < accepted < 360
