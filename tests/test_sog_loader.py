"""SOG archive loading (gs_load_sog) and lossless WebP decoding
(gs_webp_decode_rgba) against the reference loader and the libwebp decoder it
calls, both compiled from the reference's sources (gaussian_load_sog,
src/gaussian_loader_sog.cpp:126-551; WebPGetInfo + WebPDecodeRGBA).

Accepted archives must decode to the same GpuGaussian rows bit for bit;
every failure the reference checks (meta fields, file presence, image sizes,
quaternion modes, shN labels and centroid sizes, damaged images and
archives) must fail here too.  The WebP decoder must give libwebp's pixels
for lossless images of every transform and code path the encoder emits, and
the same verdict on damaged ones.  CPU only.
"""
from __future__ import annotations

import copy
import io
import json
import struct
import zipfile

import numpy as np
import pytest

from gamesplat_b200 import GsError, load_sog, webp_decode
from gamesplat_b200 import _lib as L
from oracle import oracle as O
from tests import sog_fixture as S

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference CPU build (oracle/_ref) not present")


def ours(path):
    try:
        return load_sog(path)
    except GsError as e:
        assert e.status == L.GS_ERR_FORMAT, e
        return None


def same(path) -> bool:
    """Both loaders agree on `path`; True if they accepted it."""
    r, o = O.ref_sog_rows(path), ours(path)
    assert (r is None) == (o is None), f"reference {'rejects' if r is None else 'accepts'}, ours does not"
    if r is None:
        return False
    assert r.shape == o.shape
    assert np.array_equal(r.view(np.uint32), o.view(np.uint32))
    return True


def decode_ours(data: bytes):
    try:
        return webp_decode(data)
    except GsError as e:
        assert e.status == L.GS_ERR_FORMAT, e
        return None


def same_webp(data: bytes) -> bool:
    r, o = O.ref_webp_decode(data), decode_ours(data)
    assert (r is None) == (o is None), f"libwebp {'rejects' if r is None else 'accepts'}, ours does not"
    if r is None:
        return False
    assert r.shape == o.shape and np.array_equal(r, o)
    return True


@pytest.fixture
def sog(tmp_path):
    return tmp_path / "asset.sog"


# ---- valid archives -----------------------------------------------------------------

@pytest.mark.parametrize("compression", [zipfile.ZIP_STORED, zipfile.ZIP_DEFLATED])
@pytest.mark.parametrize("n,bands", [(1, 0), (2, 1), (50, 2), (333, 3), (1000, 0)])
def test_assets_match_reference(sog, compression, n, bands):
    meta, imgs = S.sog_asset(n, seed=n + bands, bands=bands)
    S.pack(sog, S.entries(meta, imgs), compression)
    assert same(sog)
    rows = load_sog(sog)
    assert rows.shape == (n, 64)
    assert np.all(rows[:, 3] == imgs["sh0.webp"].reshape(-1, 4)[:n, 3] / np.float32(255))


def test_decode_formulas(sog):
    """Spot checks of the decode itself: signed exp(|v|) - 1 positions,
    exp(codebook) scales, smallest-three quaternions, alpha / 255 opacity."""
    meta, imgs = S.sog_asset(9, seed=3)
    S.pack(sog, S.entries(meta, imgs))
    rows = load_sog(sog)
    px = {k: v.reshape(-1, 4)[:9].astype(np.int64) for k, v in imgs.items()}
    q = px["means_u.webp"][:, :3] << 8 | px["means_l.webp"][:, :3]
    lo, hi = np.float32(meta["means"]["mins"]), np.float32(meta["means"]["maxs"])
    v = lo + (hi - lo) * (q.astype(np.float32) / np.float32(65535))
    np.testing.assert_allclose(rows[:, 0:3], np.sign(v) * np.expm1(np.abs(v)), rtol=2e-6, atol=1e-7)
    cb = np.float32(meta["scales"]["codebook"])
    np.testing.assert_allclose(rows[:, 4:7], np.exp(cb[px["scales.webp"][:, :3]]), rtol=2e-6)
    quat = rows[:, 8:12]
    mode = px["quats.webp"][:, 3] - 252
    stored = ((px["quats.webp"][:, :3] / 255.0 - 0.5) * 2 / np.sqrt(2)).astype(np.float32)
    for i in range(9):
        others = [quat[i, s] for s in range(4) if s != mode[i]]
        np.testing.assert_allclose(others, stored[i], rtol=1e-6, atol=1e-7)
        # the omitted component completes a unit quaternion (0 when the stored three exceed one)
        rest = float(np.sum(stored[i].astype(np.float64) ** 2))
        np.testing.assert_allclose(quat[i, mode[i]], np.sqrt(max(0.0, 1.0 - rest)), atol=1e-6)


# ---- invalid meta, files and images ------------------------------------------------------

def mutate(meta, path, value):
    m = copy.deepcopy(meta)
    node = m
    for k in path[:-1]:
        node = node[k]
    if value is DELETE:
        del node[path[-1]]
    else:
        node[path[-1]] = value
    return m


DELETE = object()

META_CASES = [
    (("version",), 1), (("version",), 3), (("version",), "2"), (("version",), DELETE), (("version",), 1.9),
    (("count",), 0), (("count",), -3), (("count",), "5"), (("count",), DELETE), (("count",), 10 ** 12),
    (("antialias",), 1), (("antialias",), None),
    (("means",), DELETE), (("means",), []), (("means", "mins"), [0, 0]), (("means", "mins"), [0, 0, 0, 0]),
    (("means", "mins"), DELETE), (("means", "maxs"), ["a", 1, 2]), (("means", "files"), ["means_l.webp"]),
    (("means", "files"), DELETE), (("means", "files"), ["means_l.webp", "nothere.webp"]),
    (("scales",), DELETE), (("scales", "codebook"), [0.0] * 255), (("scales", "codebook"), [0.0] * 257),
    (("scales", "files"), []), (("scales", "files"), ["scales.webp", "scales.webp"]),
    (("quats",), DELETE), (("quats", "files"), DELETE), (("quats", "files"), [3]),
    (("sh0",), DELETE), (("sh0", "codebook"), DELETE), (("sh0", "files"), "sh0.webp"),
    (("shN", "count"), 0), (("shN", "count"), 65537), (("shN", "bands"), 0), (("shN", "bands"), 4),
    (("shN", "count"), DELETE), (("shN", "codebook"), [0.5] * 3), (("shN", "files"), ["shN_centroids.webp"]),
    (("shN", "files"), ["shN_labels.webp", "shN_centroids.webp"]), (("shN", "count"), 1),
]


def test_invalid_meta(sog):
    meta, imgs = S.sog_asset(20, seed=5, bands=1, shn_count=70)
    e = S.entries(meta, imgs)
    for path, value in META_CASES:
        S.pack(sog, {**e, "meta.json": json.dumps(mutate(meta, path, value)).encode()})
        assert not same(sog), (path, value)


def test_meta_reading_rules(sog):
    """Rules of the reference's meta reader that accept: numbers through
    strtol / strtof of their text, escaped slashes, later duplicates
    overriding earlier ones, unknown fields, a shN field without shN data."""
    meta, imgs = S.sog_asset(20, seed=6)
    e = S.entries(meta, imgs)
    text = json.dumps(meta)
    variants = [
        text.replace('"count": 20', '"count": 20.9'), text.replace('"count": 20', '"count": 2e1'),
        text.replace('"version": 2', '"version": 2.5'),
        text.replace('"quats.webp"', '"quats\\/x.webp"'),
        text[:-1] + ', "count": 4, "extra": {"deep": [[[1]]]}}',
        text[:-1] + ', "means": ' + json.dumps(meta["means"]) + '}',
        text[:-1] + ', "antialias": true}',
    ]
    expect = [True, True, True, False, True, True, True]
    for t, ok in zip(variants, expect):
        S.pack(sog, {**e, "meta.json": t.encode()})
        assert same(sog) == ok, t[:80]
    S.pack(sog, {**e, "quats/x.webp": e["quats.webp"], "meta.json": variants[3].encode()})
    assert same(sog)
    for bad in ['"quats\\u002ewebp"', '"quats\\bwebp"']:      # escapes the reader does not take
        S.pack(sog, {**e, "meta.json": text.replace('"quats.webp"', bad).encode()})
        assert not same(sog), bad
    long_name = "q" * 130 + ".webp"                             # names are cut to 127 bytes
    S.pack(sog, {**e, long_name: e["quats.webp"],
                 "meta.json": text.replace('"quats.webp"', json.dumps(long_name)).encode()})
    assert not same(sog)
    S.pack(sog, {**e, long_name[:127]: e["quats.webp"],
                 "meta.json": text.replace('"quats.webp"', json.dumps(long_name)).encode()})
    assert same(sog)


def test_invalid_images(sog):
    meta, imgs = S.sog_asset(30, seed=7, bands=2, shn_count=100)
    e = S.entries(meta, imgs)
    cases = []
    for name in imgs:
        cases.append({k: v for k, v in e.items() if k != name})            # missing file
        cases.append({**e, name: e[name][:-3]})                             # truncated image
        cases.append({**e, name: b"RIFF" + e[name][4:12] + b"VP8 " + e[name][16:]})
    q = imgs["quats.webp"].copy()
    q[0, 0, 3] = 251
    cases.append({**e, "quats.webp": S.webp(q)})                           # quaternion mode out of range
    q[0, 0, 3] = 0
    cases.append({**e, "quats.webp": S.webp(q)})
    cases.append({**e, "scales.webp": S.webp(imgs["scales.webp"][:, :-1])})  # size mismatch
    small = {k: v[:1, :1] for k, v in imgs.items() if not k.startswith("shN")}
    cases.append({**e, **{k: S.webp(v) for k, v in small.items()}})        # fewer pixels than Gaussians
    lab = imgs["shN_labels.webp"].copy()
    lab[0, 0, 0], lab[0, 0, 1] = 100 & 255, 100 >> 8                       # label == count
    cases.append({**e, "shN_labels.webp": S.webp(lab)})
    cases.append({**e, "shN_centroids.webp": S.webp(imgs["shN_centroids.webp"][:, :-1])})
    cases.append({**e, "shN_centroids.webp": S.webp(imgs["shN_centroids.webp"][:1])})
    cases.append({**e, "shN_labels.webp": S.webp(imgs["shN_labels.webp"][:1, :1])})
    cases.append({k: v for k, v in e.items() if k != "meta.json"})
    cases.append({**e, "meta.json": b""})
    for i, c in enumerate(cases):
        S.pack(sog, c)
        assert not same(sog), i
    # a label image larger than needed and centroids wider than needed are fine
    lab2 = np.zeros((lab.shape[0] + 3, lab.shape[1] + 2, 4), np.uint8)
    lab2[:lab.shape[0], :lab.shape[1]] = imgs["shN_labels.webp"]
    S.pack(sog, {**e, "shN_labels.webp": S.webp(lab2)})
    same(sog)     # the label image is read by Gaussian index, so only its pixel count matters to both loaders
    cen = np.concatenate([imgs["shN_centroids.webp"], imgs["shN_centroids.webp"]], axis=1)
    S.pack(sog, {**e, "shN_centroids.webp": S.webp(cen)})
    assert same(sog)


def test_archive_entries(sog):
    """Every entry is read (one damaged entry fails the archive, even one the
    meta does not name), directories are skipped, the first of two entries
    with one name is used, data in front of the archive is allowed."""
    meta, imgs = S.sog_asset(12, seed=8)
    e = S.entries(meta, imgs)
    S.pack(sog, {**e, "notes/": b"", "extra.bin": b"anything"})
    assert same(sog)
    S.pack(sog, list(e.items()) + [("quats.webp", b"not an image")])
    assert same(sog)
    S.pack(sog, [("quats.webp", b"not an image")] + list(e.items()))
    assert not same(sog)
    S.pack(sog, e)
    with zipfile.ZipFile(sog) as z:
        info = z.getinfo("extra.bin") if "extra.bin" in z.namelist() else z.getinfo("sh0.webp")
    blob = bytearray(sog.read_bytes())
    n, extra = struct.unpack_from("<HH", blob, info.header_offset + 26)
    blob[info.header_offset + 30 + n + extra] ^= 0x10
    sog.write_bytes(bytes(blob))
    assert not same(sog)
    S.pack(sog, e, zipfile.ZIP_DEFLATED)
    sog.write_bytes(b"prefix bytes " * 7 + sog.read_bytes())
    assert same(sog)
    S.pack(sog, e, zipfile.ZIP_BZIP2)
    assert not same(sog)


def test_random_meta_and_image_mutations(sog):
    """Seeded byte edits of meta.json and of the images: the same verdict,
    and for accepted archives the same rows."""
    rng = np.random.default_rng(11)
    meta, imgs = S.sog_asset(25, seed=9, bands=1, shn_count=20)
    e = S.entries(meta, imgs)
    names = list(e)
    accepted = 0
    for trial in range(240):
        name = names[trial % len(names)]
        blob = bytearray(e[name])
        for _ in range(int(rng.integers(1, 3))):
            pos = int(rng.integers(0, len(blob)))
            if rng.integers(0, 2):
                blob[pos] ^= 1 << int(rng.integers(0, 8))
            else:
                blob[pos] = int(rng.integers(0, 256))
        text = bytes(blob)
        if name == "meta.json":
            try:
                json.loads(text.decode("utf-8"))
            except (ValueError, UnicodeDecodeError):
                continue          # malformed JSON: the reference's token reader may accept some, ours never
        S.pack(sog, {**e, name: text})
        accepted += same(sog)
    assert accepted > 0


# ---- WebP ---------------------------------------------------------------------------------

def varied_images(rng):
    out = []
    for h, w in [(1, 1), (2, 3), (9, 17), (40, 33), (130, 70)]:
        out.append(rng.integers(0, 256, (h, w, 4)).astype(np.uint8))
        y, x = np.mgrid[0:h, 0:w]
        out.append(np.stack([(x * 3) % 256, (y * 5) % 256, ((x + y) * 2) % 256, np.full_like(x, 255)],
                            -1).astype(np.uint8))
        for colors in (2, 3, 5, 16, 17, 256):
            pal = rng.integers(0, 256, (colors, 4)).astype(np.uint8)
            out.append(pal[rng.integers(0, colors, (h, w))])
        tile = rng.integers(0, 256, (3, 5, 4)).astype(np.uint8)
        out.append(np.tile(tile, (h // 3 + 1, w // 5 + 1, 1))[:h, :w])
    return out


def test_webp_lossless_matches_libwebp():
    rng = np.random.default_rng(12)
    for a in varied_images(rng):
        for kw in ({}, {"method": 0}, {"method": 6, "quality": 100}):
            data = S.webp(a, **kw)
            assert same_webp(data)
            assert np.array_equal(decode_ours(data), a)


def test_webp_containers():
    rng = np.random.default_rng(13)
    a = rng.integers(0, 256, (6, 10, 4)).astype(np.uint8)
    data = S.webp(a)
    assert data[12:16] == b"VP8L"
    vp8l = data[20:20 + struct.unpack_from("<I", data, 16)[0]]
    assert same_webp(vp8l)                                        # raw bitstream
    vp8x = b"VP8X" + struct.pack("<I", 10) + bytes([0x10, 0, 0, 0]) + (9).to_bytes(3, "little") + (5).to_bytes(3, "little")
    extra = b"EXTR" + struct.pack("<I", 3) + b"abc\x00"
    body = b"WEBP" + vp8x + extra + data[12:]
    assert same_webp(b"RIFF" + struct.pack("<I", len(body)) + body)   # extended container
    anim = bytearray(vp8x)
    anim[8] |= 0x02
    body = b"WEBP" + bytes(anim) + data[12:]
    assert not same_webp(b"RIFF" + struct.pack("<I", len(body)) + body)   # animation
    assert not same_webp(b"")
    assert not same_webp(data[:-1])
    assert not same_webp(b"RIFF" + struct.pack("<I", len(data)) + data[8:])   # RIFF size past the end


def test_lossy_webp_is_rejected():
    """libwebp also decodes lossy (VP8) images; SOG writes lossless ones and
    this decoder reads only those."""
    from PIL import Image

    a = np.random.default_rng(14).integers(0, 256, (8, 8, 4)).astype(np.uint8)
    b = io.BytesIO()
    Image.fromarray(a, "RGBA").save(b, "WEBP", quality=80)
    assert O.ref_webp_decode(b.getvalue()) is not None
    assert decode_ours(b.getvalue()) is None


def test_webp_mutations_agree():
    rng = np.random.default_rng(15)
    sources = [S.webp(a) for a in varied_images(np.random.default_rng(16))[::3]]
    decoded = 0
    for trial in range(1500):
        blob = bytearray(sources[trial % len(sources)])
        for _ in range(int(rng.integers(1, 3))):
            pos = int(rng.integers(0, len(blob)))
            kind = int(rng.integers(0, 3))
            if kind == 0:
                blob[pos] ^= 1 << int(rng.integers(0, 8))
            elif kind == 1:
                blob[pos] = int(rng.integers(0, 256))
            else:
                del blob[pos]
        decoded += same_webp(bytes(blob))
    assert 0 < decoded < 1500


def test_webp_declared_size_beyond_the_data():
    """A 16384 x 16384 lossless stream whose pixels need one bit each but
    ends after 16 bytes of them: both decoders reject it, and this one does
    so without committing memory for the declared size."""
    import resource

    bits = []

    def put(value, n):
        bits.extend((value >> i) & 1 for i in range(n))

    put(0x2F, 8)
    put(16383, 14)
    put(16383, 14)
    put(0, 1)
    put(0, 3)
    put(0, 1)      # no transform
    put(0, 1)      # no color cache
    put(0, 1)      # no meta prefix codes
    put(1, 1); put(1, 1); put(1, 1); put(0, 8); put(1, 8)     # green: symbols 0 and 1, one bit each
    for _ in range(4):                                         # red, blue, alpha, distance: one symbol
        put(1, 1); put(0, 1); put(0, 1); put(0, 1)
    put(0x5A5A5A5A5A5A5A5A5A5A5A5A5A5A5A5A, 128)            # 128 pixels of data, then the stream ends
    data = bytes(sum(b << i for i, b in enumerate(bits[k:k + 8])) for k in range(0, len(bits), 8))
    before = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss
    assert decode_ours(data) is None
    grown_kb = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss - before
    assert grown_kb < 64 * 1024, grown_kb          # far below the 1 GiB the header declares
    assert O.ref_webp_decode(data) is None
