"""gs_load_ply against the reference PLY loader compiled from its sources
(gaussian_load_ply + pack_gpu_gaussians, src/gaussian_loader_ply.cpp:14-228,
src/gaussian.cpp:53-73): the same verdict on every file and, where both
load it, the same GpuGaussian rows bit for bit.  Files: a valid 3DGS PLY,
its header rules (format lines, atoi vertex counts, property types and
orders, lists, other elements, the 128-name limit, long and CRLF lines) and
seeded mutations of header and body.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from gamesplat_b200 import _lib as L
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference CPU build (oracle/_ref) not present")

NAMES = (["x", "y", "z", "nx", "ny", "nz"] + [f"f_dc_{i}" for i in range(3)] + [f"f_rest_{i}" for i in range(45)] +
         ["opacity"] + [f"scale_{i}" for i in range(3)] + [f"rot_{i}" for i in range(4)])


def ply(n=6, seed=0, header=None, body=None):
    rng = np.random.default_rng(seed)
    vals = rng.normal(0, 1, (n, len(NAMES))).astype("<f4")
    lines = header if header is not None else (
        ["ply", "format binary_little_endian 1.0", f"element vertex {n}"] + [f"property float {p}" for p in NAMES] +
        ["end_header"])
    return ("\n".join(lines) + "\n").encode() + (body if body is not None else vals.tobytes())


def ours(path):
    lib = L.lib()
    n = lib.gs_load_ply(str(path).encode(), None, 0)
    if n <= 0:
        return None
    rows = np.zeros((n, 64), np.float32)
    got = lib.gs_load_ply(str(path).encode(), rows.ctypes.data, n)
    return rows if got == n else None


def reference(path):
    R = O.ref()
    n = R.ref_load_ply_rows(str(path).encode(), None, 0)
    if n == 0:
        return None
    rows = np.zeros((n, 64), np.float32)
    R.ref_load_ply_rows(str(path).encode(), rows.ctypes.data, n)
    return rows


ATTRS = ["x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3", "opacity",
         "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{k}" for k in range(45)]
SIZES = {"float": 4, "float32": 4, "int": 4, "int32": 4, "uint": 4, "uint32": 4, "double": 8, "float64": 8,
         "uchar": 1, "uint8": 1, "short": 2, "int16": 2, "ushort": 2, "uint16": 2}


def defined_in_reference(data: bytes) -> bool:
    """False when the reference loader's decode of this header is undefined:
    a group (scale, rotation, DC) named by its first member only, whose
    missing members it reads a byte before the row, or a used value whose 4
    bytes run past the row.  Follows its header reading: fgets of 511 bytes,
    trailing CR/LF stripped, sscanf("property %31s %63s"), the first 128
    vertex property names kept, every vertex property advancing the stride."""
    names, stride, pos, in_vertex = [], 0, 0, False
    while pos < len(data):
        nl = data.find(b"\n", pos, pos + 511)
        end = nl + 1 if nl != -1 else min(pos + 511, len(data))
        line = data[pos:end].split(b"\0")[0].rstrip(b"\r\n")
        pos = end
        if line == b"end_header":
            break
        if line.startswith(b"element vertex "):
            in_vertex = True
            continue
        if line.startswith(b"element "):
            in_vertex = False
            continue
        if in_vertex and line.startswith(b"property "):
            rest = line[len(b"property"):].lstrip()
            tok = rest.split(None, 1)
            if not tok:
                continue
            typ, after = tok[0][:31], rest[len(tok[0][:31]):]
            after = after.lstrip() if len(tok[0]) <= 31 else after
            ntok = after.split(None, 1)
            if not ntok:
                continue
            if len(names) < 128:
                names.append((ntok[0][:63].decode("latin-1"), stride))
            stride += SIZES.get(typ.decode("latin-1"), 4)
    off = {a: next((o for nm, o in names if nm == a), -1) for a in ATTRS}
    for first, members in (("scale_0", 3), ("rot_0", 4), ("f_dc_0", 3)):
        group = ATTRS[ATTRS.index(first):ATTRS.index(first) + members]
        if off[first] >= 0 and any(off[m] < 0 for m in group):
            return False
    return all(o < 0 or o + 4 <= stride for o in off.values())


def same(path, data) -> bool:
    path.write_bytes(data)
    if not defined_in_reference(data):
        ours(path)                     # must not crash; the reference has no defined result to match
        return False
    r, o = reference(path), ours(path)
    assert (r is None) == (o is None), f"reference {'rejects' if r is None else 'accepts'}, ours does not"
    if r is None:
        return False
    assert r.shape == o.shape and np.array_equal(r.view(np.uint32), o.view(np.uint32))
    return True


def test_header_rules(tmp_path):
    p = tmp_path / "a.ply"
    base = ["ply", "format binary_little_endian 1.0", "element vertex 6"] + [f"property float {n}" for n in NAMES]
    body = ply(6)[len(ply(6, header=base + ["end_header"], body=b"")):]
    cases = {
        "valid": (base + ["end_header"], True),
        "no format line": ([l for l in base if not l.startswith("format")] + ["end_header"], True),
        "ascii": ([l.replace("binary_little_endian", "ascii") for l in base] + ["end_header"], False),
        "two formats": (base[:2] + ["format ascii 1.0"] + base[2:] + ["end_header"], False),
        "count with letters": ([l.replace("vertex 6", "vertex 6abc") for l in base] + ["end_header"], True),
        "count zero": ([l.replace("vertex 6", "vertex 0") for l in base] + ["end_header"], False),
        "count negative": ([l.replace("vertex 6", "vertex -1") for l in base] + ["end_header"], False),
        "count 2^32 + 6": ([l.replace("vertex 6", "vertex 4294967302") for l in base] + ["end_header"], None),
        "no end_header": (base, False),
        "other element after": (base + ["element face 2", "property list uchar int vertex_indices", "end_header"], True),
        "comments": (base[:2] + ["comment made by a test", "obj_info x"] + base[2:] + ["end_header"], True),
        "CRLF": ([l + "\r" for l in base] + ["end_header\r"], True),
        "no position": ([l for l in base if l != "property float x"] + ["end_header"], False),
        "no scale": ([l for l in base if "scale_" not in l] + ["end_header"], True),
        "no rotation": ([l for l in base if "rot_" not in l] + ["end_header"], True),
        "double x": ([l.replace("property float x", "property double x") for l in base] + ["end_header"], False),
        "unknown type": ([l.replace("property float nx", "property half nx") for l in base] + ["end_header"], True),
    }
    for name, (header, expect) in cases.items():
        got = same(p, ply(6, header=header, body=body))
        if expect is not None:
            assert got == expect, name
    many = base[:3] + [f"property float extra_{i}" for i in range(130)] + base[3:] + ["end_header"]
    rng = np.random.default_rng(1)
    same(p, ply(6, header=many, body=rng.normal(0, 1, (6, 130 + len(NAMES))).astype("<f4").tobytes()))
    long_line = base[:2] + ["comment " + "x" * 700] + base[2:] + ["end_header"]
    same(p, ply(6, header=long_line, body=body))


def test_truncated_and_trailing(tmp_path):
    p = tmp_path / "a.ply"
    data = ply(9, seed=3)
    assert same(p, data)
    assert not same(p, data[:-1])
    assert not same(p, data[:-248 * 3])
    assert same(p, data + b"trailing")


def test_random_header_mutations(tmp_path):
    p = tmp_path / "a.ply"
    rng = np.random.default_rng(7)
    data = ply(5, seed=8)
    head_len = data.index(b"end_header\n") + len(b"end_header\n")
    accepted = 0
    for _ in range(400):
        blob = bytearray(data)
        for _ in range(int(rng.integers(1, 3))):
            pos = int(rng.integers(0, head_len))
            kind = int(rng.integers(0, 3))
            if kind == 0:
                blob[pos] = int(rng.choice(list(b"0123456789 \nabcdefxyz_-")))
            elif kind == 1:
                del blob[pos]
            else:
                blob.insert(pos, int(rng.choice(list(b"0123456789 \nex_"))))
        accepted += same(p, bytes(blob))
    assert 0 < accepted < 400
