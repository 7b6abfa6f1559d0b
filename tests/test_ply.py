"""readSplatPly / writeSplatPly (engine/src/splat/SplatPly.cpp:261-342) on files of many shapes: the
library's reader (ply.cpp, through the C ABI) against the reference's own reader on the same bytes.

Covers both binary byte orders and ASCII, every scalar type, list properties and other elements
before and after the vertex table, extra and repeated vertex properties, missing sibling columns
(read as NaN), non-finite positions (dropped), 8- and 16-bit colours, and malformed files (both
readers must refuse them)."""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import pytest

from univeral_3d_reconstruction_system_b200 import api
from univeral_3d_reconstruction_system_b200.types import GROUPS_ORDER, GaussianModel

FMT = {"char": "b", "uchar": "B", "short": "h", "ushort": "H", "int": "i", "uint": "I", "float": "f", "double": "d",
       "int8": "b", "uint8": "B", "int16": "h", "uint16": "H", "int32": "i", "uint32": "I", "float32": "f",
       "float64": "d"}


def ply_bytes(encoding: str, elements) -> bytes:
    """elements: [(name, [(type, name) or ("list", count_type, item_type, name)], rows)]; a row holds one
    value per scalar property and a list per list property."""
    head = ["ply", f"format {encoding} 1.0", "comment made by tests/test_ply.py"]
    for name, props, rows in elements:
        head.append(f"element {name} {len(rows)}")
        for p in props:
            head.append("property " + " ".join(p))
    head.append("end_header")
    out = bytearray(("\n".join(head) + "\n").encode())
    order = ">" if encoding == "binary_big_endian" else "<"
    for _, props, rows in elements:
        for row in rows:
            words = []
            for p, v in zip(props, row):
                if p[0] == "list":
                    if encoding == "ascii":
                        words += [str(len(v))] + [repr(x) for x in v]
                    else:
                        out += struct.pack(order + FMT[p[1]], len(v))
                        for x in v:
                            out += struct.pack(order + FMT[p[2]], x)
                elif encoding == "ascii":
                    words.append(repr(v) if isinstance(v, float) else str(v))
                else:
                    out += struct.pack(order + FMT[p[0]], v)
            if encoding == "ascii":
                out += (" ".join(words) + "\n").encode()
    return bytes(out)


SPLAT = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
         "rot_0", "rot_1", "rot_2", "rot_3"]


def splat_rows(rng, n, names):
    rows = rng.normal(size=(n, len(names))).astype(np.float32).tolist()
    return rows


def read_both(reference, path):
    ours, splat = api.readSplatPly(str(path))
    cnt, flag = C.c_size_t(), C.c_int()
    ok = reference.lib.ref_read_splat_ply(str(path).encode(), None, C.byref(cnt), C.byref(flag))
    theirs = None
    if ok:
        theirs = GaussianModel.zeros(cnt.value)
        v = theirs.view()
        assert reference.lib.ref_read_splat_ply(str(path).encode(), C.byref(v), C.byref(cnt), C.byref(flag)) == 1
    return (ours, splat), (theirs, bool(flag.value) if ok else False)


def assert_same(reference, path):
    (ours, splat), (theirs, their_splat) = read_both(reference, path)
    assert (ours is None) == (theirs is None), (ours, theirs)
    if ours is None:
        return None
    assert splat == their_splat
    assert ours.size() == theirs.size()
    for name in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(ours, name), getattr(theirs, name))  # NaN == NaN here
    return ours, splat


@pytest.mark.parametrize("encoding", ["binary_little_endian", "binary_big_endian", "ascii"])
def test_splat_files_with_extra_elements_and_columns(reference, tmp_path, encoding):
    rng = np.random.default_rng(11)
    names = SPLAT + ["f_rest_0", "f_rest_1"]
    props = [("double" if k % 5 == 0 else "float", nm) for k, nm in enumerate(names)]
    rows = splat_rows(rng, 40, names)
    rows[7][0] = float("nan") if encoding != "ascii" else rows[7][0]  # dropped vertex (binary only)
    rows[9][2] = float("inf") if encoding != "ascii" else rows[9][2]
    face = ("face", [("list", "uchar", "int", "vertex_indices"), ("uchar", "flags")],
            [[[0, 1, 2], 3], [[4, 5, 6, 7], 1], [[], 0]])
    tail = ("camera", [("float", "fx"), ("short", "w")], [[1.5, 640]])
    path = tmp_path / "s.ply"
    path.write_bytes(ply_bytes(encoding, [face, ("vertex", props, rows), tail]))
    got = assert_same(reference, path)
    assert got is not None and got[1]
    assert got[0].size() == (38 if encoding != "ascii" else 40)


def test_missing_and_repeated_columns(reference, tmp_path):
    rng = np.random.default_rng(12)
    names = ["x", "y", "z", "f_dc_0", "opacity", "scale_0", "rot_0", "rot_1", "x"]  # siblings missing; x twice
    props = [("float", nm) for nm in names]
    path = tmp_path / "m.ply"
    path.write_bytes(ply_bytes("binary_little_endian", [("vertex", props, splat_rows(rng, 9, names))]))
    ours, splat = assert_same(reference, path)
    assert splat and np.isnan(ours.colors[:, 1:]).all() and np.isnan(ours.scales[:, 1:]).all()


@pytest.mark.parametrize("ctype,scale", [("uchar", 255), ("ushort", 65535), ("float", 1), ("char", 1)])
def test_point_clouds_with_colour_types(reference, tmp_path, ctype, scale):
    rng = np.random.default_rng(13)
    n = 200
    xyz = rng.normal(size=(n, 3)).astype(np.float32)
    cols = rng.integers(0, min(scale, 127) + 1, size=(n, 3)) if ctype != "float" else rng.uniform(size=(n, 3))
    rows = [[*map(float, p), *(int(c) if ctype != "float" else float(c) for c in cc)] for p, cc in zip(xyz, cols)]
    rows[5][1] = float("inf")
    props = [("float", "x"), ("float", "y"), ("float", "z"), (ctype, "red"), (ctype, "green"), (ctype, "blue")]
    path = tmp_path / "p.ply"
    path.write_bytes(ply_bytes("binary_big_endian", [("vertex", props, rows)]))
    ours, splat = assert_same(reference, path)
    assert not splat and ours.size() == n - 1


def test_uncoloured_point_cloud(reference, tmp_path):
    rng = np.random.default_rng(14)
    rows = rng.normal(size=(50, 3)).tolist()
    path = tmp_path / "g.ply"
    path.write_bytes(ply_bytes("ascii", [("vertex", [("double", "x"), ("double", "y"), ("double", "z")], rows)]))
    ours, splat = assert_same(reference, path)
    assert not splat and ours.size() == 50


def test_large_binary_file_round_trip(reference, tmp_path):
    """The writer's bytes equal the reference writer's; both readers read them back exactly."""
    rng = np.random.default_rng(15)
    n = 150_000  # more than one write block of the writer
    m = GaussianModel(*(rng.normal(size=s).astype(np.float32) for s in ((n, 3), (n, 3), (n, 4), (n,), (n, 3))))
    ours, theirs = tmp_path / "o.ply", tmp_path / "t.ply"
    assert api.writeSplatPly(str(ours), m)
    v = m.view()
    assert reference.lib.ref_write_splat_ply(str(theirs).encode(), C.byref(v)) == 1
    assert ours.read_bytes() == theirs.read_bytes()
    r, splat = assert_same(reference, ours)
    assert splat
    for name in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(r, name), getattr(m, name))


def malformed(tmp_path):
    rng = np.random.default_rng(16)
    good = ply_bytes("binary_little_endian", [("vertex", [("float", nm) for nm in SPLAT], splat_rows(rng, 6, SPLAT))])
    cases = {
        "truncated_body": good[:-10],
        "no_end_header": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\n",
        "bad_magic": b"plx\n" + good[4:],
        "bad_format": good.replace(b"binary_little_endian", b"binary_middle_endian"),
        "bad_type": good.replace(b"property float nx", b"property half nx"),
        "no_vertex": b"ply\nformat ascii 1.0\nelement face 0\nproperty list uchar int i\nend_header\n",
        "no_xyz": ply_bytes("ascii", [("vertex", [("float", "a"), ("float", "b")], [[1.0, 2.0]])]),
        "ascii_word": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\n"
                      b"property float z\nend_header\n1 nan 3\n",
        "truncated_list": ply_bytes("binary_little_endian", [("face", [("list", "uchar", "int", "v")], [[[1, 2, 3]]]),
                                                              ("vertex", [("float", "x")], [])])[:-5],
    }
    for name, data in cases.items():
        p = tmp_path / f"{name}.ply"
        p.write_bytes(data)
        yield name, p


def test_malformed_files_are_refused_by_both(reference, tmp_path):
    for name, path in malformed(tmp_path):
        (ours, _), (theirs, _) = read_both(reference, path)
        assert ours is None and theirs is None, name
        res = api.PlyResult()
        api.readSplatPly(str(path), res)
        assert res.error, name


def test_ascii_numbers(reference, tmp_path):
    """Signs, exponents, leading points and integer columns in ASCII bodies."""
    text = (b"ply\nformat ascii 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty int z\n"
            b"property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n"
            b"+1.5 -2e-3 7 255 0 12\n.25 -.5 -3 1 2 3\n1E2 3.0e+1 0 9 9 9\n   0   0   1   0   0   0   \n")
    path = tmp_path / "a.ply"
    path.write_bytes(text)
    ours, splat = assert_same(reference, path)
    assert not splat and ours.size() == 4


@pytest.mark.parametrize("degree", [1, 3])
def test_sh_coefficients_written_as_f_rest(reference, tmp_path, degree):
    """writeSplatPly with higher-order SH (u3dg_write_splat_ply_sh): the common 3DGS properties
    f_rest_0 .. f_rest_{3K-1} after f_dc_2, channel-major, and both readers still read the same
    Gaussians (they ignore the extra properties, SplatPly.cpp:286-288)."""
    rng = np.random.default_rng(21)
    n, K = 70_000, (degree + 1) ** 2 - 1  # more than one write block
    m = GaussianModel(*(rng.normal(size=s).astype(np.float32) for s in ((n, 3), (n, 3), (n, 4), (n,), (n, 3))))
    sh = rng.normal(size=(n, K, 3)).astype(np.float32)
    path = tmp_path / "sh.ply"
    assert api.writeSplatPlySh(str(path), m, sh, degree)
    data = path.read_bytes()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    props = [l.split()[-1] for l in data[:end].decode().splitlines() if l.startswith("property")]
    rest = [f"f_rest_{i}" for i in range(3 * K)]
    assert props == ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2", *rest, "opacity",
                     "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    rec = np.frombuffer(data[end:], "<f4").reshape(n, len(props))
    np.testing.assert_array_equal(rec[:, 9:9 + 3 * K], sh.transpose(0, 2, 1).reshape(n, 3 * K))
    np.testing.assert_array_equal(rec[:, 6:9], m.colors)
    np.testing.assert_array_equal(rec[:, 9 + 3 * K], m.opacities)
    np.testing.assert_array_equal(rec[:, -4:], m.quats)
    r, splat = assert_same(reference, path)
    assert splat
    for name in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(r, name), getattr(m, name))
    for bad in (0, 4):
        assert not api.writeSplatPlySh(str(tmp_path / "bad.ply"), m, sh, bad)
