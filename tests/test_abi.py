"""The C ABI library without a GPU: it loads, exports every entry point include/u3dg.h declares,
its host-only entry points (defaults, PLY I/O with the host-side initGaussiansFromPoints for point
clouds) match the reference, and
entry points that need a GPU fail with a status code instead of crashing when there is none."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from univeral_3d_reconstruction_system_b200 import _abi, _lib, api
from univeral_3d_reconstruction_system_b200.types import GROUPS_ORDER, GaussianModel, TrainOptions

HEADER = Path(__file__).resolve().parents[1] / "include" / "u3dg.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(u3dg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) > 40
    for name in names:
        assert hasattr(lib, name), name
    # The Python binding declares a signature for each of them.
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert lib.u3dg_abi_version() == 1


def test_struct_layouts_match_header_sizes():
    # Sizes of the boundary structs (x86-64, natural alignment).
    assert C.sizeof(_abi.Camera) == 4 * (2 + 4 + 9 + 3)
    assert C.sizeof(_abi.RasterSettings) == 4 * 8
    assert C.sizeof(_abi.TrainOptions) == 4 * (3 + 5 + 3 + 4 + 1 + 1) + C.sizeof(_abi.RasterSettings)
    assert C.sizeof(_abi.TrainStats) == 24  # int, 2 floats, padding, uint64
    assert C.sizeof(_abi.ModelView) == 6 * 8


def test_option_defaults_match_reference(reference):
    lib = _lib.load()
    for it in (0, 1, 99, 1500, 6000, 7000):
        o = _abi.TrainOptions()
        if it:
            lib.u3dg_train_options_for_iterations(it, C.byref(o))
        else:
            lib.u3dg_train_options_default(C.byref(o))
        r = _abi.TrainOptions()
        reference.lib.ref_options_for_iterations(it, C.byref(r))
        assert TrainOptions.from_struct(o).struct_tuple() == TrainOptions.from_struct(r).struct_tuple()
        if it:
            assert TrainOptions.for_iterations(it).struct_tuple() == TrainOptions.from_struct(o).struct_tuple()


def test_ply_round_trip_and_reference_compatibility(reference, tmp_path):
    """ply_round_trip (test_splat.cpp:270-298): our writer / reader against the reference's."""
    rng = np.random.default_rng(5)
    n = 50
    m = GaussianModel(*(rng.normal(size=s).astype(np.float32) for s in ((n, 3), (n, 3), (n, 4), (n,), (n, 3))))
    ours, theirs = tmp_path / "ours.ply", tmp_path / "theirs.ply"
    assert api.writeSplatPly(str(ours), m)
    v = m.view()
    assert reference.lib.ref_write_splat_ply(str(theirs).encode(), C.byref(v)) == 1
    assert ours.read_bytes() == theirs.read_bytes()
    r, is_splat = api.readSplatPly(str(theirs))
    assert is_splat and r.size() == n
    for name in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(r, name), getattr(m, name))
    # A plain point cloud becomes opaque Gaussians (SplatPly.cpp:301-321) through the host-side
    # initGaussiansFromPoints (hash-grid 3-NN); compare with the reference, on 4 points and on a
    # clustered cloud whose hash-grid buckets have many members and repeated keys.
    rng2 = np.random.default_rng(9)
    clustered = (rng2.normal(size=(3000, 3)) * rng2.choice([0.01, 1.0], size=(3000, 1))).astype(np.float32)
    for k, xyz in enumerate((np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32), clustered)):
        pts = tmp_path / f"points{k}.ply"
        cols = rng2.integers(0, 256, (len(xyz), 3))
        lines = ["ply", "format ascii 1.0", f"element vertex {len(xyz)}", "property float x", "property float y",
                 "property float z", "property uchar red", "property uchar green", "property uchar blue",
                 "end_header"]
        lines += [f"{x!r} {y!r} {z!r} {r_} {g_} {b_}" for (x, y, z), (r_, g_, b_) in
                  zip(xyz.tolist(), cols.tolist())]
        pts.write_text("\n".join(lines) + "\n")
        r, is_splat = api.readSplatPly(str(pts))
        assert not is_splat and r.size() == len(xyz)
        cnt, flag = C.c_size_t(), C.c_int()
        out = GaussianModel.zeros(len(xyz))
        ov = out.view()
        assert reference.lib.ref_read_splat_ply(str(pts).encode(), C.byref(ov), C.byref(cnt), C.byref(flag)) == 1
        for name in GROUPS_ORDER:
            np.testing.assert_array_equal(getattr(r, name), getattr(out, name))
    res = api.PlyResult()
    assert api.readSplatPly(str(tmp_path / "missing.ply"), res) == (None, False)
    assert "Cannot open" in res.error


def test_gpu_entry_points_fail_cleanly_without_a_device():
    if _lib.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(api.U3dgError) as e:
        api.Rasterizer()
    assert e.value.status == _abi.ERR_NO_DEVICE
    m = GaussianModel.zeros(3)
    with pytest.raises(api.U3dgError):
        api.Trainer(m, [], 1.0, TrainOptions())
    with pytest.raises(api.U3dgError):
        api.psnr(np.zeros(3, np.float32), np.zeros(3, np.float32))
    with pytest.raises(api.U3dgError) as e:
        api.initGaussiansFromPoints(np.zeros((4, 3), np.float32))
    assert e.value.status == _abi.ERR_NO_DEVICE


def test_invalid_arguments_are_rejected():
    lib = _lib.load()
    assert lib.u3dg_trainer_step(None, 1) == _abi.ERR_INVALID_ARG
    assert b"NULL" in lib.u3dg_last_error()
    assert lib.u3dg_init_gaussians_from_points(None, None, 5, None) == _abi.ERR_INVALID_ARG
    assert lib.u3dg_read_splat_ply(b"/nonexistent/x.ply", None, 0, C.byref(C.c_size_t()), None) == _abi.ERR_IO
