"""One High-preset step against the CPU oracle at full size: 640x480, 300k and 250k Gaussians.

The unit-boundary rasterizer runs the trainers' configuration (tile culling on, 8x8 forward CTAs,
persistent heaviest-first backward) on the High scene's first view, and the oracle (the reference's
Rasterizer restated, Rasterizer.cpp:137-545) runs the same projection, binning, compositing and
backward. Checked per step, as one training step computes them:
  - tile lists and their depth order: bit-exact against binTiles on identical projected records
    (the 300k depth sort and ~2.5M intersections), and with culling on, every tile's list is an
    order-preserving subsequence of the reference's list for that tile;
  - image within 1e-5 absolute per channel, final transmittance within 1e-5, contributor counts exact
    (with culling, a count indexes the culled list: it must name the same last contributor);
  - per-parameter gradients of the L1 + 0.2 D-SSIM loss against the view's target within 1e-4
    relative (floor: 1% of the group's largest magnitude) for at least 99.99% of the elements, and
    every element within 1e-3, and the same for the NDC densification statistic. At this size a few
    near-cancelling sums of tens of thousands of pixels round past 1e-4 in ANY other summation order:
    the reference's own backward with all host threads (its default; CAS atomics in arrival order)
    lands up to 1.6e-4 from its one-thread result (the oracle) on the scales and quaternions of the
    250k model, a different amount on every run; the test prints that spread beside the GPU's. The
    quaternion gradients of the isotropic 300k model are zero in exact arithmetic and rounding noise
    on every side: they are checked to be negligible instead.
Models: the bench workload (initGaussiansFromPoints of every true centre plus 50k re-samples:
isotropic, opacity 0.1) and the ground truth itself (anisotropic, opacity 0.3-1)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from univeral_3d_reconstruction_system_b200.scenes import dense_init_points, make_scene
from univeral_3d_reconstruction_system_b200.types import RasterSettings, TrainImage

pytestmark = pytest.mark.gpu

GROUPS = ("means", "scales", "quats", "opacities", "colors")
THREADS = max(1, min(os.cpu_count() or 1, 32))


@pytest.fixture(scope="module")
def high(oracle):
    sc = make_scene("high", 0)
    st = RasterSettings()
    cam = sc.cameras[0]
    target = TrainImage.quantize(oracle.render(sc.truth, cam, st, sc.sh_rest, 3, threads=THREADS))
    return sc, cam, target.astype(np.float32) / np.float32(255.0)


@pytest.fixture(scope="module", params=["bench-300k", "truth-250k"])
def model(request, high, oracle):
    sc = high[0]
    if request.param == "truth-250k":
        return sc.truth
    xyz, rgb = dense_init_points(sc, 300_000)
    return oracle.init_from_points(xyz, rgb)


def _subsequence_lists(off, lst, roff, rlst, n):
    """Every tile's list in (off, lst) is an order-preserving subsequence of its list in (roff, rlst);
    returns the position in rlst of every entry of lst."""
    tiles = len(roff) - 1
    rt = np.repeat(np.arange(tiles, dtype=np.int64), np.diff(roff))
    rkey = rt * n + rlst.astype(np.int64)  # unique per (tile, Gaussian), increasing position in rlst
    order = np.argsort(rkey, kind="stable")
    t = np.repeat(np.arange(tiles, dtype=np.int64), np.diff(off))
    key = t * n + lst.astype(np.int64)
    idx = np.searchsorted(rkey[order], key)
    assert np.all(idx < len(rkey)) and np.array_equal(rkey[order][np.minimum(idx, len(rkey) - 1)], key), \
        "a culled list holds an entry the reference's list does not"
    pos = order[idx]  # position of each culled entry in the reference list
    same_tile = t[1:] == t[:-1]
    assert np.all(pos[1:][same_tile] > pos[:-1][same_tile]), "culled lists changed the depth order"
    return pos


def _culled_counts_as_reference(nc, off, pos, roff, width, height, tile=16):
    """Contributor counts over culled lists (an index into the pixel's tile's culled list) expressed as
    counts over the reference's lists: the last contributor's position in the reference list + 1."""
    ys, xs = np.mgrid[0:height, 0:width]
    t = ((ys // tile) * ((width + tile - 1) // tile) + xs // tile).reshape(-1)
    nc = nc.reshape(-1).astype(np.int64)
    last = off[t].astype(np.int64) + nc - 1  # global index of the last contributor in lst
    out = np.zeros_like(nc)
    has = nc > 0
    out[has] = pos[last[has]] - roff[t[has]] + 1
    return out


def _ratios(a, b):
    """|a - b| / (1e-4 max(|b|, 1% of the group's largest |b|)), per element (helpers.grad_close's measure)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    floor = 1e-2 * max(float(np.max(np.abs(b))), 1e-30)
    return np.abs(a - b) / (1e-4 * np.maximum(np.abs(b), floor))


def _reference_spread(reference, model, cam, st, dl, og, ondc):
    """Per group: (worst ratio, fraction of ratios > 1) of the reference's multithreaded backward against
    the oracle (which equals the reference run with one thread)."""
    r = reference.raster(THREADS)
    r.forward(model, cam, st)
    rg, rndc = r.backward(dl)
    out = {name: _ratios(getattr(rg, name), getattr(og, name)) for name in GROUPS}
    out["ndc"] = _ratios(rndc, ondc)
    return {k: (float(v.max()), float(np.mean(v > 1.0))) for k, v in out.items()}


def test_high_step_matches_oracle(u3dg, oracle, reference, high, model):
    sc, cam, target = high
    st = RasterSettings()
    n = model.size()
    o = oracle.raster(THREADS)
    ref_img = o.forward(model, cam, st)
    ref_off, ref_list = o.tiles()
    ref_ft, ref_nc = o.pixel_state()
    assert len(ref_list) > 1_000_000

    # Tile lists bit-exact on identical projected records (the full-size depth sort and bucketing).
    p = o.projection()
    tx, ty = (cam.width + 15) // 16, (cam.height + 15) // 16
    g_off, g_list = u3dg.binTiles(p["depth"], p["radius"], p["rect"], tx, ty)
    np.testing.assert_array_equal(g_off, ref_off)
    np.testing.assert_array_equal(g_list, ref_list)

    # The trainers' configuration: culled lists, 8x8 forward CTAs.
    r = u3dg.Rasterizer()
    r.set_tile_culling(True)
    img = r.forward(model, cam, st)
    assert float(np.max(np.abs(img - ref_img))) <= 1e-5
    ft, nc = r.pixel_state()
    assert float(np.max(np.abs(ft - ref_ft))) <= 1e-5
    off, lst = r.tiles()
    assert len(lst) < len(ref_list)
    pos = _subsequence_lists(off, lst, ref_off, ref_list, n)
    # A pixel's contributor count indexes its tile's (culled) list: the same last contributor.
    np.testing.assert_array_equal(_culled_counts_as_reference(nc, off, pos, ref_off, cam.width, cam.height), ref_nc)

    # The step's loss gradient (oracle's loss on the oracle's image), through both backward passes.
    _, dl = oracle.photometric_loss(ref_img, target, cam.width, cam.height, 0.2)
    dl = dl.reshape(ref_img.shape)
    ndc = np.zeros(n, np.float32)
    g = r.backward(model, dl, None, ndc)
    og, ondc = o.backward(dl)
    spread = _reference_spread(reference, model, cam, st, dl, og, ondc)
    isotropic = bool(np.all(model.scales == model.scales[:, :1]) and np.all(model.quats[:, 1:] == 0))
    for name in GROUPS + ("ndc",):
        got = _ratios(ndc, ondc) if name == "ndc" else _ratios(getattr(g, name), getattr(og, name))
        worst, frac = float(got.max()), float(np.mean(got > 1.0))
        ref_worst, ref_frac = spread[name]
        print(f"{name}: worst {worst:.3g} (reference threads {ref_worst:.3g}), beyond 1e-4: {frac:.2e} "
              f"(reference threads {ref_frac:.2e})")
        if name == "quats" and isotropic:
            scale = max(float(np.max(np.abs(og.means))), float(np.max(np.abs(og.scales))))
            assert float(np.max(np.abs(g.quats))) <= 1e-3 * scale
            assert float(np.max(np.abs(og.quats))) <= 1e-3 * scale
            continue
        assert frac <= 1e-4 and worst <= 10.0, (name, worst, frac)

    # Culling off at the unit boundary: the reference's own lists and contributor counts.
    r.set_tile_culling(False)
    img2 = r.forward(model, cam, st)
    np.testing.assert_array_equal(img2, img)
    off2, lst2 = r.tiles()
    np.testing.assert_array_equal(off2, ref_off)
    np.testing.assert_array_equal(lst2, ref_list)
    ft2, nc2 = r.pixel_state()
    np.testing.assert_array_equal(nc2, ref_nc)
    np.testing.assert_array_equal(ft2, ft)
