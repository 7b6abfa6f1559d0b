"""The CPU oracle against the reference itself (oracle/_ref, the reference's own sources), live.

Covers paths the golden fixtures do not: several tile sizes and cut-off settings, degenerate and
off-screen Gaussians, the greedy densification budget, opacity reset with the prune-after-reset rule,
and Adam over several steps. With one reference thread every comparison is bit-exact.
"""
import numpy as np
import pytest

from helpers import make_camera, orbit_camera, random_model
from univeral_3d_reconstruction_system_b200.types import (GROUPS_ORDER, GaussianModel, RasterSettings, TrainImage,
                                                          TrainOptions, logit)


def _equal_models(a, b):
    assert a.size() == b.size()
    for n in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(a, n), getattr(b, n), err_msg=n)


@pytest.mark.parametrize("tile,min_alpha,min_t", [(16, 1 / 255, 1e-4), (8, 1 / 255, 1e-4), (32, 0.0, 0.0),
                                                  (64, 1 / 255, 0.0)])
def test_raster_matches_reference(oracle, reference, tile, min_alpha, min_t):
    rng = np.random.default_rng(tile)
    m = random_model(300, rng, 1.2, 0.0, 0.01, 0.3)
    # Degenerate and extreme members: zero quaternion, behind the camera, far off-screen, huge.
    m.quats[0] = 0
    m.means[1] = [0, 0, -10]
    m.means[2] = [40, 0, 0]
    m.scales[3] = np.log(5.0)
    st = RasterSettings(tile_size=tile, min_alpha=float(np.float32(min_alpha)), min_transmittance=min_t,
                        background=(0.05, 0.1, 0.2))
    for ang in (0.0, 1.3, 4.0):
        cam = orbit_camera(90, 70, 75.0, ang, 3.0, 0.4)
        o, r = oracle.raster(4), reference.raster(1)
        np.testing.assert_array_equal(o.forward(m, cam, st), r.forward(m, cam, st))
        np.testing.assert_array_equal(o.projection()["radius"], r.radii())
        w = rng.uniform(-1, 1, (cam.height, cam.width, 3)).astype(np.float32)
        og, ondc = o.backward(w)
        rg, rndc = r.backward(w)
        _equal_models(og, rg)
        np.testing.assert_array_equal(ondc, rndc)


@pytest.mark.parametrize("W,H,lam", [(1, 1, 0.2), (5, 3, 0.2), (64, 48, 0.2), (33, 70, 0.7), (50, 20, 0.0)])
def test_loss_matches_reference(oracle, reference, W, H, lam):
    rng = np.random.default_rng(W * H)
    t = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
    r = np.clip(t + rng.normal(0, 0.1, t.shape), 0, 1).astype(np.float32)
    ov, og = oracle.photometric_loss(r, t, W, H, lam)
    rv, rg = reference.photometric_loss(r, t, W, H, lam, threads=1)
    assert (ov.total, ov.l1, ov.ssim) == (rv.total, rv.l1, rv.ssim)
    np.testing.assert_array_equal(og, rg)
    assert oracle.psnr(r, t) == reference.psnr(r, t)
    assert oracle.psnr(t, t) == reference.psnr(t, t) == 99.0


def test_init_and_options_match_reference(oracle, reference):
    rng = np.random.default_rng(0)
    for n in (1, 2, 3, 50, 3000):
        xyz = rng.normal(size=(n, 3)).astype(np.float32)
        rgb = rng.uniform(size=(n, 3)).astype(np.float32)
        _equal_models(oracle.init_from_points(xyz, rgb), reference.init_from_points(xyz, rgb))
    for it in (1, 10, 1500, 4000, 6000, 7000, 30000):
        assert TrainOptions.for_iterations(it).struct_tuple() == _ref_options(reference, it)


def _ref_options(reference, it):
    import ctypes as C

    from univeral_3d_reconstruction_system_b200 import _abi
    o = _abi.TrainOptions()
    reference.lib.ref_options_for_iterations(it, C.byref(o))
    return TrainOptions.from_struct(o).struct_tuple()


def _scene(seed, n_truth=150, views=8, w=48, h=36):
    rng = np.random.default_rng(seed)
    truth = random_model(n_truth, rng, 1.0, 0.0, 0.04, 0.12)
    truth.opacities[:] = logit(0.8)
    return truth, rng, w, h, views


@pytest.mark.parametrize("case", ["budget", "reset"])
def test_trainer_matches_reference(oracle, reference, case):
    truth, rng, w, h, views = _scene(11 if case == "budget" else 12)
    images = []
    for k in range(views):
        cam = orbit_camera(w, h, 40.0, 6.2831853 * k / views, 4.0, -0.6 + 0.2 * (k % 3))
        images.append(TrainImage(cam, TrainImage.quantize(reference.raster(1).forward(truth, cam, RasterSettings()))))
    xyz = np.stack([truth.means[i] + rng.normal(0, 0.05, 3) for i in range(0, truth.size(), 2)]).astype(np.float32)
    init = reference.init_from_points(xyz, np.full_like(xyz, 0.5))
    if case == "budget":
        # A tight cap: the greedy budget rejects splits and later still accepts a clone.
        opt = TrainOptions.for_iterations(300).replace(max_gaussians=init.size() + 7, densify_grad_threshold=5e-5)
    else:
        # Opacity reset inside the refinement window, then pruning of large Gaussians after it.
        opt = TrainOptions.for_iterations(400).replace(opacity_reset_interval=200, refine_stop=350,
                                                       refine_start=50, densify_grad_threshold=1e-4)
    o = oracle.trainer(init, images, 1.0 if case == "reset" else 4.4, opt, threads=4)
    r = reference.trainer(init, images, 1.0 if case == "reset" else 4.4, opt, threads=1)
    for _ in range(4):
        o.step(opt.iterations // 4)
        r.step(opt.iterations // 4)
        so, sr = o.stats(), r.stats()
        assert (so.iteration, so.loss, so.psnr, so.gaussians) == (sr.iteration, sr.loss, sr.psnr, sr.gaussians)
        _equal_models(o.model(), r.model())
    assert o.evaluate_psnr() == r.evaluate_psnr()


def test_adam_matches_reference(oracle, reference):
    import ctypes as C
    rng = np.random.default_rng(9)
    n = 500
    p = GaussianModel(*(rng.normal(size=s).astype(np.float32) for s in ((n, 3), (n, 3), (n, 4), (n,), (n, 3))))
    po = p.copy()
    m, v = GaussianModel.zeros(n), GaussianModel.zeros(n)
    h = reference.lib.ref_adam_create(n, 1)
    lr = TrainOptions().lr
    try:
        for step in range(1, 8):
            g = GaussianModel(*(rng.normal(size=a.shape).astype(np.float32) * 0.1 for a in
                                (p.means, p.scales, p.quats, p.opacities, p.colors)))
            pv, gv = p.view(), g.view()
            lrs = lr.struct()
            reference.lib.ref_adam_step(h, C.byref(pv), C.byref(gv), C.byref(lrs))
            oracle.adam_step(po, g, m, v, step, lr)
            np.testing.assert_array_equal(p.flat(), po.flat())
    finally:
        reference.lib.ref_adam_destroy(h)


def test_closed_form_projection_oracle(oracle):
    """splat_projection_matches_closed_form (test_splat.cpp:153-191) on the oracle."""
    sx, sy, angle = 0.05, 0.12, 0.6
    m = GaussianModel(np.array([[0, 0, 3]], np.float32), np.log(np.array([[sx, sy, 0.02]], np.float32)),
                      np.array([[np.cos(angle / 2), 0, 0, np.sin(angle / 2)]], np.float32),
                      np.array([logit(0.5)], np.float32), np.full((1, 3), 0.5 / 0.28209479177387814, np.float32))
    rgb = oracle.render(m, make_camera(201, 201, 300.0), RasterSettings(min_alpha=0.0, min_transmittance=0.0))
    v = rgb[..., 0].astype(np.float64)
    ys, xs = np.mgrid[0:201, 0:201]
    wsum = v.sum()
    assert abs((v * xs).sum() / wsum - 100) < 0.01 and abs((v * ys).sum() / wsum - 100) < 0.01


def _crop_models():
    rng = np.random.default_rng(31)
    out = []
    for n, spread in ((5000, 1.0), (777, 3.0), (1, 1.0)):
        means = (rng.normal(size=(n, 3)) * spread).astype(np.float32)
        means[: n // 50] *= 20.0  # far floaters
        m = GaussianModel(means, rng.normal(-4, 1, (n, 3)).astype(np.float32), rng.normal(size=(n, 4)).astype(np.float32),
                          rng.normal(-0.5, 2.0, n).astype(np.float32), rng.normal(size=(n, 3)).astype(np.float32))
        out.append(m)
    faint = out[1].copy()
    faint.opacities[:] = -9.0  # nothing 0.3 opaque: the boxes fall back to all centres
    out.append(faint)
    out.append(GaussianModel.zeros(0))
    return out


def test_crop_matches_reference(oracle, reference):
    """cropModel, suggestCropBox and modelBounds (Crop.cpp:12-62): the oracle's restatement against the
    reference, bit for bit, on models with floaters, an all-faint model, one Gaussian and none."""
    for m in _crop_models():
        for lo, hi, margin in ((0.05, 0.95, 0.1), (0.0, 1.0, 0.0), (0.2, 0.6, 0.5)):
            a, b = oracle.suggest_crop_box(m, lo, hi, margin), reference.suggest_crop_box(m, lo, hi, margin)
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1], b[1])
        a, b = oracle.model_bounds(m), reference.model_bounds(m)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        box = oracle.suggest_crop_box(m)
        for floor in (0.0, 0.3, 0.7):
            _equal_models(oracle.crop_model(m, box, floor), reference.crop_model(m, box, floor))
