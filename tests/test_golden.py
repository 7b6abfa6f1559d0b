"""The CPU oracle against golden outputs of the reference (tests/golden/golden.npz, written by
tests/golden/make_golden.py from the reference's own sources, one worker thread).

With one worker thread the reference is deterministic, and the oracle keeps its operation order, so
every comparison here is bit-exact (==), except the training run's evaluatePsnr, whose double sum
the oracle also reproduces exactly.
"""
from pathlib import Path

import numpy as np
import pytest

from univeral_3d_reconstruction_system_b200.types import (GROUPS_ORDER, GaussianModel, RasterSettings, RenderCamera,
                                                          TrainImage, TrainOptions)

G = np.load(Path(__file__).resolve().parent / "golden" / "golden.npz")


def model(prefix):
    return GaussianModel(*(G[f"{prefix}_{n}"] for n in GROUPS_ORDER))


def cam(key):
    a = G[key]
    return RenderCamera(int(a[0]), int(a[1]), float(a[2]), float(a[3]), float(a[4]), float(a[5]),
                        a[6:15].astype(np.float32), a[15:18].astype(np.float32))


def assert_grads_equal(g, prefix):
    for n in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(g, n), G[f"{prefix}_{n}"], err_msg=n)


def test_fd_scene_forward_backward(oracle):
    m = model("fd_model")
    st = RasterSettings(tile_size=64, min_alpha=0.0, min_transmittance=0.0, background=(0.1, 0.2, 0.3))
    r = oracle.raster(1)
    np.testing.assert_array_equal(r.forward(m, cam("fd_cam"), st), G["fd_rgb"])
    np.testing.assert_array_equal(r.projection()["radius"], G["fd_radii"])
    g, ndc = r.backward(G["fd_w"])
    assert_grads_equal(g, "fd_grad")
    np.testing.assert_array_equal(ndc, G["fd_ndc"])


@pytest.mark.parametrize("k", [0, 1])
def test_orbit_scene_forward_backward(oracle, k):
    m = model("orbit_model")
    r = oracle.raster(3)
    np.testing.assert_array_equal(r.forward(m, cam(f"orbit{k}_cam"), RasterSettings()), G[f"orbit{k}_rgb"])
    np.testing.assert_array_equal(r.projection()["radius"], G[f"orbit{k}_radii"])
    g, ndc = r.backward(G[f"orbit{k}_w"])
    assert_grads_equal(g, f"orbit{k}_grad")
    np.testing.assert_array_equal(ndc, G[f"orbit{k}_ndc"])


@pytest.mark.parametrize("k", [0, 1])
def test_loss(oracle, k):
    render, target = G[f"loss{k}_in"]
    W, H, lam = G[f"loss{k}_meta"]
    v, grad = oracle.photometric_loss(render, target, int(W), int(H), float(lam))
    np.testing.assert_array_equal(np.array([v.total, v.l1, v.ssim], np.float32), G[f"loss{k}_value"])
    np.testing.assert_array_equal(grad, G[f"loss{k}_grad"])


def test_training_run(oracle):
    imgs = [TrainImage(cam_from(c), im) for c, im in zip(G["train_cams"], G["train_images"])]
    init = oracle.init_from_points(G["train_xyz"], np.full_like(G["train_xyz"], 0.5))
    for n in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(init, n), G[f"train_init_{n}"])
    opt = TrainOptions.for_iterations(150)
    opt.max_gaussians = 200
    t = oracle.trainer(init, imgs, 4.4, opt, threads=4)
    t.step(150)
    s = t.stats()
    np.testing.assert_array_equal(np.array([s.iteration, s.loss, s.psnr, s.gaussians], np.float64),
                                  G["train_stats"])
    fin = t.model()
    for n in GROUPS_ORDER:
        np.testing.assert_array_equal(getattr(fin, n), G[f"train_final_{n}"], err_msg=n)
    assert np.float32(t.evaluate_psnr()) == G["train_eval_psnr"][0]


def cam_from(a):
    return RenderCamera(int(a[0]), int(a[1]), float(a[2]), float(a[3]), float(a[4]), float(a[5]),
                        a[6:15].astype(np.float32), a[15:18].astype(np.float32))
