"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs the reference splat core (oracle/_ref/libu3dref.so, built by oracle/Makefile from the
reference's own sources) with one worker thread on small seeded inputs, and stores inputs and outputs
together in golden.npz. tests/test_golden.py checks the CPU oracle against these outputs, so the oracle
stays pinned to the reference even where the reference tree is not available.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from helpers import fd_setup, orbit_camera, random_model  # noqa: E402
from oracle.binding import Reference  # noqa: E402
from univeral_3d_reconstruction_system_b200.types import (GROUPS_ORDER, RasterSettings, TrainImage,  # noqa: E402
                                                          TrainOptions, logit)

OUT = Path(__file__).resolve().parent / "golden.npz"


def model_arrays(prefix, m):
    return {f"{prefix}_{name}": getattr(m, name) for name in GROUPS_ORDER}


def cam_array(c):
    return np.concatenate([[c.width, c.height, c.fx, c.fy, c.cx, c.cy], np.asarray(c.R).ravel(),
                           np.asarray(c.t).ravel()]).astype(np.float64)


def main():
    ref = Reference()
    out = {}
    # 1. The finite-difference scene (tile 64, no cut-offs, background): forward + backward.
    model, cam, st, rng = fd_setup()
    r = ref.raster(1)
    rgb = r.forward(model, cam, st)
    w = rng.uniform(-1, 1, rgb.shape).astype(np.float32)
    g, ndc = r.backward(w)
    out.update(model_arrays("fd_model", model))
    out.update(fd_cam=cam_array(cam), fd_w=w, fd_rgb=rgb, fd_ndc=ndc, fd_radii=r.radii())
    out.update(model_arrays("fd_grad", g))
    # 2. A 400-Gaussian orbit scene with default settings (1/255 and 1e-4 cut-offs), two views.
    rng = np.random.default_rng(21)
    model = random_model(400, rng, 1.0, 0.0, 0.02, 0.15)
    out.update(model_arrays("orbit_model", model))
    for k, ang in enumerate((0.3, 2.1)):
        cam = orbit_camera(80, 60, 70.0, ang, 3.5, -0.5)
        r = ref.raster(1)
        rgb = r.forward(model, cam, RasterSettings())
        w = rng.uniform(-1, 1, rgb.shape).astype(np.float32)
        g, ndc = r.backward(w)
        out[f"orbit{k}_cam"] = cam_array(cam)
        out[f"orbit{k}_w"] = w
        out[f"orbit{k}_rgb"] = rgb
        out[f"orbit{k}_radii"] = r.radii()
        out[f"orbit{k}_ndc"] = ndc
        out.update(model_arrays(f"orbit{k}_grad", g))
    # 3. Loss on random images: lambda 0.2 and pure D-SSIM.
    rng = np.random.default_rng(3)
    for k, (W, H, lam) in enumerate(((21, 17, 1.0), (40, 31, 0.2))):
        target = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
        render = (0.5 * target + 0.5 * rng.uniform(0, 1, (H, W, 3))).astype(np.float32)
        v, grad = ref.photometric_loss(render, target, W, H, lam, threads=1)
        out[f"loss{k}_in"] = np.stack([render, target])
        out[f"loss{k}_meta"] = np.array([W, H, lam], np.float64)
        out[f"loss{k}_value"] = np.array([v.total, v.l1, v.ssim], np.float32)
        out[f"loss{k}_grad"] = grad
    # 4. A short training run through one densification: 16 views of 120 Gaussians.
    rng = np.random.default_rng(11)
    truth = random_model(120, rng, 1.0, 0.0, 0.04, 0.12)
    truth.opacities[:] = logit(0.8)
    images = []
    for k in range(8):
        cam = orbit_camera(48, 36, 40.0, 6.2831853 * k / 8.0, 4.0, -0.6 + 0.2 * (k % 3))
        images.append(TrainImage(cam, TrainImage.quantize(ref.raster(1).forward(truth, cam, RasterSettings()))))
    xyz = np.stack([truth.means[i] + rng.normal(0, 0.05, 3) for i in range(0, 120, 2)]).astype(np.float32)
    init = ref.init_from_points(xyz, np.full_like(xyz, 0.5))
    opt = TrainOptions.for_iterations(150)
    opt.max_gaussians = 200
    t = ref.trainer(init, images, 4.4, opt, threads=1)
    t.step(150)
    s = t.stats()
    final = t.model()
    out["train_images"] = np.stack([im.rgb for im in images])
    out["train_cams"] = np.stack([cam_array(im.camera) for im in images])
    out["train_xyz"] = xyz
    out.update(model_arrays("train_init", init))
    out.update(model_arrays("train_final", final))
    out["train_stats"] = np.array([s.iteration, s.loss, s.psnr, s.gaussians], np.float64)
    out["train_eval_psnr"] = np.array([t.evaluate_psnr()], np.float32)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
