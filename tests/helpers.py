"""Shared scene builders and comparison helpers for the tests.

The builders restate the reference test fixtures (tests/test_splat.cpp:18-72) with numpy's
generator instead of std::mt19937; the parity tests feed identical inputs to the GPU path and to
the CPU oracle, so the random stream itself does not need to match the reference's.
"""
from __future__ import annotations

import math

import numpy as np

from univeral_3d_reconstruction_system_b200.types import SH_C0, GaussianModel, RasterSettings, RenderCamera, logit


def make_camera(w: int, h: int, f: float) -> RenderCamera:
    """makeCamera (test_splat.cpp:18-27)."""
    return RenderCamera(w, h, f, f, np.float32(0.5) * np.float32(w - 1), np.float32(0.5) * np.float32(h - 1))


def orbit_camera(w, h, f, angle, radius, height) -> RenderCamera:
    """orbitCamera (test_splat.cpp:30-51): on a circle around the origin, looking at it."""
    c = make_camera(w, h, f)
    C = np.array([radius * math.sin(angle), height, -radius * math.cos(angle)], np.float32)
    zf = -C / np.linalg.norm(C)
    down = np.array([0, 1, 0], np.float32)
    x = np.cross(down, zf)
    x = x / -np.linalg.norm(x)
    y = np.cross(zf, x)
    R = np.stack([x, y, zf]).astype(np.float32)
    t = -(R @ C)
    return RenderCamera(w, h, c.fx, c.fy, c.cx, c.cy, R, t.astype(np.float32))


def random_model(n, rng: np.random.Generator, spread, zc, min_scale, max_scale) -> GaussianModel:
    """randomModel (test_splat.cpp:53-72)."""
    m = GaussianModel.zeros(n)
    for i in range(n):
        m.means[i] = [rng.uniform(-1, 1) * spread, rng.uniform(-1, 1) * spread * 0.8, zc + rng.uniform(-1, 1) * spread]
        for k in range(3):
            m.scales[i, k] = math.log(min_scale + (max_scale - min_scale) * rng.uniform())
            m.colors[i, k] = (0.15 + 0.7 * rng.uniform() - 0.5) / SH_C0
        m.quats[i] = [rng.uniform(-1, 1) + (1.5 if k == 0 else 0.0) for k in range(4)]
        m.opacities[i] = logit(0.25 + 0.5 * rng.uniform())
    return m


def fd_setup(seed: int = 7):
    """The finite-difference scene of splat_gradients_match_finite_differences (test_splat.cpp:110-129)."""
    rng = np.random.default_rng(seed)
    model = random_model(8, rng, 0.6, 3.0, 0.08, 0.3)
    cam = make_camera(56, 44, 45.0)
    a = 0.15
    cam.R = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]], np.float32)
    cam.t = np.array([0.1, -0.05, 0.2], np.float32)
    st = RasterSettings(tile_size=64, min_alpha=0.0, min_transmittance=0.0, background=(0.1, 0.2, 0.3))
    return model, cam, st, rng


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def grad_close(a, b, rel=1e-4, floor_frac=1e-2):
    """Per-element check |a - b| <= rel * max(|b|, floor) with floor = floor_frac * max|b| of the group.

    A per-Gaussian gradient is a float sum over all pixels of all tiles it touches; the reference adds
    pixel after pixel, the GPU adds a tree per tile. Where the terms nearly cancel, the two float sums
    legitimately differ by many ulps of the (small) result, so elements below 1% of the group's largest
    magnitude are compared on that 1% scale. Returns (ok, worst ratio)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    if b.size == 0:
        return True, 0.0
    floor = floor_frac * max(float(np.max(np.abs(b))), 1e-30)
    ratio = np.abs(a - b) / (rel * np.maximum(np.abs(b), floor))
    worst = float(np.max(ratio))
    return worst <= 1.0, worst
