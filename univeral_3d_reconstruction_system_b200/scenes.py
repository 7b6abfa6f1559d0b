"""Seeded synthetic scenes for the trainer workloads (host-side input generation).

The reference publishes no dataset; its own tests generate seeded synthetic scenes
(tests/test_splat.cpp:30-72,227-268). The workloads here follow the same pattern at the sizes of
the Fast / Balanced / High presets (engine/src/pipeline/Reconstructor.cpp:25-33):

  ground truth  centres U[-1,1]^3, log-scales N(-4, 0.5), random unit quaternions,
                opacity U(0.3, 1), SH degree 3: DC colour U(0,1) (stored as the coefficient
                (c - 0.5) / C0), higher-order coefficients N(0, 0.05)
  cameras       pinhole, looking at the origin (OpenCV convention, world y down), radius 3
  init points   a random subset of the true centres + N(0, 0.02) noise, coloured with the
                ground truth's DC colour (what a coloured SfM point cloud would give)
  extent        1.1 x the largest camera distance from the mean camera centre
                (Reconstructor.cpp:286-296)

Everything is drawn from numpy's PCG64 generator in a fixed order, so a (config, seed) pair gives
the same scene on every machine. Rendering the ground truth needs a renderer (the GPU library's
u3dg_render_sh, or the CPU oracle in tests), so it is a separate step (`render_targets`).
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np

from .types import SH_C0, GaussianModel, RenderCamera, TrainImage, TrainOptions


@dataclass
class SceneSpec:
    name: str
    gt_count: int
    views: int
    width: int
    height: int
    focal: float
    layout: str  # "ring", "two_rings", "hemisphere"
    init_count: int
    iterations: int
    max_gaussians: int
    sh_degree: int = 3
    radius: float = 3.0
    roll_deg: float = 0.0
    init_noise: float = 0.02
    opacity_reset_at: int = 0  # explicit reset iteration (0 = the forIterations schedule)


PRESETS = {
    # The Fast / Balanced / High benchmark presets.
    "fast": SceneSpec("fast", 30_000, 32, 320, 240, 300.0, "ring", 5_000, 2000, 80_000),
    "balanced": SceneSpec("balanced", 100_000, 80, 480, 360, 450.0, "two_rings", 15_000, 4000, 150_000,
                          opacity_reset_at=3000),
    "high": SceneSpec("high", 250_000, 150, 640, 480, 600.0, "hemisphere", 30_000, 7000, 300_000, roll_deg=10.0),
    # Small scenes for parity tests.
    "tiny": SceneSpec("tiny", 2_000, 8, 96, 72, 90.0, "ring", 600, 300, 4_000),
    "small": SceneSpec("small", 8_000, 12, 160, 120, 150.0, "ring", 2_000, 600, 12_000),
}


def batched_specs(seed: int = 0, count: int = 16) -> list:
    """The batched multi-scene workload: `count` scenes with ground-truth counts log-uniform in
    [20k, 300k], view counts uniform in [30, 200] and widths drawn from {320, 480, 640}; each scene
    otherwise follows the preset of its width (Fast / Balanced / High: focal length, camera layout,
    initial points, schedule and Gaussian cap 80k / 150k / 300k)."""
    rng = np.random.default_rng([seed, 3])
    by_width = {320: "fast", 480: "balanced", 640: "high"}
    specs = []
    for k in range(count):
        gt = int(round(math.exp(rng.uniform(math.log(20e3), math.log(300e3)))))
        views = int(rng.integers(30, 201))
        width = int(rng.choice(sorted(by_width)))
        base = PRESETS[by_width[width]]
        specs.append(dataclasses.replace(base, name=f"batch{k}-{base.name}", gt_count=gt, views=views))
    return specs


@dataclass
class Scene:
    spec: SceneSpec
    seed: int
    truth: GaussianModel
    sh_rest: np.ndarray  # (n, 15, 3) float32, degree 1..3 coefficients
    cameras: list
    init_xyz: np.ndarray
    init_rgb: np.ndarray
    extent: float
    images: list = field(default_factory=list)

    def options(self) -> TrainOptions:
        """TrainOptions::forIterations(iterations) + max Gaussians, with the explicit opacity-reset
        override of the Balanced config (forIterations(4000) has no reset and stops refinement at
        2400, Trainer.cpp:30-33, so the reset at 3000 needs refine_stop past it)."""
        o = TrainOptions.for_iterations(self.spec.iterations)
        o.max_gaussians = self.spec.max_gaussians
        if self.spec.opacity_reset_at > 0:
            o.opacity_reset_interval = self.spec.opacity_reset_at
            o.refine_stop = max(o.refine_stop, self.spec.opacity_reset_at + 1)
        return o


def look_at(center, width, height, focal, roll=0.0) -> RenderCamera:
    """Pinhole camera at `center` looking at the origin: z forward, y as close to world +y (down) as
    possible, x = y cross z; then rolled by `roll` radians about z."""
    c = np.asarray(center, dtype=np.float64)
    z = -c / np.linalg.norm(c)
    down = np.array([0.0, 1.0, 0.0])
    y = down - np.dot(down, z) * z
    if np.linalg.norm(y) < 1e-6:
        y = np.array([0.0, 0.0, 1.0]) - z[2] * z
    y /= np.linalg.norm(y)
    x = np.cross(y, z)
    if roll != 0.0:
        cr, sr = math.cos(roll), math.sin(roll)
        x, y = cr * x + sr * y, -sr * x + cr * y
    R = np.stack([x, y, z]).astype(np.float32)
    t = (-(R.astype(np.float64) @ c)).astype(np.float32)
    return RenderCamera(width, height, float(focal), float(focal), 0.5 * (width - 1), 0.5 * (height - 1), R, t)


def camera_centers(spec: SceneSpec, rng: np.random.Generator):
    r = spec.radius
    out = []
    if spec.layout == "ring":
        for k in range(spec.views):
            a = 2.0 * math.pi * k / spec.views
            out.append((r * math.sin(a), 0.0, -r * math.cos(a)))
    elif spec.layout == "two_rings":
        half = spec.views // 2
        for ring, el in ((0, math.radians(20.0)), (1, math.radians(-20.0))):
            count = half if ring == 0 else spec.views - half
            for k in range(count):
                a = 2.0 * math.pi * (k + 0.5 * ring) / count
                out.append((r * math.cos(el) * math.sin(a), -r * math.sin(el), -r * math.cos(el) * math.cos(a)))
    elif spec.layout == "hemisphere":
        golden = math.pi * (3.0 - math.sqrt(5.0))
        s0, s1 = math.sin(math.radians(5.0)), math.sin(math.radians(80.0))
        for k in range(spec.views):
            el = math.asin(s0 + (s1 - s0) * (k + 0.5) / spec.views)
            a = k * golden
            out.append((r * math.cos(el) * math.sin(a), -r * math.sin(el), -r * math.cos(el) * math.cos(a)))
    else:
        raise ValueError(spec.layout)
    rolls = rng.uniform(-spec.roll_deg, spec.roll_deg, size=len(out)) if spec.roll_deg > 0 else np.zeros(len(out))
    return out, rolls


def make_scene(name_or_spec, seed: int = 0) -> Scene:
    spec = PRESETS[name_or_spec] if isinstance(name_or_spec, str) else name_or_spec
    rng = np.random.default_rng(seed)
    n = spec.gt_count
    means = rng.uniform(-1.0, 1.0, size=(n, 3)).astype(np.float32)
    scales = rng.normal(-4.0, 0.5, size=(n, 3)).astype(np.float32)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opac = rng.uniform(0.3, 1.0, size=n)
    dc_rgb = rng.uniform(0.0, 1.0, size=(n, 3))
    K = (spec.sh_degree + 1) ** 2 - 1
    sh_rest = rng.normal(0.0, 0.05, size=(n, K, 3)).astype(np.float32)
    truth = GaussianModel(means, scales, q.astype(np.float32),
                          np.log(opac / (1.0 - opac)).astype(np.float32),
                          ((dc_rgb - 0.5) / SH_C0).astype(np.float32))
    centers, rolls = camera_centers(spec, rng)
    cams = [look_at(c, spec.width, spec.height, spec.focal, math.radians(float(r))) for c, r in zip(centers, rolls)]
    idx = rng.choice(n, size=min(spec.init_count, n), replace=False) if spec.init_count <= n else \
        rng.integers(0, n, size=spec.init_count)
    init_xyz = (means[idx].astype(np.float64) + rng.normal(0.0, spec.init_noise, size=(len(idx), 3))).astype(np.float32)
    init_rgb = np.clip(dc_rgb[idx], 0.0, 1.0).astype(np.float32)
    cc = np.array(centers, dtype=np.float64)
    extent = max(float(np.max(np.linalg.norm(cc - cc.mean(axis=0), axis=1))) * 1.1, 1e-3)
    return Scene(spec, seed, truth, sh_rest, cams, init_xyz, init_rgb, extent)


def dense_init_points(scene: Scene, count: int, seed: int = 1):
    """`count` initial points for a model at full capacity: every true centre (in order) and then
    noisy re-samples of random centres, all with N(0, init_noise) noise; coloured by DC colour."""
    rng = np.random.default_rng(seed)
    n = scene.truth.size()
    idx = np.concatenate([np.arange(min(n, count)), rng.integers(0, n, size=max(0, count - n))])
    xyz = (scene.truth.means[idx].astype(np.float64)
           + rng.normal(0.0, scene.spec.init_noise, size=(len(idx), 3))).astype(np.float32)
    rgb = np.clip(0.5 + SH_C0 * scene.truth.colors[idx].astype(np.float64), 0.0, 1.0).astype(np.float32)
    return xyz, rgb


def render_targets(scene: Scene, render_fn, degree: int | None = None) -> list:
    """Fills scene.images: render_fn(model, sh_rest, degree, camera) -> (h, w, 3) float32 in 0..1,
    quantised as TrainImage::quantize does."""
    deg = scene.spec.sh_degree if degree is None else degree
    scene.images = [TrainImage(cam, TrainImage.quantize(render_fn(scene.truth, scene.sh_rest, deg, cam)))
                    for cam in scene.cameras]
    return scene.images
