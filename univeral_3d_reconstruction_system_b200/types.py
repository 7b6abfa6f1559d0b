"""Host-side value types mirroring the reference's C++ structs (numpy-backed).

GaussianModel   engine/include/u3d/splat/GaussianModel.h:23-37
RenderCamera    engine/include/u3d/splat/Rasterizer.h:13-21
RasterSettings  engine/include/u3d/splat/Rasterizer.h:23-32
LearningRates   engine/include/u3d/splat/Adam.h:8-14
TrainOptions    engine/include/u3d/splat/Trainer.h:20-38
TrainImage      engine/include/u3d/splat/Trainer.h:13-18
TrainStats      engine/include/u3d/splat/Trainer.h:40-45
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

SH_C0 = 0.28209479177387814  # GaussianModel.h:10
GROUPS_ORDER = ("means", "scales", "quats", "opacities", "colors")


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-np.asarray(x, dtype=np.float32)))


def logit(p: float) -> float:
    """logit in float32 arithmetic, as GaussianModel.h:13 computes it."""
    p = np.float32(p)
    return float(np.log(np.float32(p / (np.float32(1.0) - p))))


@dataclass
class GaussianModel:
    """SoA Gaussian parameters: means (n,3), scales (n,3) log sigma, quats (n,4) w,x,y,z,
    opacities (n,) logit, colors (n,3) SH degree-0 coefficients."""

    means: np.ndarray
    scales: np.ndarray
    quats: np.ndarray
    opacities: np.ndarray
    colors: np.ndarray

    def __post_init__(self):
        for name, dim in _abi.GROUPS:
            a = np.ascontiguousarray(getattr(self, name), dtype=np.float32)
            a = a.reshape(-1) if dim == 1 else a.reshape(-1, dim)
            setattr(self, name, a)
        n = self.opacities.shape[0]
        for name, _ in _abi.GROUPS:
            if getattr(self, name).shape[0] != n:
                raise ValueError(f"GaussianModel.{name} has {getattr(self, name).shape[0]} rows, expected {n}")

    @classmethod
    def zeros(cls, n: int) -> "GaussianModel":
        return cls(np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
                   np.zeros(n, np.float32), np.zeros((n, 3), np.float32))

    def size(self) -> int:
        return int(self.opacities.shape[0])

    def __len__(self) -> int:
        return self.size()

    def copy(self) -> "GaussianModel":
        return GaussianModel(*(getattr(self, n).copy() for n, _ in _abi.GROUPS))

    def view(self) -> _abi.ModelView:
        """u3dg_model pointing at this model's arrays (valid while the model is alive)."""
        v = _abi.ModelView()
        for name, _ in _abi.GROUPS:
            setattr(v, name, _abi.fptr(getattr(self, name)))
        v.count = self.size()
        return v

    def flat(self) -> np.ndarray:
        """All parameters as one float32 vector, group after group."""
        return np.concatenate([getattr(self, n).reshape(-1) for n, _ in _abi.GROUPS])


@dataclass
class RenderCamera:
    width: int = 0
    height: int = 0
    fx: float = 0.0
    fy: float = 0.0
    cx: float = 0.0
    cy: float = 0.0
    R: np.ndarray = field(default_factory=lambda: np.eye(3, dtype=np.float32))
    t: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))

    def __post_init__(self):
        self.R = np.asarray(self.R, dtype=np.float32).reshape(3, 3)
        self.t = np.asarray(self.t, dtype=np.float32).reshape(3)

    def struct(self) -> _abi.Camera:
        return _abi.camera_struct(self)

    def center(self) -> np.ndarray:
        """Camera centre in world coordinates, -R^T t."""
        return -(self.R.astype(np.float64).T @ self.t.astype(np.float64))


@dataclass
class RasterSettings:
    tile_size: int = 16
    near_plane: float = 0.01
    eps2d: float = 0.3
    background: tuple = (0.0, 0.0, 0.0)
    min_alpha: float = float(np.float32(1.0) / np.float32(255.0))
    min_transmittance: float = 1e-4

    def struct(self) -> _abi.RasterSettings:
        s = _abi.RasterSettings()
        s.tile_size = int(self.tile_size)
        s.near_plane = self.near_plane
        s.eps2d = self.eps2d
        for k in range(3):
            s.background[k] = float(self.background[k])
        s.min_alpha = self.min_alpha
        s.min_transmittance = self.min_transmittance
        return s


@dataclass
class LearningRates:
    means: float = 1.6e-4
    scales: float = 5e-3
    quats: float = 1e-3
    opacities: float = 5e-2
    colors: float = 2.5e-3

    def struct(self) -> _abi.LearningRates:
        return _abi.LearningRates(self.means, self.scales, self.quats, self.opacities, self.colors)


@dataclass
class TrainOptions:
    iterations: int = 3000
    max_gaussians: int = 200000
    ssim_lambda: float = 0.2
    lr: LearningRates = field(default_factory=LearningRates)
    means_lr_final: float = 1.6e-6
    densify_grad_threshold: float = 2e-4
    percent_dense: float = 0.01
    refine_start: int = 500
    refine_stop: int = 15000
    refine_interval: int = 100
    opacity_reset_interval: int = 3000
    prune_opacity: float = 0.005
    seed: int = 42
    raster: RasterSettings = field(default_factory=RasterSettings)

    @classmethod
    def for_iterations(cls, iterations: int) -> "TrainOptions":
        """TrainOptions::forIterations (engine/src/splat/Trainer.cpp:26-35)."""
        o = cls()
        o.iterations = max(1, int(iterations))
        o.refine_start = min(500, o.iterations // 10)
        o.refine_stop = o.iterations * 6 // 10
        o.refine_interval = 100
        o.opacity_reset_interval = 3000 if o.iterations >= 6000 else 0
        return o

    def struct(self) -> _abi.TrainOptions:
        o = _abi.TrainOptions()
        for f in dataclasses.fields(self):
            if f.name == "lr":
                o.lr = self.lr.struct()
            elif f.name == "raster":
                o.raster = self.raster.struct()
            else:
                setattr(o, f.name, getattr(self, f.name))
        return o

    def replace(self, **kw) -> "TrainOptions":
        return dataclasses.replace(self, **kw)

    @classmethod
    def from_struct(cls, o: _abi.TrainOptions) -> "TrainOptions":
        r = o.raster
        return cls(o.iterations, o.max_gaussians, o.ssim_lambda,
                   LearningRates(o.lr.means, o.lr.scales, o.lr.quats, o.lr.opacities, o.lr.colors),
                   o.means_lr_final, o.densify_grad_threshold, o.percent_dense, o.refine_start, o.refine_stop,
                   o.refine_interval, o.opacity_reset_interval, o.prune_opacity, o.seed,
                   RasterSettings(r.tile_size, r.near_plane, r.eps2d, tuple(r.background), r.min_alpha,
                                  r.min_transmittance))

    def struct_tuple(self) -> tuple:
        """Every field as stored in the C struct (float32 rounding applied), for comparisons."""
        o = self.struct()
        r = o.raster
        return (o.iterations, o.max_gaussians, o.ssim_lambda, o.lr.means, o.lr.scales, o.lr.quats, o.lr.opacities,
                o.lr.colors, o.means_lr_final, o.densify_grad_threshold, o.percent_dense, o.refine_start,
                o.refine_stop, o.refine_interval, o.opacity_reset_interval, o.prune_opacity, o.seed, r.tile_size,
                r.near_plane, r.eps2d, tuple(r.background), r.min_alpha, r.min_transmittance)


@dataclass
class TrainImage:
    camera: RenderCamera
    rgb: np.ndarray  # (height, width, 3) uint8

    def __post_init__(self):
        self.rgb = np.ascontiguousarray(self.rgb, dtype=np.uint8).reshape(self.camera.height, self.camera.width, 3)

    @staticmethod
    def quantize(rgb01: np.ndarray) -> np.ndarray:
        """TrainImage::quantize (Trainer.cpp:10-16): lround(clamp(v, 0, 1) * 255)."""
        v = np.clip(np.asarray(rgb01, dtype=np.float32), 0.0, 1.0) * np.float32(255.0)
        # lround rounds half away from zero; values are non-negative here.
        return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)


@dataclass
class TrainStats:
    iteration: int = 0
    loss: float = 0.0
    psnr: float = 0.0
    gaussians: int = 0


@dataclass
class LossValue:
    total: float = 0.0
    l1: float = 0.0
    ssim: float = 0.0


def images_struct(images):
    """(array of u3dg_image, keep-alive list) for a list of TrainImage."""
    arr = (_abi.Image * max(1, len(images)))()
    keep = []
    for k, img in enumerate(images):
        arr[k].camera = img.camera.struct()
        arr[k].rgb = _abi.u8ptr(img.rgb)
        keep.append(img.rgb)
    return arr, keep


def quat_normalize(q: np.ndarray) -> np.ndarray:
    q = np.asarray(q, dtype=np.float64)
    return q / np.linalg.norm(q, axis=-1, keepdims=True)


def math_isfinite(x: float) -> bool:
    return math.isfinite(x)
