"""ctypes mirror of the C ABI types in include/u3dg.h.

Only plain data types live here (no library loading), so the product binding
(`_lib.py`) and the test-side oracle binding share one definition of every struct.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

OK = 0
ERR_INVALID_ARG = 1
ERR_OOM = 2
ERR_CUDA = 3
ERR_TIMEOUT = 4
ERR_CAPACITY = 5
ERR_IO = 6
ERR_NO_DEVICE = 7
ERR_STATE = 8

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int)
u8p = C.POINTER(C.c_uint8)


class Camera(C.Structure):
    """u3dg_camera == RenderCamera (engine/include/u3d/splat/Rasterizer.h:13-21)."""

    _fields_ = [
        ("width", C.c_int),
        ("height", C.c_int),
        ("fx", C.c_float),
        ("fy", C.c_float),
        ("cx", C.c_float),
        ("cy", C.c_float),
        ("R", C.c_float * 9),
        ("t", C.c_float * 3),
    ]


class RasterSettings(C.Structure):
    """u3dg_raster_settings == RasterSettings (Rasterizer.h:23-32)."""

    _fields_ = [
        ("tile_size", C.c_int),
        ("near_plane", C.c_float),
        ("eps2d", C.c_float),
        ("background", C.c_float * 3),
        ("min_alpha", C.c_float),
        ("min_transmittance", C.c_float),
    ]


class CropBox(C.Structure):
    """u3dg_crop_box == CropBox (engine/include/u3d/splat/Crop.h:9-19)."""

    _fields_ = [("min", C.c_float * 3), ("max", C.c_float * 3)]


class LearningRates(C.Structure):
    """u3dg_learning_rates == LearningRates (engine/include/u3d/splat/Adam.h:8-14)."""

    _fields_ = [(n, C.c_float) for n in ("means", "scales", "quats", "opacities", "colors")]


class TrainOptions(C.Structure):
    """u3dg_train_options == TrainOptions (engine/include/u3d/splat/Trainer.h:20-38)."""

    _fields_ = [
        ("iterations", C.c_int),
        ("max_gaussians", C.c_int),
        ("ssim_lambda", C.c_float),
        ("lr", LearningRates),
        ("means_lr_final", C.c_float),
        ("densify_grad_threshold", C.c_float),
        ("percent_dense", C.c_float),
        ("refine_start", C.c_int),
        ("refine_stop", C.c_int),
        ("refine_interval", C.c_int),
        ("opacity_reset_interval", C.c_int),
        ("prune_opacity", C.c_float),
        ("seed", C.c_uint),
        ("raster", RasterSettings),
    ]


class TrainStats(C.Structure):
    """u3dg_train_stats == TrainStats (Trainer.h:40-45)."""

    _fields_ = [
        ("iteration", C.c_int),
        ("loss", C.c_float),
        ("psnr", C.c_float),
        ("gaussians", C.c_uint64),
    ]


class LossValue(C.Structure):
    """u3dg_loss_value == LossValue (engine/include/u3d/splat/Loss.h:9-13)."""

    _fields_ = [("total", C.c_float), ("l1", C.c_float), ("ssim", C.c_float)]


class ModelView(C.Structure):
    """u3dg_model: pointers to the five GaussianModel arrays (GaussianModel.h:23-37)."""

    _fields_ = [
        ("means", f32p),
        ("scales", f32p),
        ("quats", f32p),
        ("opacities", f32p),
        ("colors", f32p),
        ("count", C.c_size_t),
    ]


class Image(C.Structure):
    """u3dg_image == TrainImage (Trainer.h:13-18)."""

    _fields_ = [("camera", Camera), ("rgb", u8p)]


class PhaseTimes(C.Structure):
    """u3dg_phase_times: per-phase device time of profiled trainer steps."""

    _fields_ = [
        ("steps", C.c_int),
        ("project_ms", C.c_float),
        ("sort_ms", C.c_float),
        ("forward_ms", C.c_float),
        ("loss_ms", C.c_float),
        ("backward_ms", C.c_float),
        ("update_ms", C.c_float),
        ("densify_ms", C.c_float),
        ("total_ms", C.c_float),
        ("intersections", C.c_uint64),
        ("visible", C.c_uint64),
        ("gaussians", C.c_uint64),
        ("pixels", C.c_uint64),
    ]


GROUPS = (("means", 3), ("scales", 3), ("quats", 4), ("opacities", 1), ("colors", 3))


def fptr(a: np.ndarray):
    """float* of a C-contiguous float32 array."""
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(f32p)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(i32p)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(u8p)


def camera_struct(cam) -> Camera:
    """Camera struct from any object with width/height/fx/fy/cx/cy/R/t attributes."""
    c = Camera()
    c.width, c.height = int(cam.width), int(cam.height)
    c.fx, c.fy, c.cx, c.cy = float(cam.fx), float(cam.fy), float(cam.cx), float(cam.cy)
    R = np.asarray(cam.R, dtype=np.float32).reshape(9)
    t = np.asarray(cam.t, dtype=np.float32).reshape(3)
    for k in range(9):
        c.R[k] = float(R[k])
    for k in range(3):
        c.t[k] = float(t[k])
    return c
