"""ctypes binding of the CPU checkers. TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the CPU restatement, oracle.cpp) and, when it was built,
oracle/_ref/libu3dref.so (the reference's own sources behind ref_shim.cpp). Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference legs import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from univeral_3d_reconstruction_system_b200 import _abi
from univeral_3d_reconstruction_system_b200.types import GaussianModel, images_struct

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libu3dref.so"

_P = C.c_void_p
_MV = C.POINTER(_abi.ModelView)
_CAM = C.POINTER(_abi.Camera)
_ST = C.POINTER(_abi.RasterSettings)
_OPT = C.POINTER(_abi.TrainOptions)
_IMG = C.POINTER(_abi.Image)
_F = _abi.f32p
_I = _abi.i32p


def build(quiet: bool = True) -> None:
    """make -C oracle (liboracle.so always; _ref/libu3dref.so when the reference tree exists)."""
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _load(path: Path):
    if not path.exists():
        build()
    return C.CDLL(str(path))


def _sig(lib, name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


class _Lib:
    """Common signatures of liboracle (prefix orc_) and libu3dref (prefix ref_)."""

    def __init__(self, lib, prefix):
        self.lib = lib
        p = prefix
        _sig(lib, p + "raster_create", _P, C.c_int)
        _sig(lib, p + "raster_destroy", None, _P)
        _sig(lib, p + "raster_backward", None, _P, _F, _MV, _F)
        _sig(lib, p + "photometric_loss", None, _F, _F, C.c_int, C.c_int, C.c_float, _F,
             *([C.c_int] if p == "ref_" else []), C.POINTER(_abi.LossValue))
        _sig(lib, p + "psnr", C.c_float, _F, _F, C.c_size_t)
        _sig(lib, p + "trainer_create", _P, _MV, _IMG, C.c_int, C.c_float, _OPT, C.c_int)
        _sig(lib, p + "trainer_step", None, _P, C.c_int)
        _sig(lib, p + "trainer_stats", None, _P, C.POINTER(_abi.TrainStats))
        _sig(lib, p + "trainer_size", C.c_size_t, _P)
        _sig(lib, p + "trainer_download", None, _P, _MV)
        _sig(lib, p + "trainer_eval_psnr", C.c_float, _P)
        _sig(lib, p + "trainer_destroy", None, _P)
        _sig(lib, p + "init_from_points", None, _F, _F, C.c_size_t, _MV)
        _sig(lib, p + "options_for_iterations", None, C.c_int, _OPT)
        _sig(lib, p + "crop_model", C.c_size_t, _MV, C.POINTER(_abi.CropBox), C.c_float, _MV)
        self.p = p

    def crop_model(self, model: GaussianModel, box, min_opacity: float = 0.0) -> GaussianModel:
        """cropModel (Crop.cpp:44-52); box = (min xyz, max xyz)."""
        mv, cb = model.view(), _crop_box(box)
        n = int(self.fn("crop_model")(C.byref(mv), C.byref(cb), float(min_opacity), None))
        out = GaussianModel.zeros(n)
        ov = out.view()
        self.fn("crop_model")(C.byref(mv), C.byref(cb), float(min_opacity), C.byref(ov))
        return out

    def fn(self, name):
        return getattr(self.lib, self.p + name)


def _crop_box(b) -> _abi.CropBox:
    out = _abi.CropBox()
    for k in range(3):
        out.min[k], out.max[k] = float(b[0][k]), float(b[1][k])
    return out


def _unbox(b: _abi.CropBox):
    return np.array(list(b.min), np.float32), np.array(list(b.max), np.float32)


class Raster:
    """A Rasterizer: forward keeps state for backward (Rasterizer.h:38-54)."""

    def __init__(self, lib: _Lib, threads: int = 1):
        self.L = lib
        self.h = lib.fn("raster_create")(threads)
        self.model = None

    def __del__(self):
        if getattr(self, "h", None):
            self.L.fn("raster_destroy")(self.h)
            self.h = None

    def backward(self, dl_drgb: np.ndarray, with_ndc: bool = True):
        m = self.model
        g = GaussianModel.zeros(m.size())
        ndc = np.zeros(m.size(), np.float32)
        gv = g.view()
        self.L.fn("raster_backward")(self.h, _abi.fptr(np.ascontiguousarray(dl_drgb, np.float32)), C.byref(gv),
                                     _abi.fptr(ndc) if with_ndc else None)
        return g, ndc


class Trainer:
    def __init__(self, lib: _Lib, init: GaussianModel, images, extent: float, options, threads: int = 1):
        self.L = lib
        arr, self._keep = images_struct(images)
        iv = init.view()
        opt = options.struct() if hasattr(options, "struct") else options
        self.h = lib.fn("trainer_create")(C.byref(iv), arr, len(images), float(extent), C.byref(opt), threads)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.fn("trainer_destroy")(self.h)
            self.h = None

    def step(self, count: int = 1):
        self.L.fn("trainer_step")(self.h, count)

    def stats(self):
        s = _abi.TrainStats()
        self.L.fn("trainer_stats")(self.h, C.byref(s))
        return s

    def size(self) -> int:
        return int(self.L.fn("trainer_size")(self.h))

    def model(self) -> GaussianModel:
        g = GaussianModel.zeros(self.size())
        v = g.view()
        self.L.fn("trainer_download")(self.h, C.byref(v))
        return g

    def evaluate_psnr(self) -> float:
        return float(self.L.fn("trainer_eval_psnr")(self.h))


class Oracle(_Lib):
    """The CPU restatement (oracle.cpp)."""

    def __init__(self):
        lib = _load(ORACLE_SO)
        super().__init__(lib, "orc_")
        _sig(lib, "orc_raster_forward", None, _P, _MV, _F, C.c_int, _CAM, _ST, _F)
        _sig(lib, "orc_raster_project", None, _P, _MV, _CAM, _ST)
        _sig(lib, "orc_bin_tiles", None, _F, _I, _I, C.c_size_t, C.c_int, C.c_int, _I, _I, C.c_size_t,
             C.POINTER(C.c_size_t))
        _sig(lib, "orc_raster_projection", None, _P, _F, _F, _F, _F, _F, _F, _I, _I, _abi.u8p)
        _sig(lib, "orc_raster_list_length", C.c_size_t, _P)
        _sig(lib, "orc_raster_tiles", None, _P, _I, _I)
        _sig(lib, "orc_raster_pixel_state", None, _P, _F, _I)
        _sig(lib, "orc_raster_g2d", None, _P, _F)
        _sig(lib, "orc_adam_step", None, _MV, _MV, _MV, _MV, C.c_int, C.POINTER(_abi.LearningRates))
        _sig(lib, "orc_densify", None, _MV, _MV, _MV, _F, _I, C.c_size_t, C.c_float, _OPT, C.c_int, C.c_uint,
             C.POINTER(C.c_size_t), _I)
        _sig(lib, "orc_trainer_iteration", C.c_int, _P)
        _sig(lib, "orc_trainer_view_log", C.c_int, _P, _I, C.c_int)
        _sig(lib, "orc_crop_box", None, _MV, C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(_abi.CropBox))

    def suggest_crop_box(self, model: GaussianModel, lo=0.05, hi=0.95, margin=0.1):
        """suggestCropBox (Crop.cpp:54-57): quantileBox with an opacity floor of 0.3."""
        mv, out = model.view(), _abi.CropBox()
        self.lib.orc_crop_box(C.byref(mv), lo, hi, margin, 0.3, C.byref(out))
        return _unbox(out)

    def model_bounds(self, model: GaussianModel):
        """modelBounds (Crop.cpp:59-62)."""
        mv, out = model.view(), _abi.CropBox()
        self.lib.orc_crop_box(C.byref(mv), 0.005, 0.995, 0.1, 0.0, C.byref(out))
        return _unbox(out)

    # -- rasterizer
    def raster(self, threads: int = os.cpu_count() or 1) -> "OracleRaster":
        return OracleRaster(self, threads)

    def bin_tiles(self, depth, radius, rect, tiles_x, tiles_y):
        depth = np.ascontiguousarray(depth, np.float32)
        radius = np.ascontiguousarray(radius, np.int32)
        rect = np.ascontiguousarray(rect, np.int32).reshape(-1)
        n = depth.size
        offsets = np.zeros(tiles_x * tiles_y + 1, np.int32)
        cap = int(np.sum(np.maximum(rect[2::4] - rect[0::4], 0) * np.maximum(rect[3::4] - rect[1::4], 0)
                         * (radius > 0)))
        lst = np.zeros(max(cap, 1), np.int32)
        length = C.c_size_t(0)
        self.lib.orc_bin_tiles(_abi.fptr(depth), _abi.iptr(radius), _abi.iptr(rect), n, tiles_x, tiles_y,
                               _abi.iptr(offsets), _abi.iptr(lst), lst.size, C.byref(length))
        return offsets, lst[: length.value].copy()

    def photometric_loss(self, render, target, width, height, lam):
        render = np.ascontiguousarray(render, np.float32).reshape(-1)
        target = np.ascontiguousarray(target, np.float32).reshape(-1)
        grad = np.zeros_like(render)
        out = _abi.LossValue()
        self.lib.orc_photometric_loss(_abi.fptr(render), _abi.fptr(target), width, height, lam, _abi.fptr(grad),
                                      C.byref(out))
        return out, grad

    def psnr(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32).reshape(-1)
        b = np.ascontiguousarray(b, np.float32).reshape(-1)
        return float(self.lib.orc_psnr(_abi.fptr(a), _abi.fptr(b), a.size))

    def adam_step(self, params: GaussianModel, grads: GaussianModel, m: GaussianModel, v: GaussianModel, step: int, lr):
        pv, gv, mv, vv = params.view(), grads.view(), m.view(), v.view()
        lrs = lr.struct() if hasattr(lr, "struct") else lr
        self.lib.orc_adam_step(C.byref(pv), C.byref(gv), C.byref(mv), C.byref(vv), step, C.byref(lrs))

    def densify(self, model, m, v, grad_accum, grad_count, extent, options, opacity_was_reset, seed):
        cap = max(options.max_gaussians, model.size())
        out = [GaussianModel.zeros(cap) for _ in range(3)]
        for dst, src in zip(out, (model, m, v)):
            for name, _ in _abi.GROUPS:
                getattr(dst, name)[: src.size()] = getattr(src, name)
        views = [o.view() for o in out]
        for vw in views:
            vw.count = model.size()
        count = C.c_size_t(0)
        counts = np.zeros(3, np.int32)
        opt = options.struct()
        self.lib.orc_densify(C.byref(views[0]), C.byref(views[1]), C.byref(views[2]),
                             _abi.fptr(np.ascontiguousarray(grad_accum, np.float32)),
                             _abi.iptr(np.ascontiguousarray(grad_count, np.int32)), cap, float(extent), C.byref(opt),
                             int(opacity_was_reset), seed, C.byref(count), _abi.iptr(counts))
        n = count.value
        res = [GaussianModel(*(getattr(o, name)[:n].copy() for name, _ in _abi.GROUPS)) for o in out]
        return res[0], res[1], res[2], counts

    def trainer(self, init, images, extent, options, threads: int = os.cpu_count() or 1) -> "OracleTrainer":
        return OracleTrainer(self, init, images, extent, options, threads)

    def init_from_points(self, xyz, rgb=None) -> GaussianModel:
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1)
        n = xyz.size // 3
        out = GaussianModel.zeros(n)
        v = out.view()
        rgb_p = _abi.fptr(np.ascontiguousarray(rgb, np.float32).reshape(-1)) if rgb is not None else None
        self.lib.orc_init_from_points(_abi.fptr(xyz), rgb_p, n, C.byref(v))
        return out

    def render(self, model: GaussianModel, cam, settings, sh_rest=None, degree: int = 0, threads=None):
        r = self.raster(threads or os.cpu_count() or 1)
        return r.forward(model, cam, settings, sh_rest, degree)


class OracleRaster(Raster):
    def forward(self, model: GaussianModel, cam, settings, sh_rest=None, degree: int = 0):
        self.model = model
        self.cam = cam
        mv = model.view()
        cs = cam.struct() if hasattr(cam, "struct") else cam
        ss = settings.struct() if hasattr(settings, "struct") else settings
        rgb = np.zeros((cs.height, cs.width, 3), np.float32)
        shp = None
        if sh_rest is not None and degree > 0:
            shp = _abi.fptr(np.ascontiguousarray(sh_rest, np.float32).reshape(-1))
        self.L.lib.orc_raster_forward(self.h, C.byref(mv), shp, degree, C.byref(cs), C.byref(ss), _abi.fptr(rgb))
        self._cs, self._ss = cs, ss
        return rgb

    def project(self, model: GaussianModel, cam, settings):
        self.model = model
        mv = model.view()
        cs = cam.struct() if hasattr(cam, "struct") else cam
        ss = settings.struct() if hasattr(settings, "struct") else settings
        self.L.lib.orc_raster_project(self.h, C.byref(mv), C.byref(cs), C.byref(ss))

    def projection(self):
        n = self.model.size()
        out = dict(mean2d=np.zeros((n, 2), np.float32), conic=np.zeros((n, 3), np.float32),
                   cov2d=np.zeros((n, 3), np.float32), depth=np.zeros(n, np.float32), rgb=np.zeros((n, 3), np.float32),
                   alpha=np.zeros(n, np.float32), radius=np.zeros(n, np.int32), rect=np.zeros((n, 4), np.int32),
                   flags=np.zeros(n, np.uint8))
        self.L.lib.orc_raster_projection(self.h, *(_abi.fptr(out[k]) for k in
                                                   ("mean2d", "conic", "cov2d", "depth", "rgb", "alpha")),
                                         _abi.iptr(out["radius"]), _abi.iptr(out["rect"]),
                                         out["flags"].ctypes.data_as(_abi.u8p))
        return out

    def tiles(self):
        L = int(self.L.lib.orc_raster_list_length(self.h))
        tx = (self._cs.width + self._ss.tile_size - 1) // self._ss.tile_size
        ty = (self._cs.height + self._ss.tile_size - 1) // self._ss.tile_size
        offsets = np.zeros(tx * ty + 1, np.int32)
        lst = np.zeros(max(L, 1), np.int32)
        self.L.lib.orc_raster_tiles(self.h, _abi.iptr(offsets), _abi.iptr(lst))
        return offsets, lst[:L]

    def pixel_state(self):
        P = self._cs.width * self._cs.height
        ft = np.zeros(P, np.float32)
        nc = np.zeros(P, np.int32)
        self.L.lib.orc_raster_pixel_state(self.h, _abi.fptr(ft), _abi.iptr(nc))
        return ft, nc

    def g2d(self):
        out = np.zeros((self.model.size(), 9), np.float32)
        self.L.lib.orc_raster_g2d(self.h, _abi.fptr(out))
        return out


class OracleTrainer(Trainer):
    def iteration(self) -> int:
        return int(self.L.lib.orc_trainer_iteration(self.h))

    def view_log(self):
        n = int(self.L.lib.orc_trainer_view_log(self.h, None, 0))
        out = np.zeros(max(n, 1), np.int32)
        self.L.lib.orc_trainer_view_log(self.h, _abi.iptr(out), n)
        return out[:n]


class Reference(_Lib):
    """The reference's own splat core (oracle/_ref/libu3dref.so)."""

    def __init__(self):
        if not REF_SO.exists():
            build()
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} was not built (reference sources absent)")
        lib = C.CDLL(str(REF_SO))
        super().__init__(lib, "ref_")
        _sig(lib, "ref_raster_forward", None, _P, _MV, _CAM, _ST, _F)
        _sig(lib, "ref_raster_radii", None, _P, _I)
        _sig(lib, "ref_adam_create", _P, C.c_size_t, C.c_int)
        _sig(lib, "ref_adam_step", None, _P, _MV, _MV, C.POINTER(_abi.LearningRates))
        _sig(lib, "ref_adam_compact", None, _P, _abi.u8p, C.c_size_t)
        _sig(lib, "ref_adam_grow", None, _P, C.c_size_t)
        _sig(lib, "ref_adam_reset_opacity_moments", None, _P)
        _sig(lib, "ref_adam_destroy", None, _P)
        _sig(lib, "ref_trainer_done", C.c_int, _P)
        _sig(lib, "ref_trainer_render", None, _P, _CAM, _F)
        _sig(lib, "ref_pool_threads", C.c_int, C.c_int)
        _sig(lib, "ref_write_splat_ply", C.c_int, C.c_char_p, _MV)
        _sig(lib, "ref_read_splat_ply", C.c_int, C.c_char_p, _MV, C.POINTER(C.c_size_t), C.POINTER(C.c_int))
        _sig(lib, "ref_crop_box", None, _MV, C.c_float, C.c_float, C.c_float, C.c_int, C.POINTER(_abi.CropBox))

    def suggest_crop_box(self, model: GaussianModel, lo=0.05, hi=0.95, margin=0.1):
        mv, out = model.view(), _abi.CropBox()
        self.lib.ref_crop_box(C.byref(mv), lo, hi, margin, 0, C.byref(out))
        return _unbox(out)

    def model_bounds(self, model: GaussianModel):
        mv, out = model.view(), _abi.CropBox()
        self.lib.ref_crop_box(C.byref(mv), 0.0, 0.0, 0.0, 1, C.byref(out))
        return _unbox(out)

    @staticmethod
    def available() -> bool:
        if not REF_SO.exists():
            try:
                build()
            except Exception:
                return False
        return REF_SO.exists()

    def raster(self, threads: int = 1) -> "RefRaster":
        return RefRaster(self, threads)

    def photometric_loss(self, render, target, width, height, lam, threads=1):
        render = np.ascontiguousarray(render, np.float32).reshape(-1)
        target = np.ascontiguousarray(target, np.float32).reshape(-1)
        grad = np.zeros_like(render)
        out = _abi.LossValue()
        self.lib.ref_photometric_loss(_abi.fptr(render), _abi.fptr(target), width, height, lam, _abi.fptr(grad),
                                      threads, C.byref(out))
        return out, grad

    def psnr(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32).reshape(-1)
        b = np.ascontiguousarray(b, np.float32).reshape(-1)
        return float(self.lib.ref_psnr(_abi.fptr(a), _abi.fptr(b), a.size))

    def trainer(self, init, images, extent, options, threads: int = 0) -> Trainer:
        return Trainer(self, init, images, extent, options, threads)

    def init_from_points(self, xyz, rgb=None) -> GaussianModel:
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1)
        n = xyz.size // 3
        out = GaussianModel.zeros(n)
        v = out.view()
        rgb_p = _abi.fptr(np.ascontiguousarray(rgb, np.float32).reshape(-1)) if rgb is not None else None
        self.lib.ref_init_from_points(_abi.fptr(xyz), rgb_p, n, C.byref(v))
        return out

    def pool_threads(self, threads: int = 0) -> int:
        return int(self.lib.ref_pool_threads(threads))


class RefRaster(Raster):
    def forward(self, model: GaussianModel, cam, settings):
        self.model = model
        mv = model.view()
        cs = cam.struct() if hasattr(cam, "struct") else cam
        ss = settings.struct() if hasattr(settings, "struct") else settings
        rgb = np.zeros((cs.height, cs.width, 3), np.float32)
        self.L.lib.ref_raster_forward(self.h, C.byref(mv), C.byref(cs), C.byref(ss), _abi.fptr(rgb))
        return rgb

    def radii(self):
        out = np.zeros(self.model.size(), np.int32)
        self.L.lib.ref_raster_radii(self.h, _abi.iptr(out))
        return out
