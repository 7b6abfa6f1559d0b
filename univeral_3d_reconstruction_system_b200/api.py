"""Python mirror of the reference's splat API over the CUDA library (libu3dg.so).

Same classes, method names and argument meaning as engine/include/u3d/splat:
  Trainer             Trainer.h:47-93     (step, done, iteration, model, stats, images, evaluatePsnr, render)
  Rasterizer          Rasterizer.h:38-90  (forward, backward, radii)
  photometricLoss     Loss.h:18-19
  psnr                Loss.h:21
  Adam                Adam.h:18-31
  initGaussiansFromPoints  GaussianModel.h:41
  writeSplatPly / readSplatPly  SplatPly.h:12-24
Errors raise U3dgError (the reference has no error channel besides bool returns for PLY I/O;
writeSplatPly / readSplatPly keep that: they return False and set .error).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._lib import U3dgError, check, load
from .types import GaussianModel, LossValue, RasterSettings, RenderCamera, TrainImage, TrainOptions, TrainStats, \
    images_struct


def _cam(camera):
    return camera.struct() if hasattr(camera, "struct") else camera


def _settings(settings):
    return (settings or RasterSettings()).struct() if not isinstance(settings, _abi.RasterSettings) else settings


class Trainer:
    """GPU drop-in for u3d::Trainer. `pool` is accepted for API compatibility and ignored."""

    def __init__(self, initial: GaussianModel, images, scene_extent: float, options: TrainOptions | None = None,
                 pool=None, background_upload: bool = False):
        """background_upload: images go to the GPU on a host thread while the first steps run
        (u3dg_trainer_create_background_upload); the trainer keeps the pixel arrays alive."""
        L = load()
        self._images = list(images)
        self._options = options or TrainOptions()
        arr, keep = images_struct(self._images)
        iv = initial.view()
        opt = self._options.struct()
        h = C.c_void_p()
        create = L.u3dg_trainer_create_background_upload if background_upload else L.u3dg_trainer_create
        check(create(C.byref(iv), arr, len(self._images), float(scene_extent), C.byref(opt), C.byref(h)))
        self._h = h
        # The pixel arrays the C side reads (contiguous copies where needed) live as long as the trainer.
        self._keep = keep if background_upload else None

    def crop(self, box, min_opacity: float = 0.0) -> None:
        """cropModel of the trainer's model on the GPU (with its Adam moments); box = (min, max)."""
        cb = _box(box)
        check(load().u3dg_trainer_crop(self._h, C.byref(cb), float(min_opacity)))

    def suggestCropBox(self, low_fraction: float = 0.05, high_fraction: float = 0.95, margin: float = 0.1):
        """suggestCropBox of the trainer's model (low_fraction < 0: modelBounds)."""
        out = _abi.CropBox()
        check(load().u3dg_trainer_suggest_crop_box(self._h, low_fraction, high_fraction, margin, C.byref(out)))
        return _unbox(out)

    def wait_uploads(self) -> None:
        """Blocks until every training image is on the GPU (background upload)."""
        check(load().u3dg_trainer_wait_uploads(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            load().u3dg_trainer_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    def step(self, count: int = 1) -> None:
        check(load().u3dg_trainer_step(self._h, count))

    def done(self) -> bool:
        d = C.c_int()
        check(load().u3dg_trainer_done(self._h, C.byref(d)))
        return bool(d.value)

    def iteration(self) -> int:
        it = C.c_int()
        check(load().u3dg_trainer_iteration(self._h, C.byref(it)))
        return it.value

    def size(self) -> int:
        n = C.c_size_t()
        check(load().u3dg_trainer_size(self._h, C.byref(n)))
        return int(n.value)

    def model(self) -> GaussianModel:
        n = self.size()
        m = GaussianModel.zeros(n)
        v = m.view()
        cnt = C.c_size_t()
        check(load().u3dg_trainer_download(self._h, C.byref(v), n, C.byref(cnt)))
        return m

    def stats(self) -> TrainStats:
        s = _abi.TrainStats()
        check(load().u3dg_trainer_stats(self._h, C.byref(s)))
        return TrainStats(s.iteration, s.loss, s.psnr, int(s.gaussians))

    def images(self):
        return self._images

    def evaluatePsnr(self) -> float:
        p = C.c_float()
        check(load().u3dg_trainer_eval_psnr(self._h, C.byref(p)))
        return float(p.value)

    def writeSplatPly(self, path: str) -> None:
        """writeSplatPly(path, model()) in one call (u3dg_trainer_write_splat_ply)."""
        check(load().u3dg_trainer_write_splat_ply(self._h, str(path).encode()))

    evaluate_psnr = evaluatePsnr

    def render(self, camera: RenderCamera) -> np.ndarray:
        cs = _cam(camera)
        rgb = np.zeros((cs.height, cs.width, 3), np.float32)
        check(load().u3dg_trainer_render(self._h, C.byref(cs), _abi.fptr(rgb)))
        return rgb

    # -- measurement helpers (no reference counterpart)
    def stream(self) -> int:
        p = C.c_void_p()
        check(load().u3dg_trainer_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def synchronize(self) -> None:
        check(load().u3dg_trainer_synchronize(self._h))

    def time_steps(self, count: int) -> float:
        """Device milliseconds of `count` steps (CUDA events on the trainer's stream)."""
        ms = C.c_float()
        check(load().u3dg_trainer_time_steps(self._h, count, C.byref(ms)))
        return float(ms.value)

    def set_intersection_capacity(self, capacity: int) -> None:
        check(load().u3dg_trainer_set_intersection_capacity(self._h, int(capacity)))

    def replays(self) -> int:
        r = C.c_int()
        check(load().u3dg_trainer_replays(self._h, C.byref(r)))
        return r.value

    def set_graphs(self, enable: bool) -> None:
        """Graph launches of 10-step runs without densification (identical results either way)."""
        check(load().u3dg_trainer_set_graphs(self._h, 1 if enable else 0))

    def graph_launches(self) -> int:
        v = C.c_longlong()
        check(load().u3dg_trainer_graph_launches(self._h, C.byref(v)))
        return int(v.value)

    def set_raster_schedule(self, forward_block: int = 8, forward_depth: int = 1, backward_depth: int = 1) -> None:
        """Compositing schedule (identical results for every setting): the forward kernel's pixel block
        edge for tiles of 16 and 32 pixels (8 or 16) and the list entries each forward / backward
        thread stages per shared-memory batch (1 or 2)."""
        check(load().u3dg_trainer_set_raster_schedule(self._h, forward_block, forward_depth, backward_depth))

    def set_tile_culling(self, enable: bool) -> None:
        """List Gaussians only in tiles their contributing ellipse reaches (default on; same models)."""
        check(load().u3dg_trainer_set_tile_culling(self._h, 1 if enable else 0))

    def set_profiling(self, enable: bool) -> None:
        check(load().u3dg_trainer_set_profiling(self._h, 1 if enable else 0))

    def phase_times(self) -> dict:
        t = _abi.PhaseTimes()
        check(load().u3dg_trainer_phase_times(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in t._fields_}


class Batch:
    """Many scenes trained at once on one GPU (u3dg_batch_*; no reference counterpart).

    scenes: a list of (initial GaussianModel, images, scene extent, TrainOptions). Each scene keeps its
    own trainer and stream; step() advances every scene by `count` iterations, interleaving them so
    their kernels run concurrently. With autotune, each scene's tile size (8, 16 or 32) is picked at
    creation from short timed runs."""

    def __init__(self, scenes, autotune: bool = True):
        L = load()
        S = len(scenes)
        if S == 0:
            raise ValueError("no scenes")
        models = (_abi.ModelView * S)()
        images = (C.POINTER(_abi.Image) * S)()
        counts = (C.c_int32 * S)()
        extents = (C.c_float * S)()
        opts = (_abi.TrainOptions * S)()
        keep = []
        self._scenes = []
        for k, (init, imgs, extent, options) in enumerate(scenes):
            imgs = list(imgs)
            models[k] = init.view()
            arr, kp = images_struct(imgs)
            keep += [init, arr, kp]
            images[k] = C.cast(arr, C.POINTER(_abi.Image))
            counts[k] = len(imgs)
            extents[k] = float(extent)
            options = options or TrainOptions()
            opts[k] = options.struct()
            self._scenes.append((imgs, options))
        h = C.c_void_p()
        check(L.u3dg_batch_create(models, images, counts, extents, opts, S, 1 if autotune else 0, C.byref(h)))
        self._h = h
        del keep

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            load().u3dg_batch_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    def __len__(self) -> int:
        return len(self._scenes)

    def step(self, count: int = 1) -> None:
        check(load().u3dg_batch_step(self._h, count))

    def time_steps(self, count: int) -> float:
        """Device milliseconds of `count` iterations of every scene."""
        ms = C.c_float()
        check(load().u3dg_batch_time_steps(self._h, count, C.byref(ms)))
        return float(ms.value)

    def tile_size(self, scene: int):
        """(tile size, tuned ms per step) of a scene."""
        tile, ms = C.c_int32(), C.c_float()
        check(load().u3dg_batch_tile_size(self._h, scene, C.byref(tile), C.byref(ms)))
        return int(tile.value), float(ms.value)

    def schedule(self, scene: int):
        """(tile size, (forward block, forward depth, backward depth), tuned ms per step) of a scene;
        the middle triple is the argument list of Trainer.set_raster_schedule."""
        tile, fb, fd, bd, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_float()
        check(load().u3dg_batch_schedule(self._h, scene, C.byref(tile), C.byref(fb), C.byref(fd), C.byref(bd),
                                         C.byref(ms)))
        return int(tile.value), (int(fb.value), int(fd.value), int(bd.value)), float(ms.value)

    def graph_launches(self):
        """(rounds run as one graph launch holding every scene, recordings of that graph)."""
        launches, captures = C.c_longlong(), C.c_longlong()
        check(load().u3dg_batch_graph_launches(self._h, C.byref(launches), C.byref(captures)))
        return int(launches.value), int(captures.value)

    def trainer(self, scene: int) -> "Trainer":
        """The scene's trainer (borrowed: valid while this batch is alive)."""
        h = C.c_void_p()
        check(load().u3dg_batch_trainer(self._h, scene, C.byref(h)))
        t = Trainer.__new__(Trainer)
        t._h = h
        t._images, t._options = self._scenes[scene]
        t._owner = self
        return t


class Rasterizer:
    """GPU drop-in for u3d::Rasterizer (forward keeps the state backward needs)."""

    def __init__(self, pool=None):
        h = C.c_void_p()
        check(load().u3dg_rasterizer_create(C.byref(h)))
        self._h = h
        self._n = 0
        self._cam = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            load().u3dg_rasterizer_destroy(h)
            self._h = None

    def forward(self, model: GaussianModel, camera, settings: RasterSettings | None = None) -> np.ndarray:
        cs, ss = _cam(camera), _settings(settings)
        rgb = np.zeros((cs.height, cs.width, 3), np.float32)
        mv = model.view()
        check(load().u3dg_rasterizer_forward(self._h, C.byref(mv), C.byref(cs), C.byref(ss), _abi.fptr(rgb)))
        self._n, self._cam, self._ss = model.size(), cs, ss
        return rgb

    def backward(self, model: GaussianModel, dl_drgb: np.ndarray, grads: GaussianModel | None = None,
                 mean2d_grad_ndc: np.ndarray | None = None):
        """ADDS dL/dparams into `grads` (zeros if None) and |dL/dmean2d| into mean2d_grad_ndc; returns grads."""
        g = grads if grads is not None else GaussianModel.zeros(model.size())
        mv, gv = model.view(), g.view()
        dl = np.ascontiguousarray(dl_drgb, np.float32)
        ndc = _abi.fptr(mean2d_grad_ndc) if mean2d_grad_ndc is not None else None
        check(load().u3dg_rasterizer_backward(self._h, C.byref(mv), _abi.fptr(dl), C.byref(gv), ndc))
        return g

    def radii(self) -> np.ndarray:
        out = np.zeros(self._n, np.int32)
        check(load().u3dg_rasterizer_radii(self._h, _abi.iptr(out), self._n))
        return out

    def projection(self) -> dict:
        n = self._n
        out = dict(mean2d=np.zeros((n, 2), np.float32), conic=np.zeros((n, 3), np.float32),
                   cov2d=np.zeros((n, 3), np.float32), depth=np.zeros(n, np.float32), rgb=np.zeros((n, 3), np.float32),
                   alpha=np.zeros(n, np.float32), rect=np.zeros((n, 4), np.int32), flags=np.zeros(n, np.uint8))
        check(load().u3dg_rasterizer_projection(self._h, n, *(_abi.fptr(out[k]) for k in
                                                              ("mean2d", "conic", "cov2d", "depth", "rgb", "alpha")),
                                                _abi.iptr(out["rect"]), out["flags"].ctypes.data_as(_abi.u8p)))
        out["radius"] = self.radii()
        return out

    def tiles(self):
        tx, ty, L = C.c_int(), C.c_int(), C.c_size_t()
        check(load().u3dg_rasterizer_tiles(self._h, C.byref(tx), C.byref(ty), None, 0, None, 0, C.byref(L)))
        offsets = np.zeros(tx.value * ty.value + 1, np.int32)
        lst = np.zeros(max(L.value, 1), np.int32)
        check(load().u3dg_rasterizer_tiles(self._h, None, None, _abi.iptr(offsets), offsets.size, _abi.iptr(lst),
                                           lst.size, C.byref(L)))
        return offsets, lst[: L.value]

    def pixel_state(self):
        P = self._cam.width * self._cam.height
        ft = np.zeros(P, np.float32)
        nc = np.zeros(P, np.int32)
        check(load().u3dg_rasterizer_pixel_state(self._h, _abi.fptr(ft), _abi.iptr(nc), P))
        return ft, nc

    def set_tile_culling(self, enable: bool) -> None:
        """List each Gaussian only in the tiles its contributing ellipse reaches (the trainers'
        default); the lists become subsequences of the reference's, results are unchanged."""
        check(load().u3dg_rasterizer_set_tile_culling(self._h, 1 if enable else 0))


def binTiles(depth, radius, rect, tiles_x: int, tiles_y: int):
    """GPU tile binning of given projected records (Rasterizer::binTiles); returns (offsets, list)."""
    depth = np.ascontiguousarray(depth, np.float32)
    radius = np.ascontiguousarray(radius, np.int32)
    rect = np.ascontiguousarray(rect, np.int32).reshape(-1)
    offsets = np.zeros(tiles_x * tiles_y + 1, np.int32)
    L = C.c_size_t()
    check(load().u3dg_bin_tiles(_abi.fptr(depth), _abi.iptr(radius), _abi.iptr(rect), depth.size, tiles_x, tiles_y,
                                _abi.iptr(offsets), None, 0, C.byref(L)))
    lst = np.zeros(max(L.value, 1), np.int32)
    check(load().u3dg_bin_tiles(_abi.fptr(depth), _abi.iptr(radius), _abi.iptr(rect), depth.size, tiles_x, tiles_y,
                                _abi.iptr(offsets), _abi.iptr(lst), lst.size, C.byref(L)))
    return offsets, lst[: L.value]


def photometricLoss(render: np.ndarray, target: np.ndarray, width: int, height: int, ssim_lambda: float):
    """Returns (LossValue, dLoss/drender) (Loss.h:18-19)."""
    r = np.ascontiguousarray(render, np.float32).reshape(-1)
    t = np.ascontiguousarray(target, np.float32).reshape(-1)
    g = np.zeros_like(r)
    out = _abi.LossValue()
    check(load().u3dg_photometric_loss(_abi.fptr(r), _abi.fptr(t), width, height, float(ssim_lambda), _abi.fptr(g),
                                       C.byref(out)))
    return LossValue(out.total, out.l1, out.ssim), g.reshape(np.shape(render))


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32).reshape(-1)
    b = np.ascontiguousarray(b, np.float32).reshape(-1)
    out = C.c_float()
    check(load().u3dg_psnr(_abi.fptr(a), _abi.fptr(b), a.size, C.byref(out)))
    return float(out.value)


class Adam:
    """u3d::Adam with the moments on the GPU (params are host arrays updated in place)."""

    def __init__(self):
        self._h = None
        self._n = 0

    def __del__(self):
        if getattr(self, "_h", None):
            load().u3dg_adam_destroy(self._h)
            self._h = None

    def reset(self, n: int) -> None:
        self.__del__()
        h = C.c_void_p()
        check(load().u3dg_adam_create(n, C.byref(h)))
        self._h, self._n = h, n

    def step(self, params: GaussianModel, grads: GaussianModel, lr) -> None:
        pv, gv = params.view(), grads.view()
        lrs = lr.struct()
        check(load().u3dg_adam_step(self._h, C.byref(pv), C.byref(gv), C.byref(lrs)))

    def compact(self, keep) -> None:
        k = np.ascontiguousarray(keep, np.uint8)
        check(load().u3dg_adam_compact(self._h, k.ctypes.data_as(_abi.u8p), k.size))
        self._n = int(np.count_nonzero(k))

    def grow(self, count: int) -> None:
        check(load().u3dg_adam_grow(self._h, count))
        self._n += count

    def resetOpacityMoments(self) -> None:
        check(load().u3dg_adam_reset_opacity_moments(self._h))

    def moments(self):
        m, v = GaussianModel.zeros(self._n), GaussianModel.zeros(self._n)
        mv, vv = m.view(), v.view()
        check(load().u3dg_adam_moments(self._h, C.byref(mv), C.byref(vv)))
        return m, v


def densifyAndPrune(model: GaussianModel, m: GaussianModel, v: GaussianModel, grad_accum, grad_count, extent: float,
                    options: TrainOptions, opacity_was_reset: bool, seed: int):
    """Trainer::densifyAndPrune on a given state (GPU path of the trainer). Returns (model, m, v, counts)."""
    cap = max(options.max_gaussians, model.size())
    bufs = [GaussianModel.zeros(cap) for _ in range(3)]
    for dst, src in zip(bufs, (model, m, v)):
        for name, _ in _abi.GROUPS:
            getattr(dst, name)[: src.size()] = getattr(src, name)
    views = [b.view() for b in bufs]
    for vw in views:
        vw.count = model.size()
    count = C.c_size_t()
    counts = np.zeros(3, np.int32)
    opt = options.struct()
    check(load().u3dg_densify_and_prune(C.byref(views[0]), C.byref(views[1]), C.byref(views[2]),
                                        _abi.fptr(np.ascontiguousarray(grad_accum, np.float32)),
                                        _abi.iptr(np.ascontiguousarray(grad_count, np.int32)), cap, float(extent),
                                        C.byref(opt), int(bool(opacity_was_reset)), seed, C.byref(count),
                                        _abi.iptr(counts)))
    k = count.value
    out = [GaussianModel(*(getattr(b, name)[:k].copy() for name, _ in _abi.GROUPS)) for b in bufs]
    return out[0], out[1], out[2], counts


def initGaussiansFromPoints(xyz: np.ndarray, rgb: np.ndarray | None = None) -> GaussianModel:
    """initGaussiansFromPoints (GaussianModel.cpp:68-144): hash-grid 3-NN scales, identity rotations,
    opacity 0.1, colours from rgb (grey without). The neighbour search runs on the GPU."""
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1)
    n = x.size // 3
    out = GaussianModel.zeros(n)
    v = out.view()
    rp = _abi.fptr(np.ascontiguousarray(rgb, np.float32).reshape(-1)) if rgb is not None else None
    check(load().u3dg_init_gaussians_from_points(_abi.fptr(x), rp, n, C.byref(v)))
    return out


class PlyResult:
    def __init__(self):
        self.error = ""


def writeSplatPly(path: str, model: GaussianModel, result: PlyResult | None = None) -> bool:
    v = model.view()
    st = load().u3dg_write_splat_ply(str(path).encode(), C.byref(v))
    if st != _abi.OK and result is not None:
        result.error = load().u3dg_last_error().decode()
    return st == _abi.OK


def writeSplatPlySh(path: str, model: GaussianModel, sh_rest: np.ndarray, degree: int,
                    result: PlyResult | None = None) -> bool:
    """writeSplatPly plus f_rest_* properties for SH degree 1..3 (u3dg_write_splat_ply_sh). sh_rest:
    (n, K, 3) float32, K = (degree + 1)^2 - 1, the layout renderViewsSh takes."""
    sh = np.ascontiguousarray(sh_rest, np.float32)
    v = model.view()
    st = load().u3dg_write_splat_ply_sh(str(path).encode(), C.byref(v), _abi.fptr(sh), int(degree))
    if st != _abi.OK and result is not None:
        result.error = load().u3dg_last_error().decode()
    return st == _abi.OK


def readSplatPly(path: str, result: PlyResult | None = None):
    """Returns (model or None, is_splat)."""
    L = load()
    n = C.c_size_t()
    is_splat = C.c_int()
    st = L.u3dg_read_splat_ply(str(path).encode(), None, 0, C.byref(n), C.byref(is_splat))
    if st != _abi.OK:
        if result is not None:
            result.error = L.u3dg_last_error().decode()
        return None, False
    m = GaussianModel.zeros(n.value)
    v = m.view()
    check(L.u3dg_read_splat_ply(str(path).encode(), C.byref(v), n.value, C.byref(n), C.byref(is_splat)))
    return m, bool(is_splat.value)


def _box(b) -> _abi.CropBox:
    if isinstance(b, _abi.CropBox):
        return b
    lo, hi = b
    out = _abi.CropBox()
    for k in range(3):
        out.min[k], out.max[k] = float(lo[k]), float(hi[k])
    return out


def _unbox(b: _abi.CropBox):
    return np.array(list(b.min), np.float32), np.array(list(b.max), np.float32)


def cropModel(model: GaussianModel, box, min_opacity: float = 0.0) -> GaussianModel:
    """cropModel (Crop.h:21-23) on the GPU; box = (min xyz, max xyz)."""
    mv, cb, n = model.view(), _box(box), C.c_size_t()
    check(load().u3dg_crop_model(C.byref(mv), C.byref(cb), float(min_opacity), None, 0, C.byref(n)))
    out = GaussianModel.zeros(n.value)
    ov = out.view()
    check(load().u3dg_crop_model(C.byref(mv), C.byref(cb), float(min_opacity), C.byref(ov), n.value, C.byref(n)))
    return out


def suggestCropBox(model: GaussianModel, low_fraction: float = 0.05, high_fraction: float = 0.95,
                   margin: float = 0.1):
    """suggestCropBox (Crop.h:25-31) on the GPU: (min xyz, max xyz)."""
    mv, out = model.view(), _abi.CropBox()
    check(load().u3dg_suggest_crop_box(C.byref(mv), low_fraction, high_fraction, margin, C.byref(out)))
    return _unbox(out)


def modelBounds(model: GaussianModel):
    """modelBounds (Crop.h:33-35) on the GPU: (min xyz, max xyz)."""
    mv, out = model.view(), _abi.CropBox()
    check(load().u3dg_model_bounds(C.byref(mv), C.byref(out)))
    return _unbox(out)


def renderSh(model: GaussianModel, sh_rest: np.ndarray | None, degree: int, camera,
             settings: RasterSettings | None = None) -> np.ndarray:
    """Render with SH colours of degree 0..3 (ground-truth rendering of the synthetic scenes)."""
    cs, ss = _cam(camera), _settings(settings)
    rgb = np.zeros((cs.height, cs.width, 3), np.float32)
    mv = model.view()
    shp = _abi.fptr(np.ascontiguousarray(sh_rest, np.float32).reshape(-1)) if (sh_rest is not None and degree > 0) \
        else None
    check(load().u3dg_render_sh(C.byref(mv), shp, int(degree), C.byref(cs), C.byref(ss), _abi.fptr(rgb)))
    return rgb


def renderViewsSh(model: GaussianModel, sh_rest: np.ndarray | None, degree: int, cameras,
                  settings: RasterSettings | None = None) -> list:
    """Quantised (uint8) SH renders of many views with the model uploaded once: training targets."""
    cams = (_abi.Camera * max(1, len(cameras)))()
    sizes = []
    for k, c in enumerate(cameras):
        cams[k] = _cam(c)
        sizes.append((cams[k].height, cams[k].width))
    total = sum(h * w * 3 for h, w in sizes)
    out = np.zeros(max(total, 1), np.uint8)
    mv = model.view()
    ss = _settings(settings)
    shp = _abi.fptr(np.ascontiguousarray(sh_rest, np.float32).reshape(-1)) if (sh_rest is not None and degree > 0) \
        else None
    check(load().u3dg_render_views_sh(C.byref(mv), shp, int(degree), cams, len(cameras), C.byref(ss),
                                      out.ctypes.data_as(_abi.u8p)))
    res, o = [], 0
    for h, w in sizes:
        res.append(out[o:o + h * w * 3].reshape(h, w, 3).copy())
        o += h * w * 3
    return res


MLP_INPUTS, MLP_OUTPUTS, MLP_PARAMS = 134, 11, 51723


class WarmStartNet:
    """The learned warm-start MLP (134 -> 128 -> 128 -> 128 -> 11, FP32) on the GPU."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        h = C.c_void_p()
        p = None
        if params is not None:
            params = np.ascontiguousarray(params, np.float32).reshape(-1)
            if params.size != MLP_PARAMS:
                raise ValueError(f"expected {MLP_PARAMS} parameters, got {params.size}")
            p = _abi.fptr(params)
        check(load().u3dg_mlp_create(p, seed, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            load().u3dg_mlp_destroy(h)
            self._h = None

    def params(self) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, np.float32)
        check(load().u3dg_mlp_params(self._h, _abi.fptr(out)))
        return out

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_INPUTS)
        y = np.zeros((x.shape[0], MLP_OUTPUTS), np.float32)
        check(load().u3dg_mlp_forward(self._h, _abi.fptr(x), x.shape[0], _abi.fptr(y)))
        return y

    def loss_grad(self, x, t, weights=None):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_INPUTS)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, MLP_OUTPUTS)
        w = _abi.fptr(np.ascontiguousarray(weights, np.float32)) if weights is not None else None
        loss = C.c_float()
        grad = np.zeros(MLP_PARAMS, np.float32)
        check(load().u3dg_mlp_loss_grad(self._h, _abi.fptr(x), _abi.fptr(t), w, x.shape[0], C.byref(loss),
                                        _abi.fptr(grad)))
        return float(loss.value), grad

    def train(self, x, t, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0, weights=None):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_INPUTS)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, MLP_OUTPUTS)
        w = _abi.fptr(np.ascontiguousarray(weights, np.float32)) if weights is not None else None
        losses = np.zeros(max(epochs, 1), np.float32)
        check(load().u3dg_mlp_train(self._h, _abi.fptr(x), _abi.fptr(t), w, x.shape[0], epochs, batch, lr, seed,
                                    _abi.fptr(losses)))
        return losses[:epochs]


def knn(queries: np.ndarray, points: np.ndarray, k: int, exclude_self: bool = False):
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 3)
    p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    idx = np.zeros((q.shape[0], k), np.int32)
    d2 = np.zeros((q.shape[0], k), np.float32)
    check(load().u3dg_knn(_abi.fptr(q), q.shape[0], _abi.fptr(p), p.shape[0], k, int(exclude_self),
                          _abi.iptr(idx), _abi.fptr(d2)))
    return idx, d2


def warmstartFeatures(xyz, rgb, images) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    rgbp = _abi.fptr(np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)) if rgb is not None else None
    arr, keep = images_struct(images)
    f = np.zeros((xyz.shape[0], MLP_INPUTS), np.float32)
    check(load().u3dg_warmstart_features(_abi.fptr(xyz), rgbp, xyz.shape[0], arr, len(images), _abi.fptr(f)))
    del keep
    return f


def warmstartInit(net: WarmStartNet | None, xyz, rgb, images) -> GaussianModel:
    """Initial model through the network; net=None gives initGaussiansFromPoints exactly."""
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    rgbp = _abi.fptr(np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)) if rgb is not None else None
    arr, keep = images_struct(images)
    out = GaussianModel.zeros(xyz.shape[0])
    v = out.view()
    check(load().u3dg_warmstart_init(net._h if net is not None else None, _abi.fptr(xyz), rgbp, xyz.shape[0], arr,
                                     len(images), C.byref(v)))
    del keep
    return out


__all__ = ["Trainer", "Rasterizer", "binTiles", "photometricLoss", "psnr", "Adam", "densifyAndPrune",
           "initGaussiansFromPoints", "writeSplatPly", "readSplatPly", "renderSh", "U3dgError", "TrainImage"]
