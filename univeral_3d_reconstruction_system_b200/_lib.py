"""Loads libu3dg.so (the in-tree CUDA library) and declares the C ABI of include/u3dg.h.

There is no fallback: if the library is missing, importing the binding raises, and calls that
need a GPU fail with U3dgError(ERR_NO_DEVICE) when none is present.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import _abi

LIB_PATH = Path(__file__).resolve().parent / "libu3dg.so"


class U3dgError(RuntimeError):
    """A non-OK status from the C ABI; .status holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"u3dg status {status}: {message}")
        self.status = status


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_MV = C.POINTER(_abi.ModelView)
_CAM = C.POINTER(_abi.Camera)
_ST = C.POINTER(_abi.RasterSettings)
_OPT = C.POINTER(_abi.TrainOptions)
_F = _abi.f32p
_I = _abi.i32p
_SZ = C.POINTER(C.c_size_t)

# name: (restype, argtypes). Every entry point of include/u3dg.h.
SIGNATURES = {
    "u3dg_last_error": (C.c_char_p, []),
    "u3dg_abi_version": (C.c_int, []),
    "u3dg_launch_count": (C.c_uint64, []),
    "u3dg_device_count": (C.c_int, []),
    "u3dg_set_device": (C.c_int, [C.c_int]),
    "u3dg_raster_settings_default": (None, [_ST]),
    "u3dg_train_options_default": (None, [_OPT]),
    "u3dg_train_options_for_iterations": (None, [C.c_int, _OPT]),
    "u3dg_trainer_create": (C.c_int, [_MV, C.POINTER(_abi.Image), C.c_int, C.c_float, _OPT, _PP]),
    "u3dg_trainer_create_background_upload": (C.c_int, [_MV, C.POINTER(_abi.Image), C.c_int, C.c_float, _OPT, _PP]),
    "u3dg_trainer_wait_uploads": (C.c_int, [_P]),
    "u3dg_trainer_step": (C.c_int, [_P, C.c_int]),
    "u3dg_trainer_done": (C.c_int, [_P, _I]),
    "u3dg_trainer_iteration": (C.c_int, [_P, _I]),
    "u3dg_trainer_stats": (C.c_int, [_P, C.POINTER(_abi.TrainStats)]),
    "u3dg_trainer_size": (C.c_int, [_P, _SZ]),
    "u3dg_trainer_download": (C.c_int, [_P, _MV, C.c_size_t, _SZ]),
    "u3dg_trainer_eval_psnr": (C.c_int, [_P, _F]),
    "u3dg_trainer_write_splat_ply": (C.c_int, [_P, C.c_char_p]),
    "u3dg_trainer_render": (C.c_int, [_P, _CAM, _F]),
    "u3dg_trainer_stream": (C.c_int, [_P, _PP]),
    "u3dg_trainer_synchronize": (C.c_int, [_P]),
    "u3dg_trainer_set_profiling": (C.c_int, [_P, C.c_int]),
    "u3dg_trainer_phase_times": (C.c_int, [_P, C.POINTER(_abi.PhaseTimes)]),
    "u3dg_trainer_time_steps": (C.c_int, [_P, C.c_int, _F]),
    "u3dg_trainer_set_intersection_capacity": (C.c_int, [_P, C.c_size_t]),
    "u3dg_trainer_replays": (C.c_int, [_P, _I]),
    "u3dg_trainer_set_graphs": (C.c_int, [_P, C.c_int]),
    "u3dg_trainer_graph_launches": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    "u3dg_trainer_set_raster_schedule": (C.c_int, [_P, C.c_int, C.c_int, C.c_int]),
    "u3dg_trainer_set_tile_culling": (C.c_int, [_P, C.c_int]),
    "u3dg_trainer_destroy": (None, [_P]),
    "u3dg_rasterizer_create": (C.c_int, [_PP]),
    "u3dg_rasterizer_forward": (C.c_int, [_P, _MV, _CAM, _ST, _F]),
    "u3dg_rasterizer_backward": (C.c_int, [_P, _MV, _F, _MV, _F]),
    "u3dg_rasterizer_radii": (C.c_int, [_P, _I, C.c_size_t]),
    "u3dg_rasterizer_projection": (C.c_int, [_P, C.c_size_t, _F, _F, _F, _F, _F, _F, _I, _abi.u8p]),
    "u3dg_rasterizer_tiles": (C.c_int, [_P, _I, _I, _I, C.c_size_t, _I, C.c_size_t, _SZ]),
    "u3dg_rasterizer_pixel_state": (C.c_int, [_P, _F, _I, C.c_size_t]),
    "u3dg_rasterizer_set_tile_culling": (C.c_int, [_P, C.c_int]),
    "u3dg_rasterizer_destroy": (None, [_P]),
    "u3dg_bin_tiles": (C.c_int, [_F, _I, _I, C.c_size_t, C.c_int, C.c_int, _I, _I, C.c_size_t, _SZ]),
    "u3dg_densify_and_prune": (C.c_int, [_MV, _MV, _MV, _F, _I, C.c_size_t, C.c_float, _OPT, C.c_int, C.c_uint,
                                         _SZ, _I]),
    "u3dg_batch_create": (C.c_int, [_MV, C.POINTER(C.POINTER(_abi.Image)), _I, _F, _OPT, C.c_int, C.c_int, _PP]),
    "u3dg_batch_step": (C.c_int, [_P, C.c_int]),
    "u3dg_batch_time_steps": (C.c_int, [_P, C.c_int, _F]),
    "u3dg_batch_size": (C.c_int, [_P, _I]),
    "u3dg_batch_trainer": (C.c_int, [_P, C.c_int, _PP]),
    "u3dg_batch_tile_size": (C.c_int, [_P, C.c_int, _I, _F]),
    "u3dg_batch_schedule": (C.c_int, [_P, C.c_int, _I, _I, _I, _I, _F]),
    "u3dg_batch_graph_launches": (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "u3dg_batch_destroy": (None, [_P]),
    "u3dg_photometric_loss": (C.c_int, [_F, _F, C.c_int, C.c_int, C.c_float, _F, C.POINTER(_abi.LossValue)]),
    "u3dg_psnr": (C.c_int, [_F, _F, C.c_size_t, _F]),
    "u3dg_photometric_loss_noalloc": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_float, _P, C.POINTER(_abi.LossValue),
                                                _P]),
    "u3dg_adam_create": (C.c_int, [C.c_size_t, _PP]),
    "u3dg_adam_step": (C.c_int, [_P, _MV, _MV, C.POINTER(_abi.LearningRates)]),
    "u3dg_adam_compact": (C.c_int, [_P, _abi.u8p, C.c_size_t]),
    "u3dg_adam_grow": (C.c_int, [_P, C.c_size_t]),
    "u3dg_adam_reset_opacity_moments": (C.c_int, [_P]),
    "u3dg_adam_moments": (C.c_int, [_P, _MV, _MV]),
    "u3dg_adam_destroy": (None, [_P]),
    "u3dg_init_gaussians_from_points": (C.c_int, [_F, _F, C.c_size_t, _MV]),
    "u3dg_write_splat_ply": (C.c_int, [C.c_char_p, _MV]),
    "u3dg_write_splat_ply_sh": (C.c_int, [C.c_char_p, _MV, _F, C.c_int]),
    "u3dg_crop_model": (C.c_int, [_MV, C.POINTER(_abi.CropBox), C.c_float, _MV, C.c_size_t, _SZ]),
    "u3dg_suggest_crop_box": (C.c_int, [_MV, C.c_float, C.c_float, C.c_float, C.POINTER(_abi.CropBox)]),
    "u3dg_model_bounds": (C.c_int, [_MV, C.POINTER(_abi.CropBox)]),
    "u3dg_trainer_crop": (C.c_int, [_P, C.POINTER(_abi.CropBox), C.c_float]),
    "u3dg_trainer_suggest_crop_box": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, C.POINTER(_abi.CropBox)]),
    "u3dg_read_splat_ply": (C.c_int, [C.c_char_p, _MV, C.c_size_t, _SZ, _I]),
    "u3dg_render_sh": (C.c_int, [_MV, _F, C.c_int, _CAM, _ST, _F]),
    "u3dg_render_views_sh": (C.c_int, [_MV, _F, C.c_int, _CAM, C.c_int, _ST, _abi.u8p]),
    "u3dg_mlp_param_count": (C.c_int, []),
    "u3dg_mlp_create": (C.c_int, [_F, C.c_uint, _PP]),
    "u3dg_mlp_params": (C.c_int, [_P, _F]),
    "u3dg_mlp_forward": (C.c_int, [_P, _F, C.c_size_t, _F]),
    "u3dg_mlp_loss_grad": (C.c_int, [_P, _F, _F, _F, C.c_size_t, _F, _F]),
    "u3dg_mlp_train": (C.c_int, [_P, _F, _F, _F, C.c_size_t, C.c_int, C.c_int, C.c_float, C.c_uint, _F]),
    "u3dg_mlp_destroy": (None, [_P]),
    "u3dg_knn": (C.c_int, [_F, C.c_size_t, _F, C.c_size_t, C.c_int, C.c_int, _I, _F]),
    "u3dg_warmstart_features": (C.c_int, [_F, _F, C.c_size_t, C.POINTER(_abi.Image), C.c_int, _F]),
    "u3dg_warmstart_init": (C.c_int, [_P, _F, _F, C.c_size_t, C.POINTER(_abi.Image), C.c_int, _MV]),
}

_lib = None


def load():
    """The loaded library (raises if libu3dg.so was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
                               " or `make -C univeral_3d_reconstruction_system_b200/csrc`")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != _abi.OK:
        msg = load().u3dg_last_error()
        raise U3dgError(status, msg.decode() if msg else "")


def device_count() -> int:
    return int(load().u3dg_device_count())


def loaded_path() -> str:
    return os.fspath(LIB_PATH)
