"""u3dg_photometric_loss_noalloc: the photometric loss on device buffers with no allocation in the
call, against the allocating entry point u3dg_photometric_loss, through the C ABI. Collected last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from univeral_3d_reconstruction_system_b200 import _abi

pytestmark = pytest.mark.gpu

TOL = 1e-6  # relative to the largest magnitude of each compared quantity


def _images(h, w, seed):
    rng = np.random.default_rng(seed)
    render = rng.uniform(0, 1, (h, w, 3)).astype(np.float32)
    target = np.clip(render + rng.normal(0, 0.1, render.shape), 0, 1).astype(np.float32)
    return render, target


def _allocating(lib, render, target, lam):
    h, w, _ = render.shape
    grad = np.zeros_like(render)
    out = _abi.LossValue()
    st = lib.u3dg_photometric_loss(_abi.fptr(render), _abi.fptr(target), w, h, lam, _abi.fptr(grad), C.byref(out))
    assert st == 0, lib.u3dg_last_error()
    return grad, (out.total, out.l1, out.ssim)


def _noalloc(lib, torch, render, target, lam, stream=None):
    h, w, _ = render.shape
    dr = torch.from_numpy(render).cuda()
    dt = torch.from_numpy(target).cuda()
    dg = torch.full_like(dr, float("nan"))
    torch.cuda.synchronize()
    out = _abi.LossValue()
    st = lib.u3dg_photometric_loss_noalloc(dr.data_ptr(), dt.data_ptr(), w, h, lam, dg.data_ptr(), C.byref(out),
                                           stream)
    assert st == 0, lib.u3dg_last_error()
    return dg.cpu().numpy(), (out.total, out.l1, out.ssim)


def _close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert np.max(np.abs(a - b)) <= TOL * max(float(np.max(np.abs(b))), 1e-30)


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    from univeral_3d_reconstruction_system_b200 import _lib
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _lib.load(), torch


@pytest.mark.parametrize("h,w,lam", [(61, 97, 0.2), (480, 640, 0.2), (33, 40, 0.0)])
def test_noalloc_matches_allocating_entry_twice(env, h, w, lam):
    lib, torch = env
    render, target = _images(h, w, seed=h * 1000 + w)
    ref_grad, ref_val = _allocating(lib, render, target, lam)
    for _ in range(2):  # two calls in a row reuse the same scratch
        grad, val = _noalloc(lib, torch, render, target, lam)
        _close(grad, ref_grad)
        _close(val, ref_val)


def test_noalloc_on_a_caller_stream(env):
    lib, torch = env
    render, target = _images(120, 160, seed=5)
    ref_grad, ref_val = _allocating(lib, render, target, 0.2)
    s = torch.cuda.Stream()
    for _ in range(2):
        grad, val = _noalloc(lib, torch, render, target, 0.2, stream=s.cuda_stream)
        _close(grad, ref_grad)
        _close(val, ref_val)


def test_noalloc_rejects_images_beyond_the_scratch(env):
    lib, torch = env
    for h, w in ((481, 640), (1, 307_201), (1, 307_200), (307_200, 1)):
        buf = torch.zeros(h * w * 3, device="cuda")
        out = _abi.LossValue()
        st = lib.u3dg_photometric_loss_noalloc(buf.data_ptr(), buf.data_ptr(), w, h, 0.2, buf.data_ptr(),
                                               C.byref(out), None)
        assert st == _abi.ERR_CAPACITY, (h, w, st)
        assert b"scratch" in lib.u3dg_last_error() or b"blocks" in lib.u3dg_last_error()
    st = lib.u3dg_photometric_loss_noalloc(None, None, 4, 4, 0.2, None, None, None)
    assert st == _abi.ERR_INVALID_ARG
