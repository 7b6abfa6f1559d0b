"""PSNR after a full preset schedule: the GPU trainer against the reference's own CPU trainer
(oracle/_ref, all host threads) on the same seeded scene, images and initial points.

The two runs are the same algorithm but not the same float trajectory: summation orders differ in the
gradients, and densification decisions on thresholds flip on the last bit. The reference itself is not
deterministic with more than one thread (its backward adds per-Gaussian gradients from all threads):
five runs of the Fast preset on 16-core hosts ended at 29.37, 29.40, 29.45, 29.46 and 29.52 dB. The GPU
run is deterministic for a given build and tile size, but equally valid summation orders (tile sizes
8 to 64, builds that add the partials differently) end at 29.33-29.53 dB. One reference run per test
therefore carries about +-0.08 dB of its own scatter, and the assertion allows 0.1 dB plus that: 0.2
dB. The
Fast preset runs by default; U3DG_PARITY_PRESETS=fast,balanced,high selects others (Balanced takes
about ten minutes of CPU time, High about an hour)."""
from __future__ import annotations

import os
import time

import pytest

from univeral_3d_reconstruction_system_b200.scenes import make_scene
from univeral_3d_reconstruction_system_b200.types import RasterSettings, TrainImage

PRESETS = [p for p in os.environ.get("U3DG_PARITY_PRESETS", "fast").split(",") if p]


@pytest.mark.gpu
@pytest.mark.slow
@pytest.mark.parametrize("preset", PRESETS)
def test_full_schedule_psnr_matches_the_reference(u3dg, reference, preset):
    sc = make_scene(preset, 0)
    imgs = u3dg.renderViewsSh(sc.truth, sc.sh_rest, 3, sc.cameras, RasterSettings())
    sc.images = [TrainImage(c, im) for c, im in zip(sc.cameras, imgs)]
    init = reference.init_from_points(sc.init_xyz, sc.init_rgb)
    opt = sc.options()
    t = u3dg.Trainer(init, sc.images, sc.extent, opt)
    gpu_ms = t.time_steps(opt.iterations)
    psnr_gpu, n_gpu = t.evaluatePsnr(), t.size()
    r = reference.trainer(init, sc.images, sc.extent, opt, threads=0)
    t0 = time.perf_counter()
    r.step(opt.iterations)
    cpu_s = time.perf_counter() - t0
    psnr_cpu, n_cpu = r.evaluate_psnr(), r.size()
    print(f"\n{preset}: {opt.iterations} iterations; GPU {gpu_ms / 1e3:.2f} s, PSNR {psnr_gpu:.4f} dB, {n_gpu} Gaussians; "
          f"reference CPU ({os.cpu_count()} threads) {cpu_s:.1f} s, PSNR {psnr_cpu:.4f} dB, {n_cpu} Gaussians")
    assert abs(psnr_gpu - psnr_cpu) <= 0.2, (psnr_gpu, psnr_cpu)
