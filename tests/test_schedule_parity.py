"""PSNR after a full preset schedule: the GPU trainer against the reference's own CPU trainer.

The reference runs are recorded in tests/golden/schedule_psnr.json by tests/golden/make_schedule_psnr.py
(the reference Trainer built from its sources, all host threads, on the same seeded scene, targets and
initial points; Trainer.cpp:26-35, 53-192). The reference is not deterministic with more than one
thread (its backward adds per-Gaussian gradients from all threads in arrival order), so each preset was
run several times; the bar is the north star's: the GPU run's final evaluatePsnr within 0.1 dB of the
mean of the reference runs. The targets are rendered here exactly as the script rendered them (the CPU
oracle's SH-degree-3 forward, quantised), checked by their SHA-256.

Fast (2000 iterations), Balanced (4000, opacity reset at 3000) and High (forIterations(7000), max
300k) run by default; U3DG_PARITY_PRESETS selects a subset."""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import pytest

from univeral_3d_reconstruction_system_b200.scenes import make_scene

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from make_schedule_psnr import images_sha256, render_targets_cpu  # noqa: E402

FIXTURE = Path(__file__).resolve().parent / "golden" / "schedule_psnr.json"
RECORDED = json.loads(FIXTURE.read_text()) if FIXTURE.exists() else {}
PRESETS = [p for p in os.environ.get("U3DG_PARITY_PRESETS", "fast,balanced,high").split(",") if p]


@pytest.mark.gpu
@pytest.mark.slow
@pytest.mark.parametrize("preset", PRESETS)
def test_full_schedule_psnr_matches_the_reference(u3dg, oracle, preset):
    rec = RECORDED.get(preset)
    if not rec or not rec.get("runs"):
        pytest.skip(f"no recorded reference runs for {preset}")
    sc = make_scene(preset, 0)
    render_targets_cpu(sc, threads=os.cpu_count())
    assert images_sha256(sc.images) == rec["targets_sha256"], "targets differ from the recorded reference runs'"
    init = oracle.init_from_points(sc.init_xyz, sc.init_rgb)
    opt = sc.options()
    assert (opt.iterations, opt.max_gaussians, opt.opacity_reset_interval, opt.refine_stop) == \
        (rec["iterations"], rec["max_gaussians"], rec["opacity_reset_interval"], rec["refine_stop"])
    t = u3dg.Trainer(init, sc.images, sc.extent, opt)
    t0 = time.perf_counter()
    ms = t.time_steps(opt.iterations)
    wall = time.perf_counter() - t0
    psnr, n = t.evaluatePsnr(), t.size()
    ref = [r["psnr"] for r in rec["runs"]]
    mean = sum(ref) / len(ref)
    print(f"\n{preset}: {opt.iterations} iterations; GPU {ms / 1e3:.2f} s device ({wall:.2f} s wall), "
          f"PSNR {psnr:.4f} dB, {n} Gaussians; reference ({len(ref)} runs, {rec['runs'][0]['threads']} threads, "
          f"{rec['runs'][0]['seconds']:.0f} s each) {min(ref):.4f}-{max(ref):.4f} dB, mean {mean:.4f} dB "
          f"-> difference {psnr - mean:+.4f} dB")
    assert abs(psnr - mean) <= 0.1, (psnr, mean, ref)
