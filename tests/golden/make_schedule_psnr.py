"""Records the reference CPU trainer's PSNR after full preset schedules into schedule_psnr.json.

For each preset (seed 0) the script builds the seeded scene (scenes.make_scene), renders the training
targets with the CPU oracle (the reference's forward restated, SH degree 3) and quantises them as
TrainImage::quantize does, initialises with the reference's own initGaussiansFromPoints, and runs the
reference Trainer (oracle/_ref/libu3dref.so, built from the reference sources) over the preset's
whole schedule (TrainOptions::forIterations plus the preset's Gaussian cap and, for Balanced, the
explicit opacity reset at 3000; Trainer.cpp:26-35, 53-103). It records evaluatePsnr
(Trainer.cpp:180-192) and the Gaussian count after every run.

With more than one worker thread the reference is not deterministic (its backward adds per-Gaussian
gradients from all threads in arrival order), so each preset is run several times and the GPU tests
compare against the mean. The SHA-256 of the quantised targets is stored too: the GPU test renders the
same targets on the CPU and checks the hash before it compares PSNRs.

    python tests/golden/make_schedule_psnr.py fast:5 balanced:3 high:1 [--threads 0]

Runs append to the existing file; a preset's entry keeps every run recorded so far.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import platform
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.binding import Oracle, Reference  # noqa: E402
from univeral_3d_reconstruction_system_b200.scenes import make_scene  # noqa: E402
from univeral_3d_reconstruction_system_b200.types import RasterSettings, TrainImage  # noqa: E402

OUT = Path(__file__).resolve().parent / "schedule_psnr.json"


def render_targets_cpu(sc, threads: int | None = None):
    """The preset's quantised training targets rendered by the CPU oracle (SH degree 3)."""
    orc = Oracle()
    st = RasterSettings()
    imgs = [TrainImage.quantize(orc.render(sc.truth, c, st, sc.sh_rest, 3, threads=threads)) for c in sc.cameras]
    sc.images = [TrainImage(c, im) for c, im in zip(sc.cameras, imgs)]
    return sc.images


def images_sha256(images) -> str:
    h = hashlib.sha256()
    for im in images:
        h.update(np.ascontiguousarray(im.rgb, np.uint8).tobytes())
    return h.hexdigest()


def load() -> dict:
    return json.loads(OUT.read_text()) if OUT.exists() else {}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("runs", nargs="+", help="preset:count, e.g. fast:5")
    ap.add_argument("--threads", type=int, default=0, help="reference worker threads (0: all host threads)")
    args = ap.parse_args()
    ref = Reference()
    threads = ref.pool_threads(args.threads)
    for item in args.runs:
        preset, _, count = item.partition(":")
        count = int(count or 1)
        sc = make_scene(preset, 0)
        t0 = time.time()
        render_targets_cpu(sc)
        digest = images_sha256(sc.images)
        print(f"{preset}: targets rendered in {time.time() - t0:.1f} s, sha256 {digest[:16]}", flush=True)
        init = ref.init_from_points(sc.init_xyz, sc.init_rgb)
        opt = sc.options()
        for k in range(count):
            tr = ref.trainer(init, sc.images, sc.extent, opt, threads=args.threads)
            t0 = time.perf_counter()
            tr.step(opt.iterations)
            secs = time.perf_counter() - t0
            psnr, n = tr.evaluate_psnr(), tr.size()
            del tr
            data = load()
            entry = data.setdefault(preset, {"seed": 0, "iterations": opt.iterations,
                                             "max_gaussians": opt.max_gaussians,
                                             "opacity_reset_interval": opt.opacity_reset_interval,
                                             "refine_stop": opt.refine_stop, "targets_sha256": digest, "runs": []})
            if entry["targets_sha256"] != digest:
                raise SystemExit(f"{preset}: targets differ from the recorded ones ({entry['targets_sha256'][:16]})")
            entry["runs"].append({"psnr": round(psnr, 5), "gaussians": n, "seconds": round(secs, 1),
                                  "threads": threads, "host": platform.processor() or platform.machine(),
                                  "cpus": os.cpu_count()})
            ps = [r["psnr"] for r in entry["runs"]]
            entry["mean_psnr"] = round(float(np.mean(ps)), 5)
            entry["min_psnr"], entry["max_psnr"] = min(ps), max(ps)
            OUT.write_text(json.dumps(data, indent=1) + "\n")
            print(f"{preset} run {k + 1}/{count}: PSNR {psnr:.4f} dB, {n} Gaussians, {secs:.0f} s "
                  f"({threads} threads); mean of {len(ps)}: {entry['mean_psnr']:.4f}", flush=True)


if __name__ == "__main__":
    main()
