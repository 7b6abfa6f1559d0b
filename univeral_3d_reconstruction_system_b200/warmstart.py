"""Learned warm-start for the trainer: label generation, network training and evaluation.

No reference counterpart. The reference starts every run from initGaussiansFromPoints
(engine/src/splat/GaussianModel.cpp:68-144): isotropic log-scale from the 3 nearest points, identity
rotation, opacity logit(0.1), DC colour from the point colour. Here a small network
(134 -> 128 -> 128 -> 128 -> 11, FP32, ReLU; kernels in csrc/warmstart.cu) predicts, per SfM point,
a better starting value of those attributes from the point's 16-NN neighbourhood and colour samples
of the views that see it. The plain initialisation stays the fallback (no network, or a non-finite
output) and the reference point (every comparison runs the same scene from both).

Labels (what "converged" means here): for a seeded synthetic scene, the plain trainer runs from the
plain initialisation for LABEL_ITERATIONS with densification and opacity reset switched off, so
every Gaussian is still the one its SfM point started as; the optimised attributes are the labels.
They are put in a canonical form before regression:
  log-scales   sorted in decreasing order, as residuals over the plain log-scale
  rotation     columns permuted with the scales, each column signed so that its largest component is
               positive, the last column flipped if that made a reflection; quaternion with w >= 0
  opacity      the logit, clipped to [-6, 6]
  colour       DC residual over the plain colour
The network is trained on the GPU by the library's own kernels (u3dg_mlp_train) on standardised
inputs; the standardisation is then folded into the first layer, so the shipped parameters read raw
features.

Evaluation (held-out seeds): the full schedule from the plain initialisation and from the warm start,
PSNR every `chunk` iterations (not timed), time-to-PSNR = initialisation wall time (host plain init,
or plain init + features + network inference) + device training time until the PSNR first reaches
the plain run's final PSNR.

Usage:  python -m univeral_3d_reconstruction_system_b200.warmstart train --out FILE
        (or under torchrun, one rank per GPU: the label scenes are shared over the ranks)
        python -m univeral_3d_reconstruction_system_b200.warmstart evaluate --weights FILE
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import api
from .scenes import PRESETS, Scene, make_scene
from .schedule import run_schedule
from .types import GaussianModel, RasterSettings, TrainImage, TrainOptions

DATA_DIR = Path(__file__).resolve().parent / "data"
# 51,723 little-endian float32 parameters (per layer W then b), readable from C/C++ with one fread;
# the training record (seeds, losses, held-out label losses) sits beside it as <name>.json.
WEIGHTS_PATH = DATA_DIR / "warmstart_high.f32"
LABEL_ITERATIONS = 3000
TRAIN_SEEDS = tuple(range(100, 164))  # 64 label scenes
EVAL_SEEDS = tuple(range(1000, 1008))  # 8 held-out scenes
OPACITY_CLIP = 6.0
# The training loss's default output weights (warmstart_host.cu): log-scales, quaternion, opacity, colour.
LOSS_WEIGHTS = np.array([1, 1, 1, 0.5, 0.5, 0.5, 0.5, 0.25, 1, 1, 1], np.float64)


# ------------------------------------------------------------------ scenes


def scene_spec(seed: int, base: str = "high"):
    """The High preset with its ground-truth count drawn log-uniform in [100k, 250k] from the seed."""
    rng = np.random.default_rng([seed, 7])
    gt = int(round(math.exp(rng.uniform(math.log(100e3), math.log(250e3)))))
    return dataclasses.replace(PRESETS[base], gt_count=gt)


def build_scene(seed: int, spec=None) -> Scene:
    sc = make_scene(spec if spec is not None else scene_spec(seed), seed)
    imgs = api.renderViewsSh(sc.truth, sc.sh_rest, sc.spec.sh_degree, sc.cameras, RasterSettings())
    sc.images = [TrainImage(c, im) for c, im in zip(sc.cameras, imgs)]
    return sc


def label_options(iterations: int = LABEL_ITERATIONS) -> TrainOptions:
    """TrainOptions::forIterations(iterations) with densification and opacity reset off."""
    o = TrainOptions.for_iterations(iterations)
    o.refine_start = iterations + 1
    o.refine_stop = iterations + 1
    o.opacity_reset_interval = 0
    return o


# ------------------------------------------------------------------ label canonical form


def quat_to_rot(q: np.ndarray) -> np.ndarray:
    q = np.asarray(q, np.float64).reshape(-1, 4)
    q = q / np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def rot_to_quat(R: np.ndarray) -> np.ndarray:
    """Unit quaternions (w, x, y, z) with w >= 0 from rotation matrices (largest-pivot method)."""
    R = np.asarray(R, np.float64).reshape(-1, 3, 3)
    tr = R[:, 0, 0] + R[:, 1, 1] + R[:, 2, 2]
    cand = np.stack([tr, R[:, 0, 0], R[:, 1, 1], R[:, 2, 2]], 1)
    piv = np.argmax(cand, 1)
    q = np.zeros((len(R), 4))
    for p in range(4):
        m = piv == p
        if not np.any(m):
            continue
        r = R[m]
        if p == 0:
            s = np.sqrt(np.maximum(1.0 + tr[m], 1e-12)) * 2.0
            q[m] = np.stack([0.25 * s, (r[:, 2, 1] - r[:, 1, 2]) / s, (r[:, 0, 2] - r[:, 2, 0]) / s,
                             (r[:, 1, 0] - r[:, 0, 1]) / s], 1)
        else:
            i = p - 1
            j, k = (i + 1) % 3, (i + 2) % 3
            s = np.sqrt(np.maximum(1.0 + r[:, i, i] - r[:, j, j] - r[:, k, k], 1e-12)) * 2.0
            qq = np.zeros((len(r), 4))
            qq[:, 0] = (r[:, k, j] - r[:, j, k]) / s
            qq[:, 1 + i] = 0.25 * s
            qq[:, 1 + j] = (r[:, j, i] + r[:, i, j]) / s
            qq[:, 1 + k] = (r[:, k, i] + r[:, i, k]) / s
            q[m] = qq
    q /= np.maximum(np.linalg.norm(q, axis=1, keepdims=True), 1e-12)
    q *= np.where(q[:, :1] < 0, -1.0, 1.0)
    return q


def canonical_shape(scales: np.ndarray, quats: np.ndarray):
    """(sorted log-scales (n,3), canonical unit quaternion (n,4)) describing the same covariance."""
    s = np.asarray(scales, np.float64).reshape(-1, 3)
    R = quat_to_rot(quats)
    order = np.argsort(-s, axis=1, kind="stable")
    n = len(s)
    s_sorted = np.take_along_axis(s, order, 1)
    Rp = R[np.arange(n)[:, None, None], np.arange(3)[None, :, None], order[:, None, :]]
    big = np.argmax(np.abs(Rp), axis=1)  # (n, 3): row of each column's largest component
    sign = np.sign(np.take_along_axis(Rp, big[:, None, :], 1))[:, 0, :]
    sign[sign == 0] = 1.0
    Rp = Rp * sign[:, None, :]
    det = np.linalg.det(Rp)
    Rp[:, :, 2] *= np.where(det < 0, -1.0, 1.0)[:, None]
    return s_sorted, rot_to_quat(Rp)


def canonical_targets(base: GaussianModel, trained: GaussianModel) -> np.ndarray:
    """The 11 regression targets of each Gaussian (rows in the order of the initial points)."""
    if trained.size() != base.size():
        raise ValueError("label run changed the number of Gaussians")
    s, q = canonical_shape(trained.scales, trained.quats)
    t = np.zeros((base.size(), 11), np.float64)
    t[:, 0:3] = s - base.scales.astype(np.float64)
    t[:, 3:7] = q
    t[:, 7] = np.clip(trained.opacities, -OPACITY_CLIP, OPACITY_CLIP)
    t[:, 8:11] = trained.colors.astype(np.float64) - base.colors
    return t.astype(np.float32)


def plain_targets(base: GaussianModel) -> np.ndarray:
    """The plain initialisation written as network outputs (zero residuals)."""
    t = np.zeros((base.size(), 11), np.float32)
    t[:, 3:7] = base.quats
    t[:, 7] = base.opacities
    return t


def label_scene(sc: Scene, iterations: int = LABEL_ITERATIONS):
    """(features (n,134), targets (n,11), plain init) of one scene."""
    base = api.initGaussiansFromPoints(sc.init_xyz, sc.init_rgb)
    X = api.warmstartFeatures(sc.init_xyz, sc.init_rgb, sc.images)
    t = api.Trainer(base.copy(), sc.images, sc.extent, label_options(iterations))
    t.step(iterations)
    trained = t.model()
    t.close()
    return X, canonical_targets(base, trained), base


def generate_labels(seeds, label_fn, shard_dir: Path, rank: int = 0, world: int = 1, barrier=None, log=print):
    """Label rows of all `seeds`, the scenes shared over `world` ranks (one per GPU): rank r labels seeds
    r, r + world, ... (scenes are independent, so there is no collective on the data) and writes each to
    shard_dir/labels_<seed>.npz; after `barrier`, rank 0 reads every shard in seed order and returns
    (X, T); the other ranks return None. label_fn(seed) -> (X, T)."""
    seeds = list(seeds)
    shard_dir = Path(shard_dir)
    shard_dir.mkdir(parents=True, exist_ok=True)
    t0 = time.time()
    for k, seed in enumerate(seeds[rank::world]):
        X, T = label_fn(seed)
        np.savez(shard_dir / f"labels_{seed}.npz", X=X, T=T)
        log(f"rank {rank}: label scene {k + 1} (seed {seed}): {len(X)} rows, {time.time() - t0:.1f} s")
    if barrier is not None:
        barrier()
    if rank != 0:
        return None
    Xs, Ts = [], []
    for seed in seeds:
        with np.load(shard_dir / f"labels_{seed}.npz") as z:
            Xs.append(z["X"])
            Ts.append(z["T"])
    return np.concatenate(Xs), np.concatenate(Ts)


# ------------------------------------------------------------------ training


def standardiser(X: np.ndarray):
    mu = X.mean(axis=0, dtype=np.float64)
    sd = X.std(axis=0, dtype=np.float64)
    sd = np.where(sd > 1e-6, sd, 1.0)
    return mu, sd


def fold_standardiser(params: np.ndarray, mu: np.ndarray, sd: np.ndarray) -> np.ndarray:
    """Parameters of a network on raw x equal to `params` on (x - mu) / sd: W0/sd, b0 - W0 (mu/sd)."""
    p = np.asarray(params, np.float64).copy()
    n_in, n_out = api.MLP_INPUTS, 128
    W0 = p[:n_in * n_out].reshape(n_out, n_in)
    b0 = p[n_in * n_out:n_in * n_out + n_out]
    p[n_in * n_out:n_in * n_out + n_out] = b0 - W0 @ (mu / sd)
    p[:n_in * n_out] = (W0 / sd[None, :]).reshape(-1)
    return p.astype(np.float32)


def train_network(X: np.ndarray, T: np.ndarray, stages=((24, 1e-3), (12, 3e-4), (6, 1e-4)), batch: int = 4096,
                  seed: int = 0, log=print):
    """Trains on the GPU; returns (parameters on raw features, per-epoch losses)."""
    mu, sd = standardiser(X)
    Xs = ((X - mu) / sd).astype(np.float32)
    net = api.WarmStartNet(seed=seed)
    losses = []
    for k, (epochs, lr) in enumerate(stages):
        ls = net.train(Xs, T, epochs=epochs, batch=batch, lr=lr, seed=seed * 1000 + k)
        losses.extend(float(v) for v in ls)
        log(f"  stage {k}: {epochs} epochs at lr {lr:g}: loss {ls[0]:.5f} -> {ls[-1]:.5f}")
    return fold_standardiser(net.params(), mu, sd), losses


def label_loss(params, X, T) -> float:
    """Weighted MSE of the network's outputs against the labels (the training loss)."""
    net = api.WarmStartNet(params)
    loss, _ = net.loss_grad(X, T)
    return loss


def save(path: Path, params: np.ndarray, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.asarray(params, "<f4").reshape(-1).tofile(path)
    path.with_suffix(".json").write_text(json.dumps(meta, indent=1))


def load_params(path: Path = WEIGHTS_PATH):
    path = Path(path)
    params = np.fromfile(path, "<f4").astype(np.float32)
    if params.size != api.MLP_PARAMS:
        raise ValueError(f"{path}: {params.size} parameters, expected {api.MLP_PARAMS}")
    meta_path = path.with_suffix(".json")
    meta = json.loads(meta_path.read_text()) if meta_path.exists() else {}
    return params, meta


def load_network(path: Path = WEIGHTS_PATH) -> api.WarmStartNet:
    return api.WarmStartNet(load_params(path)[0])


# ------------------------------------------------------------------ evaluation


def run_from(sc: Scene, init: GaussianModel, init_seconds: float, chunk: int, iterations: int | None = None):
    """A full schedule from `init`: the scene's preset schedule, or forIterations(iterations) with the
    preset's Gaussian cap."""
    opt = sc.options()
    if iterations:
        short = TrainOptions.for_iterations(iterations)
        short.max_gaussians = opt.max_gaussians
        opt = short
    t = api.Trainer(init, sc.images, sc.extent, opt)
    r = run_schedule(t, opt.iterations, chunk=chunk)
    out = r.as_dict()
    out["init_seconds"] = round(init_seconds, 4)
    out["final_loss_ema"] = t.stats().loss
    t.close()
    return r, out


def evaluate_seed(net: api.WarmStartNet, seed: int, chunk: int = 250, spec=None,
                  short_iterations: int | None = None) -> dict:
    """Plain vs warm start on one held-out seed. With short_iterations, both inits also run the shorter
    schedule forIterations(short_iterations) (the plain one as the control): whether and when each
    reaches the plain full-schedule PSNR."""
    sc = build_scene(seed, spec if spec is not None else scene_spec(seed))
    t0 = time.perf_counter()
    plain = api.initGaussiansFromPoints(sc.init_xyz, sc.init_rgb)
    t_plain_init = time.perf_counter() - t0
    t0 = time.perf_counter()
    warm = api.warmstartInit(net, sc.init_xyz, sc.init_rgb, sc.images)
    t_warm_init = time.perf_counter() - t0
    rp, dp = run_from(sc, plain, t_plain_init, chunk)
    rw, dw = run_from(sc, warm, t_warm_init, chunk)
    target = rp.final_psnr
    plain_time = t_plain_init + rp.total_seconds
    ttp = rw.time_to_psnr(target)
    warm_time = None if ttp is None else t_warm_init + ttp
    row = {"seed": seed, "gt_count": sc.spec.gt_count, "target_psnr": round(target, 4),
           "plain_time_s": round(plain_time, 4), "warm_time_to_target_s": None if warm_time is None else
           round(warm_time, 4), "time_ratio": None if warm_time is None else round(warm_time / plain_time, 4),
           "plain_final_psnr": round(rp.final_psnr, 4), "warm_final_psnr": round(rw.final_psnr, 4),
           "plain_initial_psnr": round(rp.initial_psnr, 4), "warm_initial_psnr": round(rw.initial_psnr, 4),
           "plain": dp, "warm": dw}
    if short_iterations:
        for name, init, t_init in (("plain_short", plain, t_plain_init), ("warm_short", warm, t_warm_init)):
            r, d = run_from(sc, init, t_init, chunk, short_iterations)
            ttp = r.time_to_psnr(target)
            row[name] = {"iterations": short_iterations, "final_psnr": round(r.final_psnr, 4),
                         "time_to_target_s": None if ttp is None else round(t_init + ttp, 4),
                         "time_ratio": None if ttp is None else round((t_init + ttp) / plain_time, 4),
                         "trajectory": d}
    return row


def summarise(rows: list) -> dict:
    ratios = [r["time_ratio"] for r in rows if r["time_ratio"] is not None]
    extra = {}
    for name in ("plain_short", "warm_short"):
        if all(name in r for r in rows) and rows:
            sr = [r[name]["time_ratio"] for r in rows]
            got = [v for v in sr if v is not None]
            extra[name] = {"iterations": rows[0][name]["iterations"], "reached": f"{len(got)}/{len(rows)}",
                           "median_time_ratio": float(np.median(got)) if len(got) == len(rows) else None,
                           "mean_final_psnr_minus_target_db": float(np.mean(
                               [r[name]["final_psnr"] - r["target_psnr"] for r in rows]))}
    return extra | {"seeds": [r["seed"] for r in rows],
            "reached": f"{len(ratios)}/{len(rows)}",
            "median_time_ratio": float(np.median(ratios)) if ratios else None,
            "mean_time_ratio": float(np.mean(ratios)) if ratios else None,
            "mean_final_psnr_gain_db": float(np.mean([r["warm_final_psnr"] - r["plain_final_psnr"] for r in rows])),
            "mean_initial_psnr_gain_db": float(np.mean([r["warm_initial_psnr"] - r["plain_initial_psnr"]
                                                        for r in rows]))}


# ------------------------------------------------------------------ command line


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train", help="label runs on the training seeds, then network training")
    tr.add_argument("--out", type=Path, default=WEIGHTS_PATH)
    tr.add_argument("--scenes", type=int, default=len(TRAIN_SEEDS))
    tr.add_argument("--label-iterations", type=int, default=LABEL_ITERATIONS)
    tr.add_argument("--holdout-labels", type=int, default=2, help="held-out seeds whose label loss is reported")
    tr.add_argument("--shard-dir", type=Path, default=None,
                    help="where the ranks leave their label shards (default: label_shards beside --out)")
    ev = sub.add_parser("evaluate", help="plain vs warm start on held-out seeds")
    ev.add_argument("--weights", type=Path, default=WEIGHTS_PATH)
    ev.add_argument("--seeds", type=int, default=len(EVAL_SEEDS))
    ev.add_argument("--chunk", type=int, default=250)
    ev.add_argument("--out", type=Path, default=None)
    ev.add_argument("--short-iterations", type=int, default=0,
                    help="also run both inits on forIterations(N) (the plain one as the control)")
    a = ap.parse_args(argv)

    def log(*m):
        print(*m, file=sys.stderr, flush=True)

    if a.cmd == "train":
        t0 = time.time()
        # One process per GPU under torchrun: the label scenes are shared over the ranks, rank 0 trains.
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        barrier = None
        if world > 1:
            import datetime

            import torch.distributed as dist
            from . import _lib
            _lib.check(_lib.load().u3dg_set_device(int(os.environ.get("LOCAL_RANK", "0"))))
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=3600))
            barrier = dist.barrier

        def label_fn(seed):
            X, T, _ = label_scene(build_scene(seed), a.label_iterations)
            return X, T

        shard_dir = a.shard_dir or (Path(a.out).resolve().parent / "label_shards")
        got = generate_labels(TRAIN_SEEDS[:a.scenes], label_fn, shard_dir, rank, world, barrier, log)
        if world > 1:
            dist.destroy_process_group()
        if got is None:
            return 0
        X, T = got
        t1 = time.time()
        params, losses = train_network(X, T, log=log)
        train_s = time.time() - t1
        meta = {"label_iterations": a.label_iterations, "train_seeds": list(TRAIN_SEEDS[:a.scenes]),
                "rows": int(len(X)), "epoch_losses": losses, "train_seconds": round(train_s, 2)}
        hold = []
        net = api.WarmStartNet(params)
        for seed in EVAL_SEEDS[:a.holdout_labels]:
            sc = build_scene(seed)
            Xh, Th, base = label_scene(sc, a.label_iterations)
            mse_net = np.mean((net.forward(Xh).astype(np.float64) - Th) ** 2, axis=0)
            mse_plain = np.mean((plain_targets(base).astype(np.float64) - Th) ** 2, axis=0)
            hold.append({"seed": seed, "network_label_loss": label_loss(params, Xh, Th),
                         "plain_label_loss": float(np.sum(LOSS_WEIGHTS * mse_plain) / 11.0),
                         "per_output_mse_network": [round(float(v), 5) for v in mse_net],
                         "per_output_mse_plain": [round(float(v), 5) for v in mse_plain]})
            log(f"held-out labels seed {seed}: {hold[-1]}")
        meta["holdout_label_loss"] = hold
        save(a.out, params, meta)
        log(f"saved {a.out} ({time.time() - t0:.1f} s total)")
        print(json.dumps({k: v for k, v in meta.items() if k != "epoch_losses"}))
        return 0

    net = load_network(a.weights)
    rows = []
    for seed in EVAL_SEEDS[:a.seeds]:
        r = evaluate_seed(net, seed, a.chunk, short_iterations=a.short_iterations or None)
        rows.append(r)
        log(f"seed {seed}: target {r['target_psnr']:.2f} dB, plain {r['plain_time_s']:.2f} s, warm "
            f"{r['warm_time_to_target_s']} s (ratio {r['time_ratio']}), final {r['plain_final_psnr']:.2f} vs "
            f"{r['warm_final_psnr']:.2f} dB")
    res = {"summary": summarise(rows), "runs": rows}
    if a.out:
        a.out.write_text(json.dumps(res, indent=1))
    print(json.dumps(res["summary"]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
