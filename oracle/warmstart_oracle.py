"""CPU restatement of the learned warm-start kernels (test infrastructure only).

Only the tests, the smoke check and the CPU legs of the benchmark use this module; the product
path is the CUDA library. The warm-start has no counterpart in the reference, whose trainer starts
from initGaussiansFromPoints (engine/src/splat/GaussianModel.cpp:68-144); what this file restates is
the specification written in the CUDA source (warmstart.cu):

  kNN        squared distances in float32, each product and sum rounded separately, summed
             x, y, z in that order; ties keep the lower index; exclude_self skips index == query
  features   134 floats per point (16-NN relative positions / sigma, log distances, neighbour
             colours, colour samples of the 7 nearest views that see the point, visibility)
  MLP        134 -> 128 -> 128 -> 128 -> 11, ReLU between layers; parameters per layer W (out x in,
             row-major) then b; loss = sum_o w_o * mean over rows of (y - t)^2 / outputs

The MLP forward and gradient are computed in float64, which makes them the reference for the
float32 GPU kernels and for central finite differences alike.
"""
from __future__ import annotations

import numpy as np

INPUTS, HIDDEN, OUTPUTS = 134, 128, 11
LAYERS = ((INPUTS, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, OUTPUTS))
PARAMS = sum(i * o + o for i, o in LAYERS)
NEIGHBOURS, VIEWS = 16, 7
DEFAULT_WEIGHTS = np.array([1, 1, 1, 0.5, 0.5, 0.5, 0.5, 0.25, 1, 1, 1], np.float64)


def unpack(params: np.ndarray):
    """[(W (out, in), b (out,)), ...] views into a flat parameter vector."""
    p = np.asarray(params).reshape(-1)
    assert p.size == PARAMS, p.size
    out, o = [], 0
    for i, n in LAYERS:
        W = p[o:o + i * n].reshape(n, i)
        o += i * n
        b = p[o:o + n]
        o += n
        out.append((W, b))
    return out


def mlp_forward(params, x, dtype=np.float64):
    """Outputs (n, 11) and the per-layer inputs (for the gradient)."""
    h = np.asarray(x, dtype).reshape(-1, INPUTS)
    acts = [h]
    layers = unpack(np.asarray(params, dtype))
    for l, (W, b) in enumerate(layers):
        h = h @ W.T + b
        if l < len(layers) - 1:
            h = np.maximum(h, 0.0)
            acts.append(h)
    return h, acts


def mlp_loss(params, x, t, weights=None) -> float:
    y, _ = mlp_forward(params, x)
    w = DEFAULT_WEIGHTS if weights is None else np.asarray(weights, np.float64)
    e = y - np.asarray(t, np.float64).reshape(y.shape)
    return float(np.sum(w * e * e) / e.size)


def mlp_loss_grad(params, x, t, weights=None):
    """Loss and its gradient with respect to the flat parameter vector (float64)."""
    y, acts = mlp_forward(params, x)
    w = DEFAULT_WEIGHTS if weights is None else np.asarray(weights, np.float64)
    e = y - np.asarray(t, np.float64).reshape(y.shape)
    loss = float(np.sum(w * e * e) / e.size)
    d = 2.0 * w * e / e.size
    layers = unpack(np.asarray(params, np.float64))
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        a = acts[l]
        grads[l] = (d.T @ a, d.sum(axis=0))
        if l > 0:
            d = (d @ W) * (a > 0.0)
    flat = np.concatenate([np.concatenate([gW.reshape(-1), gb]) for gW, gb in grads])
    return loss, flat


def _dist2(d):
    d = d.astype(np.float32)
    return (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]


def knn(queries, points, k, exclude_self=False):
    """Indices (nq, k) int32 and squared distances (nq, k) float32; -1 / FLT_MAX where fewer exist."""
    q = np.asarray(queries, np.float32).reshape(-1, 3)
    p = np.asarray(points, np.float32).reshape(-1, 3)
    idx = np.full((len(q), k), -1, np.int32)
    d2 = np.full((len(q), k), np.finfo(np.float32).max, np.float32)
    for i in range(len(q)):
        d = _dist2(p - q[i])
        if exclude_self and i < len(p):
            d = d.copy()
            d[i] = np.inf
        order = np.argsort(d, kind="stable")[:k]
        order = order[np.isfinite(d[order])]
        idx[i, :len(order)] = order
        d2[i, :len(order)] = d[order]
    return idx, d2


def camera_centre(cam) -> np.ndarray:
    R = np.asarray(cam.R, np.float32).reshape(3, 3)
    t = np.asarray(cam.t, np.float32)
    return np.array([-((R[0, c] * t[0] + R[1, c] * t[1]) + R[2, c] * t[2]) for c in range(3)], np.float32)


def features(xyz, rgb, sigma, images) -> np.ndarray:
    """The 134 input features per point; sigma is exp of the plain initialisation's log-scale."""
    xyz = np.asarray(xyz, np.float32).reshape(-1, 3)
    n = len(xyz)
    f = np.zeros((n, INPUTS), np.float32)
    if n == 0:
        return f
    nbr, nd2 = knn(xyz, xyz, NEIGHBOURS, exclude_self=True)
    sig = np.asarray(sigma, np.float32)
    inv = np.where(sig > 0, np.float32(1.0) / np.where(sig > 0, sig, 1).astype(np.float32), 0).astype(np.float32)
    col = None if rgb is None else np.asarray(rgb, np.float32).reshape(-1, 3)
    for k in range(NEIGHBOURS):
        j = nbr[:, k]
        ok = j >= 0
        jj = np.where(ok, j, 0)
        rel = (xyz[jj] - xyz) * inv[:, None]
        f[:, 3 * k:3 * k + 3] = np.where(ok[:, None], rel, 0)
        f[:, 48 + k] = np.where(ok, np.float32(0.5) * np.log(np.maximum(nd2[:, k], np.float32(1e-20))), 0)
        c = np.full((n, 3), 0.5, np.float32) if col is None else col[jj]
        f[:, 64 + 3 * k:64 + 3 * k + 3] = np.where(ok[:, None], c, 0)
    # The 7 nearest views (by camera-centre distance) that see the point inside the image.
    best = [[] for _ in range(n)]
    for v, im in enumerate(images):
        cam = im.camera
        R = np.asarray(cam.R, np.float32).reshape(3, 3)
        t = np.asarray(cam.t, np.float32)
        cx, cy, cz = [(xyz[:, 0] * R[r, 0] + xyz[:, 1] * R[r, 1]) + xyz[:, 2] * R[r, 2] + t[r] for r in range(3)]
        fx, fy = np.float32(cam.fx), np.float32(cam.fy)
        with np.errstate(divide="ignore", invalid="ignore"):
            uf = (fx * cx) / cz + np.float32(cam.cx)
            wf = (fy * cy) / cz + np.float32(cam.cy)
        W, H = cam.width, cam.height
        vis = (cz > np.float32(1e-3)) & (uf > -0.5) & (wf > -0.5) & (uf < np.float32(W) - 0.5) & \
              (wf < np.float32(H) - 0.5)
        d = _dist2(xyz - camera_centre(cam))
        for i in np.nonzero(vis)[0]:
            u, w = int(np.rint(uf[i])), int(np.rint(wf[i]))
            best[i].append((float(d[i]), v, u, w))
    for i in range(n):
        # Strict < insertion over views in order: stable by view index for equal distances.
        chosen = sorted(best[i], key=lambda e: e[0])[:VIEWS]
        for k, (_, v, u, w) in enumerate(chosen):
            px = images[v].rgb[w, u].astype(np.float32)
            f[i, 112 + 3 * k:112 + 3 * k + 3] = px * np.float32(1.0 / 255.0) - np.float32(0.5)
        f[i, 133] = np.float32(len(chosen)) / np.float32(VIEWS)
    return f
