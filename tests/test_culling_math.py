"""Conservativeness of the compositing kernels' culling, checked on the CPU.

The trainers skip work in two places without changing any image: a staged list entry is tested
against each warp's 8x8 pixel block (`ellipseMeets`, raster_common.cuh), and a Gaussian is listed
only in the tiles of its rectangle that its contributing ellipse reaches (`cullShape` / `cullSpan`,
binning.cu). Both must never drop a pixel whose power the compositing kernels would accept
(powMin <= power <= 0). These tests restate both tests in numpy float32, operation by operation
(the kernels use rounding-explicit intrinsics, so float32 numpy rounds the same way), and compare
them with a brute-force evaluation of the kernels' per-pixel power (`columnTerms` / `powerAt`) over
random, strongly anisotropic footprints placed around block and tile boundaries. The GPU test
`test_tile_culling_renders_identically` checks the kernels themselves.
"""
import numpy as np
import pytest

f = np.float32
MIN_ALPHA = f(1.0) / f(255.0)


def _footprints(rng, m, max_sigma2=2e3):
    """Conics (A, B, C), alphas and powMin of m random footprints: eigenvalues log-uniform, condition
    numbers up to 1e4 (beyond that the kernels do not cull), the 0.3 px^2 dilation, random angles."""
    l1 = np.exp(rng.uniform(np.log(0.3), np.log(max_sigma2), m))
    l2 = l1 / np.exp(rng.uniform(0, np.log(1e4), m))
    th = rng.uniform(0, np.pi, m)
    c, s = np.cos(th), np.sin(th)
    sa = c * c * l1 + s * s * l2 + 0.3
    sc = s * s * l1 + c * c * l2 + 0.3
    sb = c * s * (l1 - l2)
    det = sa * sc - sb * sb
    A, B, C = (sc / det).astype(f), (-sb / det).astype(f), (sa / det).astype(f)
    alpha = rng.uniform(0.002, 1.0, m).astype(f)
    pow_min = (np.log(MIN_ALPHA / alpha).astype(f) - f(1e-4)).astype(f)
    lmax = 0.5 * (sa + sc) + np.sqrt(0.25 * (sa - sc) ** 2 + sb * sb)
    return A, B, C, pow_min, np.ceil(3.0 * np.sqrt(lmax))


def _contributes(mx, my, A, B, C, pow_min, xs, ys):
    """Kernel power at pixel centres xs (..., nx) x ys (..., ny): any pixel with powMin <= power <= 0."""
    dx = (mx[:, None] - xs).astype(f)[:, :, None]
    dy = (my[:, None] - ys).astype(f)[:, None, :]
    axx = ((A[:, None, None] * dx).astype(f) * dx).astype(f)
    bx = (B[:, None, None] * dx).astype(f)
    q = (axx + ((C[:, None, None] * dy).astype(f) * dy).astype(f)).astype(f)
    pw = ((f(-0.5) * q).astype(f) - (bx * dy).astype(f)).astype(f)
    return ((pw <= 0) & (pw >= pow_min[:, None, None])).any(axis=(1, 2))


def _ellipse_meets(mx, my, A, B, C, pow_min, x0, y0):
    """ellipseMeets (raster_common.cuh) in float32."""
    X0 = (x0 - mx).astype(f)
    X1 = (X0 + f(7)).astype(f)
    Y0 = (y0 - my).astype(f)
    Y1 = (Y0 + f(7)).astype(f)
    inside = (X0 <= 0) & (X1 >= 0) & (Y0 <= 0) & (Y1 >= 0)
    iA, iC = (f(1) / A).astype(f), (f(1) / C).astype(f)

    def quad(dx, dy):
        cross = (f(2) * ((B * dx).astype(f) * dy).astype(f)).astype(f)
        return ((((A * dx).astype(f) * dx).astype(f) + cross).astype(f) + ((C * dy).astype(f) * dy).astype(f)).astype(f)

    nbc, nba = (-B * iC).astype(f), (-B * iA).astype(f)
    m = quad(X0, np.minimum(np.maximum((nbc * X0).astype(f), Y0), Y1))
    m = np.minimum(m, quad(X1, np.minimum(np.maximum((nbc * X1).astype(f), Y0), Y1)))
    m = np.minimum(m, quad(np.minimum(np.maximum((nba * Y0).astype(f), X0), X1), Y0))
    m = np.minimum(m, quad(np.minimum(np.maximum((nba * Y1).astype(f), X0), X1), Y1))
    return inside | (m <= ((f(-2.08) * pow_min).astype(f) + f(1e-3)).astype(f))


def _cull_span(mx, my, A, B, C, pow_min, rx0, rx1, ty, tile):
    """cullShape + cullSpan (binning.cu) in float32 for well-conditioned footprints: columns [c0, c1)."""
    t = ((f(-2.08) * pow_min).astype(f) + f(1e-3)).astype(f)
    det = ((A * C).astype(f) - (B * B).astype(f)).astype(f)
    at = (A * t).astype(f)
    iA = (f(1) / A).astype(f)
    tp = np.maximum(t, f(0))  # t <= 0: no tile (the kernel stops before these square roots)
    ymax = np.sqrt(((tp * A).astype(f) / det).astype(f)).astype(f)
    xmax = np.sqrt(((tp * C).astype(f) / det).astype(f)).astype(f)
    dyr0 = ((-B / C).astype(f) * xmax).astype(f)
    Y0 = ((ty * tile).astype(f) - my).astype(f)
    Y1 = (Y0 + f(tile - 1)).astype(f)
    lo, hi = np.maximum(Y0, -ymax), np.minimum(Y1, ymax)
    empty = (lo > hi) | ~(t > 0)
    dyR = np.minimum(np.maximum(dyr0, lo), hi)
    dyL = np.minimum(np.maximum(-dyr0, lo), hi)
    sR = np.sqrt(np.maximum((at - (det * (dyR * dyR).astype(f)).astype(f)).astype(f), f(0))).astype(f)
    sL = np.sqrt(np.maximum((at - (det * (dyL * dyL).astype(f)).astype(f)).astype(f), f(0))).astype(f)
    xR = ((((-B) * dyR).astype(f) + sR).astype(f) * iA).astype(f)
    xL = ((((-B) * dyL).astype(f) - sL).astype(f) * iA).astype(f)
    inv = f(1) / f(tile)
    left = np.floor((((mx + xL).astype(f) - f(1)).astype(f) * inv).astype(f))
    right = np.floor((((mx + xR).astype(f) + f(1)).astype(f) * inv).astype(f)) + f(1)
    c0 = np.where(left > rx0, np.minimum(left, rx1), rx0).astype(np.int64)
    c1 = np.where(right < rx1, np.maximum(right, rx0), rx1).astype(np.int64)
    c1 = np.maximum(c1, c0)
    return np.where(empty, rx0, c0), np.where(empty, rx0, c1)


@pytest.mark.parametrize("seed", [1, 2])
def test_block_ellipse_test_keeps_every_contributing_block(seed):
    rng = np.random.default_rng(seed)
    m = 60000
    A, B, C, pow_min, rad = _footprints(rng, m, max_sigma2=400.0)
    x0 = (rng.integers(0, 13, m) * 8).astype(f)
    y0 = (rng.integers(0, 13, m) * 8).astype(f)
    # Means spread around the block, many of them just outside it.
    mx = (x0 + 3.5 + rng.uniform(-1, 1, m) * (rad + 4)).astype(f)
    my = (y0 + 3.5 + rng.uniform(-1, 1, m) * (rad + 4)).astype(f)
    offs = np.arange(8, dtype=f)
    hit = _contributes(mx, my, A, B, C, pow_min, x0[:, None] + offs, y0[:, None] + offs)
    keep = _ellipse_meets(mx, my, A, B, C, pow_min, x0, y0)
    assert hit.sum() > 1000
    assert not (hit & ~keep).any(), "a block with a contributing pixel was culled"
    # The test is tight: few kept blocks lack a contributing pixel.
    assert (keep & ~hit).sum() < 0.05 * keep.sum()


@pytest.mark.parametrize("tile", [8, 16, 32])
def test_tile_spans_keep_every_contributing_tile(tile):
    rng = np.random.default_rng(10 + tile)
    m = 4000
    A, B, C, pow_min, rad = _footprints(rng, m, max_sigma2=150.0)
    grid = 48
    mx = rng.uniform(0, grid * tile, m).astype(f)
    my = rng.uniform(0, grid * tile, m).astype(f)
    rx0 = np.clip(((mx - rad) / tile).astype(int), 0, grid)
    rx1 = np.clip(((mx + rad + tile - 1) / tile).astype(int), 0, grid)
    ry0 = np.clip(((my - rad) / tile).astype(int), 0, grid)
    ry1 = np.clip(((my + rad + tile - 1) / tile).astype(int), 0, grid)
    ok = (rx1 > rx0) & (ry1 > ry0)
    ty = ry0 + (rng.uniform(0, 1, m) * (ry1 - ry0)).astype(int)
    c0, c1 = _cull_span(mx, my, A, B, C, pow_min, rx0, rx1, ty, tile)
    offs = np.arange(tile, dtype=f)
    ys = (ty * tile).astype(f)[:, None] + offs
    needed = kept = 0
    for dxt in range(int((rx1 - rx0).max())):
        tx = rx0 + dxt
        live = ok & (tx < rx1)
        xs = (tx * tile).astype(f)[:, None] + offs
        hit = _contributes(mx, my, A, B, C, pow_min, xs, ys) & live
        inspan = live & (c0 <= tx) & (tx < c1)
        assert not (hit & ~inspan).any(), "a tile with a contributing pixel was dropped"
        needed += int(hit.sum())
        kept += int(inspan.sum())
    assert needed > 1000 and kept < 1.2 * needed
