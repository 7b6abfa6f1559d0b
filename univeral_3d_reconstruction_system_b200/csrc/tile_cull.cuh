// tile_cull.cuh - which tiles of its rectangle a Gaussian is listed in (tile culling of the trainers).
//
// A Gaussian is listed only in the tiles of its rectangle that its contributing ellipse
// {d : A dx^2 + 2 B dx dy + C dy^2 <= t} (power >= powMin) can reach. In one tile row the reachable
// tiles are contiguous: the ellipse cut by the row's strip of pixel centres spans [xL, xR] with
// xR(dy) = (-B dy + sqrt(A t - det dy^2)) / A concave in dy, so its maximum over the strip is at the
// clamped dy of the ellipse's rightmost point (and xL's minimum symmetrically). Rounding-explicit:
// the projection (which counts a Gaussian's tiles) and the emission (which lists them) are compiled
// with different contraction settings and must get the same spans. Conservative like the compositing
// kernels' block masks: t widened by 4% + 1e-3 and the span by one pixel each side. Dropping entries
// that reach no pixel of a tile changes no image and no per-entry gradient.
#pragma once

#include "kernels.h"

namespace u3dg {

constexpr int kCullRows = 8; // rows per Gaussian in the emission's row table (32 bytes: two uint4 loads)
static_assert(kCullRows == 8, "the emission reads a Gaussian's row table as two uint4");

struct CullShape {
    float mx, my, B, det, at, iA, ymax, dyR; // dyR: dy of the rightmost point, (-B / C) xmax
    int mode;                                // 0: whole rectangle, 1: no tile, 2: culled rows
};

// From a raster record's first two float4s (mean, box half-extents; conic, alpha) and its exponent floor.
__device__ __forceinline__ CullShape cullShapeOf(const float4 &p, const float4 &q, float powMin)
{
    CullShape c{};
    const float t = __fadd_rn(__fmul_rn(-2.08f, powMin), 1e-3f);
    const float det = __fsub_rn(__fmul_rn(q.x, q.z), __fmul_rn(q.y, q.y));
    // Infinite box extents: ill-conditioned covariance or no alpha floor.
    if (!(p.z < __int_as_float(0x7f800000)) || !(det > 0.0f) || !(q.x > 0.0f) || !(q.z > 0.0f))
        return c;
    if (!(t > 0.0f)) { // alpha below the floor everywhere
        c.mode = 1;
        return c;
    }
    c.mode = 2;
    c.mx = p.x;
    c.my = p.y;
    c.B = q.y;
    c.det = det;
    c.at = __fmul_rn(q.x, t);
    c.iA = __frcp_rn(q.x);
    c.ymax = __fsqrt_rn(__fdiv_rn(__fmul_rn(t, q.x), det));
    const float xmax = __fsqrt_rn(__fdiv_rn(__fmul_rn(t, q.z), det));
    c.dyR = __fmul_rn(__fdiv_rn(-q.y, q.z), xmax);
    return c;
}

__device__ __forceinline__ CullShape cullShape(const SplatRec *rec, int g)
{
    const float4 *r = reinterpret_cast<const float4 *>(rec) + size_t(g) * 3;
    return cullShapeOf(r[0], r[1], r[2].w);
}

// Tile columns [c0, c1) of tile row ty that the ellipse can reach, within rectangle q.
__device__ __forceinline__ void cullSpan(const CullShape &c, const int4 &q, int ty, int tileSize, int &c0, int &c1)
{
    c0 = q.x;
    c1 = q.z;
    if (c.mode == 0)
        return;
    const float Y0 = __fsub_rn(float(ty * tileSize), c.my), Y1 = __fadd_rn(Y0, float(tileSize - 1));
    const float lo = fmaxf(Y0, -c.ymax), hi = fminf(Y1, c.ymax);
    if (c.mode == 1 || lo > hi) {
        c1 = c0;
        return;
    }
    const float dyR = fminf(fmaxf(c.dyR, lo), hi), dyL = fminf(fmaxf(-c.dyR, lo), hi);
    const float sR = __fsqrt_rn(fmaxf(__fsub_rn(c.at, __fmul_rn(c.det, __fmul_rn(dyR, dyR))), 0.0f));
    const float sL = __fsqrt_rn(fmaxf(__fsub_rn(c.at, __fmul_rn(c.det, __fmul_rn(dyL, dyL))), 0.0f));
    const float xR = __fmul_rn(__fadd_rn(__fmul_rn(-c.B, dyR), sR), c.iA);
    const float xL = __fmul_rn(__fsub_rn(__fmul_rn(-c.B, dyL), sL), c.iA);
    const float inv = __frcp_rn(float(tileSize)); // exact: tile sizes are powers of two
    const float left = floorf(__fmul_rn(__fsub_rn(__fadd_rn(c.mx, xL), 1.0f), inv));
    const float right = __fadd_rn(floorf(__fmul_rn(__fadd_rn(__fadd_rn(c.mx, xR), 1.0f), inv)), 1.0f);
    c0 = left > float(q.x) ? int(fminf(left, float(q.z))) : q.x;
    c1 = right < float(q.z) ? int(fmaxf(right, float(q.x))) : q.z;
    c1 = max(c1, c0);
}

// Tiles a Gaussian with rectangle q is listed in: cull false, the whole rectangle (no row table);
// cull true, the reachable tiles of each row (cullSpan), with the first kCullRows rows recorded in
// row[i] as (first column << 16) | (tiles through row i), so the emission finds an entry's row
// without recomputing spans (rows beyond kCullRows, rare, are recomputed there).
__device__ __forceinline__ int listedTiles(const CullShape &cs, bool cull, const int4 &q, int tileSize, uint32_t *row)
{
    if (!cull)
        return (q.z - q.x) * (q.w - q.y);
    int c = 0;
    for (int ty = q.y; ty < q.w; ++ty) {
        int c0, c1;
        cullSpan(cs, q, ty, tileSize, c0, c1);
        c += c1 - c0;
        if (ty - q.y < kCullRows)
            row[ty - q.y] = (uint32_t(c0) << 16) | uint32_t(c);
    }
    return c;
}

} // namespace u3dg
