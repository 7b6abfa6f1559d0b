// raster_common.cuh - pixel layout and batch staging shared by the compositing kernels.
//
// A CTA covers a PB x PB pixel block (PB = 16, or 8 for tile size 8) with PB*PB/2 threads; a warp
// owns an 8 x 8 pixel block and each thread two pixels of the same column, rows r and r + 4. A tile's
// depth-sorted list is walked in batches of BD records per thread (the batch depth, 1 or 2); while
// staging a batch, each warp votes which of its 32 entries meet each warp's pixel block (the Gaussian's
// conservative contributing box, SplatRec::ex / ey, against the block), so each warp later walks only
// the set bits of its mask. The batch depth changes how many entries are staged per barrier, not any
// result: every entry is evaluated the same way in the same order.
#pragma once

#include "kernels.h"

namespace u3dg {

template <int PB, int BD = 1>
struct RasterShape {
    static constexpr int NT = PB * PB / 2; // threads
    static constexpr int NW = NT / 32;     // warps
    static constexpr int WX = PB / 8;      // warp blocks per row
    static constexpr int NB = NT * BD;     // batch entries
    static constexpr int NG = NB / 32;     // 32-entry groups of a batch (mask words per warp)
};

// This thread's two pixels and its warp's 8x8 block, in pixel block (bx, by).
template <int PB>
struct WarpBlock {
    int px, py0, py1;
    float x0, x1, y0, y1; // warp block, inclusive
    __device__ WarpBlock(int warp, int lane, int bx, int by)
    {
        constexpr int WX = RasterShape<PB>::WX;
        const int wx0 = bx * PB + (warp % WX) * 8, wy0 = by * PB + (warp / WX) * 8;
        px = wx0 + (lane & 7);
        py0 = wy0 + (lane >> 3);
        py1 = py0 + 4;
        x0 = float(wx0);
        x1 = float(wx0 + 7);
        y0 = float(wy0);
        y1 = float(wy0 + 7);
    }
};

template <int PB>
__device__ __forceinline__ bool meets(const float4 &p, int w, int bx, int by)
{
    constexpr int WX = RasterShape<PB>::WX;
    const float x0 = float(bx * PB + (w % WX) * 8), y0 = float(by * PB + (w / WX) * 8);
    return !(p.x + p.z < x0 || p.x - p.z > x0 + 7.0f || p.y + p.w < y0 || p.y - p.w > y0 + 7.0f);
}

// Whether the contributing ellipse of a staged entry, {d : A dx^2 + 2 B dx dy + C dy^2 <= -2 powMin}
// (power >= powMin), can reach a pixel centre of the 8x8 block [x0, x0 + 7] x [y0, y0 + 7]: the
// minimum of the quadratic over the block (zero if the block holds the mean, else on an edge, where it
// is a 1D quadratic minimised at a clamped stationary point) against the threshold widened by 4% and
// 1e-3. Rounding-explicit, so every kernel builds the same masks; conservative like the box extents,
// which are infinite for covariances whose condition number exceeds 1e4 (nothing is culled then).
// Rotated, elongated footprints meet far fewer 8x8 blocks than their axis-aligned boxes suggest.
__device__ __forceinline__ bool ellipseMeets(float mx, float my, const float4 &q, float powMin, float iA, float iC,
                                             float x0, float y0)
{
    const float X0 = __fsub_rn(x0, mx), X1 = __fadd_rn(X0, 7.0f);
    const float Y0 = __fsub_rn(y0, my), Y1 = __fadd_rn(Y0, 7.0f);
    if (X0 <= 0.0f && X1 >= 0.0f && Y0 <= 0.0f && Y1 >= 0.0f)
        return true;
    const float A = q.x, B = q.y, C = q.z;
    auto quad = [&](float dx, float dy) {
        const float cross = __fmul_rn(2.0f, __fmul_rn(__fmul_rn(B, dx), dy));
        return __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(A, dx), dx), cross), __fmul_rn(__fmul_rn(C, dy), dy));
    };
    const float nbc = __fmul_rn(-B, iC), nba = __fmul_rn(-B, iA);
    float m = quad(X0, fminf(fmaxf(__fmul_rn(nbc, X0), Y0), Y1));
    m = fminf(m, quad(X1, fminf(fmaxf(__fmul_rn(nbc, X1), Y0), Y1)));
    m = fminf(m, quad(fminf(fmaxf(__fmul_rn(nba, Y0), X0), X1), Y0));
    m = fminf(m, quad(fminf(fmaxf(__fmul_rn(nba, Y1), X0), X1), Y1));
    return m <= __fadd_rn(__fmul_rn(-2.08f, powMin), 1e-3f);
}

template <int PB>
__device__ __forceinline__ int tileOf(const RasterArgs &a, int bx, int by)
{
    return (by * PB / a.tileSize) * a.tilesX + bx * PB / a.tileSize;
}

// Persistent scheduling: every CTA takes pixel blocks from a device counter until none are left,
// heaviest tile lists first (a.blockOrder), so the long lists start early and no CTA waits for a
// second wave. Returns the next block index for the whole CTA (>= a.blocksX * a.blocksY: done); the
// last CTA to run out resets the counter for the next launch. counter[0] hands out blocks, counter[1]
// counts finished CTAs.
__device__ __forceinline__ int nextBlock(const RasterArgs &a, int *counter, int *sNext)
{
    const int units = a.blocksX * a.blocksY;
    __syncthreads(); // every thread is done with the previous block's shared memory
    if (threadIdx.x == 0) {
        int u = atomicAdd(counter, 1);
        if (u >= units) {
            __threadfence();
            if (atomicAdd(counter + 1, 1) == int(gridDim.x) - 1) {
                atomicExch(counter, 0);
                atomicExch(counter + 1, 0);
            }
        }
        *sNext = u;
    }
    __syncthreads();
    const int u = *sNext;
    return u < units ? a.blockOrder[u] : units;
}

// Stages batch entry `slot` (if valid) and the masks: mask[w][g] bit b <=> entry 32g + b meets warp w.
template <int PB, int BD>
__device__ __forceinline__ void stage(const float4 *rec, const int2 *entries, int idx, bool valid, int slot, float4 *sP,
                                      float4 *sQ, float4 *sR, uint32_t (*mask)[RasterShape<PB, BD>::NG], int bx,
                                      int by)
{
    constexpr int NW = RasterShape<PB, BD>::NW, WX = RasterShape<PB, BD>::WX;
    float4 p = make_float4(0.0f, 0.0f, -1.0f, -1.0f), q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float powMin = 0.0f, iA = 0.0f, iC = 0.0f;
    if (valid) {
        const float4 *r = rec + size_t(entries[idx].x) * 3;
        p = r[0];
        q = r[1];
        const float4 c = r[2];
        // The blending loops read the mean from sP and the exponent floor (SplatRec::powMin) from its
        // third slot; the contributing box is only needed for the masks below.
        sP[slot] = make_float4(p.x, p.y, c.w, p.w);
        sQ[slot] = q;
        sR[slot] = c;
        powMin = c.w;
        iA = __frcp_rn(q.x);
        iC = __frcp_rn(q.z);
    }
    // The ellipse test refines the box test where the box extents are finite (well-conditioned
    // covariances and a positive minimum alpha).
    const bool fine = p.z < __int_as_float(0x7f800000);
    const int group = slot >> 5, lane = slot & 31;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        bool hit = valid && meets<PB>(p, w, bx, by);
        if (hit && fine)
            hit = ellipseMeets(p.x, p.y, q, powMin, iA, iC, float(bx * PB + (w % WX) * 8), float(by * PB + (w / WX) * 8));
        const uint32_t bits = __ballot_sync(0xffffffffu, hit);
        if (lane == 0)
            mask[w][group] = bits;
    }
}

// Gaussian falloff exponent at one pixel, in the reference's operation order with no fused
// multiply-add (Rasterizer.cpp:305-306), so every kernel decides contributions identically:
//   power = -0.5 * ((A dx) dx + (C dy) dy) - (B dx) dy.
// A thread's two pixels share a column, so the dx terms are computed once (columnTerms) and give the
// same roundings as computing them per pixel.
struct ColumnTerms {
    float axx; // (A dx) dx
    float bx;  // B dx
};

__device__ __forceinline__ ColumnTerms columnTerms(const float4 &Q, float dx)
{
    return {__fmul_rn(__fmul_rn(Q.x, dx), dx), __fmul_rn(Q.y, dx)};
}

__device__ __forceinline__ float powerAt(const float4 &Q, const ColumnTerms &c, float dy)
{
    const float q = __fadd_rn(c.axx, __fmul_rn(__fmul_rn(Q.z, dy), dy));
    return __fsub_rn(__fmul_rn(-0.5f, q), __fmul_rn(c.bx, dy));
}

__device__ __forceinline__ float rasterExp(float x) { return expf(x); }

// Paired FP32 arithmetic (sm_100: one instruction computes two float lanes), each lane rounded like
// the scalar __fmul_rn / __fadd_rn / __fmaf_rn. One caveat, measured with CUDA 12.9: a paired add
// whose operand is a paired product is fused into a single rounding by the code generator (for the
// float2 intrinsics, for these explicit .rn instructions, and with -fmad=false alike: on random inputs
// a + (z d) d came out fused in 23 % of the cases). So in arithmetic that decides which pairs
// contribute (the falloff exponent) the products are paired and the sums scalar (a scalar add of a
// lane of a paired product rounded separately in all of 3e8 random cases), and elsewhere paired
// instructions take only steps that have no product feeding a sum, or whose rounding is free
// (gradient arithmetic, colour sums).
__device__ __forceinline__ float2 mul2rn(float2 a, float2 b)
{
    float2 d;
    asm("{ .reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd; }"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 add2rn(float2 a, float2 b)
{
    float2 d;
    asm("{ .reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd; }"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// a * b + c per lane with one rounding (fma.rn.f32x2).
__device__ __forceinline__ float2 fma2rn(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("{ .reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd; }"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

} // namespace u3dg
