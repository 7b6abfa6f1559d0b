// raster.cu - tile compositing forward (Rasterizer::forward, Rasterizer.cpp:281-329).
//
// Layout and staging in raster_common.cuh: a CTA per 16x16 pixel block, two pixels per thread, 8x8
// pixels per warp, batches of one list entry per thread staged in shared memory with per-warp masks of
// the entries whose contributing box meets the warp's block. Each warp walks its set bits in list
// order and blends both of its pixels' columns, front to back, with the reference's cut-offs
// (alpha <= 0.99, skip alpha < minAlpha, stop when T (1 - alpha) < minTransmittance). A CTA stops when
// every pixel has terminated (__syncthreads_count). Skipped entries are exactly those the reference
// skips for these pixels, so the output is unchanged.
//
// Compiled with -fmad=false: the per-pixel expressions round exactly like the reference's.

#include "raster_common.cuh"

namespace u3dg {

namespace {

// One front-to-back blending step of Rasterizer.cpp:305-318 for one pixel.
__device__ __forceinline__ void blend(const float4 &P, const float4 &Q, const float4 *sR, int j, float dx, float fy,
                                      float minA, float minT, int lastIdx, float &T, float &cr, float &cg, float &cb,
                                      int &last, bool &done)
{
    const float dy = P.y - fy;
    const float power = powerAt(Q, dx, dy);
    if (power > 0.0f)
        return;
    const float raw = Q.w * rasterExp(power);
    const float al = (raw < kMaxAlpha) ? raw : kMaxAlpha;
    if (al < minA)
        return;
    const float nextT = T * (1.0f - al);
    if (nextT < minT) {
        done = true;
        return;
    }
    const float w = al * T;
    const float4 R = sR[j];
    cr += R.x * w;
    cg += R.y * w;
    cb += R.z * w;
    T = nextT;
    last = lastIdx;
}

template <int PB>
__global__ void __launch_bounds__(RasterShape<PB>::NT) compositeForwardKernel(RasterArgs a, float *rgb, float *finalT,
                                                                              int *nContrib)
{
    using S = RasterShape<PB>;
    constexpr int NT = S::NT, NW = S::NW;
    __shared__ float4 sP[NT]; // mx, my, ex, ey
    __shared__ float4 sQ[NT]; // A, B, C, alpha
    __shared__ float4 sR[NT]; // r, g, b, depth
    __shared__ uint32_t mask[NW][NW];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const WarpBlock<PB> wb(warp, lane);
    const int tile = tileOf<PB>(a);
    const int start = a.tileOffsets[tile], end = a.tileOffsets[tile + 1];
    const bool in0 = wb.px < a.width && wb.py0 < a.height, in1 = wb.px < a.width && wb.py1 < a.height;
    bool done0 = !in0, done1 = !in1;
    float T0 = 1.0f, r0 = 0.0f, g0 = 0.0f, b0c = 0.0f;
    float T1 = 1.0f, r1 = 0.0f, g1 = 0.0f, b1c = 0.0f;
    int last0 = 0, last1 = 0;
    const float fx = float(wb.px), fy0 = float(wb.py0), fy1 = float(wb.py1);
    const float minA = a.minAlpha, minT = a.minTransmittance;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    for (int b0 = start; b0 < end; b0 += NT) {
        if (__syncthreads_count(done0 && done1) == NT)
            break;
        stage<PB>(rec, a.list, b0 + tid, b0 + tid < end, tid, sP, sQ, sR, mask);
        __syncthreads();
        for (int k = 0; k < NW && !(done0 && done1); ++k) {
            uint32_t bits = mask[warp][k];
            while (bits) {
                const int j = 32 * k + __ffs(bits) - 1;
                bits &= bits - 1;
                const float4 P = sP[j], Q = sQ[j];
                const float dx = P.x - fx;
                const int idx = b0 - start + j + 1;
                if (!done0)
                    blend(P, Q, sR, j, dx, fy0, minA, minT, idx, T0, r0, g0, b0c, last0, done0);
                if (!done1)
                    blend(P, Q, sR, j, dx, fy1, minA, minT, idx, T1, r1, g1, b1c, last1, done1);
                if (done0 && done1)
                    break;
            }
        }
    }
    if (in0) {
        const size_t pix = size_t(wb.py0) * a.width + wb.px;
        rgb[pix * 3] = r0 + T0 * a.bg[0];
        rgb[pix * 3 + 1] = g0 + T0 * a.bg[1];
        rgb[pix * 3 + 2] = b0c + T0 * a.bg[2];
        finalT[pix] = T0;
        nContrib[pix] = last0;
    }
    if (in1) {
        const size_t pix = size_t(wb.py1) * a.width + wb.px;
        rgb[pix * 3] = r1 + T1 * a.bg[0];
        rgb[pix * 3 + 1] = g1 + T1 * a.bg[1];
        rgb[pix * 3 + 2] = b1c + T1 * a.bg[2];
        finalT[pix] = T1;
        nContrib[pix] = last1;
    }
}

} // namespace

void launchCompositeForward(const RasterArgs &a, float *rgb, float *finalT, int *nContrib, cudaStream_t s)
{
    if (a.tileSize <= 8) {
        dim3 g((a.width + 7) / 8, (a.height + 7) / 8);
        { compositeForwardKernel<8><<<g, RasterShape<8>::NT, 0, s>>>(a, rgb, finalT, nContrib); countLaunch(); }
    } else {
        dim3 g((a.width + 15) / 16, (a.height + 15) / 16);
        { compositeForwardKernel<16><<<g, RasterShape<16>::NT, 0, s>>>(a, rgb, finalT, nContrib); countLaunch(); }
    }
}

} // namespace u3dg
