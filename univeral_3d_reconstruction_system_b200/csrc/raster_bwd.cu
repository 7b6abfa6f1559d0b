// raster_bwd.cu - tile compositing backward (Rasterizer::backward pass 1, Rasterizer.cpp:353-427).
//
// Same CTA / warp / batch layout as the forward (raster_common.cuh). Each pixel walks its tile list
// back to front from its contributor count with the reference's recurrence (transmittance recovered
// by division, running colour accumulation, clamp handling). A thread holds two pixels and adds their
// contributions before the warp sum, so one warp reduction covers 64 pixels. The 9 sums per list entry
// (dmean2d xy, dconic ABC, drgb, dalpha) go through a reduce-scatter (14 shuffles), land in a
// per-warp shared-memory slot, and are added over the warps in warp order after the batch: the result
// does not depend on scheduling. Each (tile, Gaussian) partial is stored once at the entry's emission
// index, zero for entries behind every pixel's last contributor; the chain-rule kernel sums a
// Gaussian's partials in tile order. Tiles of 32 or 64 pixels span 4 or 16 CTAs (16x16 blocks): each
// stores into its own slot array and the chain-rule kernel adds the slots in a fixed order, so every
// tile size gives deterministic gradients (no atomics).
//
// Contribution decisions (power, alpha, the cut-offs) and the transmittance recovery are computed with
// explicitly unfused operations, exactly as in the forward, so the backward visits the same entries;
// the gradient arithmetic may use fused multiply-add (gradients are compared within a relative
// tolerance). The recovery keeps the correctly rounded division: an approximate division (2 ulp) or a
// reciprocal-multiply made the backward 3 % faster but moved some colour gradients just past 1e-4
// relative to the reference's.

#include "raster_common.cuh"

#include <algorithm>
#include <atomic>
#include <type_traits>

namespace u3dg {

namespace {

// Per-pixel state of the back-to-front replay. The colour behind the current entry enters the
// gradient only through its dot product with dL/dpixel, so the state keeps that scalar (accd, the
// running sum over channels of accum[ch] * dpix[ch]) and the last entry's colour dot product (lcd)
// instead of three channels each: the recurrence accum = lastAlpha * lastColour + (1 - lastAlpha) *
// accum is linear, so accd follows the same recurrence on the dot products. Three fewer multiply-adds
// per channel per pair and eight fewer live registers for a thread's two pixels (no spills); the sums
// differ from the per-channel form by rounding only (within the gradient tolerance).
struct PixelState {
    float T, accd, lcd, lastAlpha;
    float fT, d0, d1, d2, bgDot, fy;
    int nC;
};

// One back-to-front step of Rasterizer.cpp:385-416 for one pixel; adds its 9 contributions to c.
// kBg: the background is not black (its term enters dAlpha).
template <bool kBg>
__device__ __forceinline__ bool pairGrad(const float4 &P, const float4 &Q, const float4 *sR, int jj, float dx,
                                         const ColumnTerms &ct, float minA, PixelState &s, float c[kG2d])
{
    const float dy = __fsub_rn(P.y, s.fy);
    const float power = powerAt(Q, ct, dy);
    if (power > 0.0f || power < P.z) // P.z: SplatRec::powMin
        return false;
    const float G = rasterExp(power);
    const float raw = __fmul_rn(Q.w, G);
    const float al = (raw < kMaxAlpha) ? raw : kMaxAlpha;
    if (al < minA)
        return false;
    const float4 R = sR[jj];
    s.T = __fdiv_rn(s.T, __fsub_rn(1.0f, al));
    const float w = al * s.T;
    // dAlpha = sum_ch (colour[ch] - accum[ch]) * dpix[ch] * T (Rasterizer.cpp:393-399), on dot products.
    const float rd = R.x * s.d0 + R.y * s.d1 + R.z * s.d2;
    s.accd = s.accd + s.lastAlpha * (s.lcd - s.accd); // lastAlpha * lcd + (1 - lastAlpha) * accd
    s.lcd = rd;
    float dAl = (rd - s.accd) * s.T;
    c[5] += w * s.d0;
    c[6] += w * s.d1;
    c[7] += w * s.d2;
    s.lastAlpha = al;
    // -finalT / (1 - alpha) * bgDot: with a black background (kBg false) it would add a signed zero,
    // which leaves dAl unchanged, so those launches compile it out.
    if (kBg)
        dAl += -s.fT / (1.0f - al) * s.bgDot;
    if (raw > kMaxAlpha)
        return true; // clamped alpha: colour gradient only
    const float t = G * dAl;
    c[8] += t;
    // The mean and conic gradients are linear in the per-pixel moments of dPow: sum dPow dx, dPow dy,
    // dPow dx^2, dPow dx dy, dPow dy^2, and combine them with the conic once per list entry
    // (finishEntry) instead of once per pixel. A thread's two pixels share dx, so the pixels add
    // sum dPow (c[0]), dPow dy (c[1]) and dPow dy^2 (c[4]) only; the thread multiplies by dx once
    // (c[0] -> dx sum dPow, c[2] = dx^2 sum dPow, c[3] = dx sum dPow dy) before the warp sum.
    const float dPow = Q.w * t;
    const float pdy = dPow * dy;
    c[0] += dPow;
    c[1] += pdy;
    c[4] += pdy * dy;
    return true;
}

// Turns an entry's summed moments (pairGrad) into dL/dmean2d and dL/dconic (Rasterizer.cpp:405-412):
// dmean = -(A m_x + B m_y, C m_y + B m_x), dA = -m_xx / 2, dB = -m_xy, dC = -m_yy / 2.
__device__ __forceinline__ void finishEntry(const float4 &Q, float g[kG2d])
{
    const float mx = g[0], my = g[1];
    g[0] = -(Q.x * mx + Q.y * my);
    g[1] = -(Q.z * my + Q.y * mx);
    g[2] = -0.5f * g[2];
    g[3] = -g[3];
    g[4] = -0.5f * g[4];
}

// Sum of c[0..8] over the warp: values 0..7 by reduce-scatter (xor 16/8/4 exchanges halve the
// values a lane holds; xor 2/1 finish), value 8 by a butterfly. Lane 4v gets value v, every lane v8.
__device__ __forceinline__ float warpReduce9(const float c[kG2d], int lane, float *v8)
{
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    float w4[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float send = b4 ? c[i] : c[i + 4];
        const float keep = b4 ? c[i + 4] : c[i];
        w4[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    float w2[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float send = b3 ? w4[i] : w4[i + 2];
        const float keep = b3 ? w4[i + 2] : w4[i];
        w2[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    float v;
    {
        const float send = b2 ? w2[0] : w2[1];
        const float keep = b2 ? w2[1] : w2[0];
        v = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    float e = c[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        e += __shfl_xor_sync(0xffffffffu, e, o);
    *v8 = e;
    return v;
}

__device__ __forceinline__ void initPixel(PixelState &s, bool inside, size_t pix, float fy, const float *dLdRgb,
                                          const float *finalT, const int *nContrib, const float *bg)
{
    s.nC = inside ? nContrib[pix] : 0;
    s.fT = inside ? finalT[pix] : 0.0f;
    s.d0 = inside ? dLdRgb[pix * 3] : 0.0f;
    s.d1 = inside ? dLdRgb[pix * 3 + 1] : 0.0f;
    s.d2 = inside ? dLdRgb[pix * 3 + 2] : 0.0f;
    s.bgDot = bg[0] * s.d0 + bg[1] * s.d1 + bg[2] * s.d2;
    s.T = s.fT;
    s.accd = s.lcd = s.lastAlpha = 0.0f;
    s.fy = fy;
}

template <int PB, int BD, bool kBg>
__device__ __forceinline__ void backwardBlock(const RasterArgs &a, int bx, int by, const float *dLdRgb,
                                              const float *finalTIn, const int *nContribIn, float *partial,
                                              float4 *sP, float4 *sQ, float4 *sR,
                                              uint32_t (*mask)[RasterShape<PB, BD>::NG], int &sMax, float *sWarp)
{
    using S = RasterShape<PB, BD>;
    constexpr int NT = S::NT, NW = S::NW, NB = S::NB, NG = S::NG;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const WarpBlock<PB> wb(warp, lane, bx, by);
    const int tile = tileOf<PB>(a, bx, by);
    const int start = a.tileOffsets[tile], end = a.tileOffsets[tile + 1];
    const bool in0 = wb.px < a.width && wb.py0 < a.height, in1 = wb.px < a.width && wb.py1 < a.height;
    if (a.subSlots > 1) { // this block's slot array: its position in the tile, row-major
        const int per = a.tileSize / PB;
        partial += size_t((by % per) * per + bx % per) * a.subStride;
    }
    PixelState s0, s1;
    initPixel(s0, in0, in0 ? size_t(wb.py0) * a.width + wb.px : 0, float(wb.py0), dLdRgb, finalTIn, nContribIn, a.bg);
    initPixel(s1, in1, in1 ? size_t(wb.py1) * a.width + wb.px : 0, float(wb.py1), dLdRgb, finalTIn, nContribIn, a.bg);
    const float fx = float(wb.px);
    const float minA = a.minAlpha;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    const int vIdx = (lane >> 2) & 7; // value held after warpReduce9 (lanes 4v)
    if (tid == 0)
        sMax = 0;
    __syncthreads();
    const int nMax = max(s0.nC, s1.nC);
    if (nMax > 0)
        atomicMax(&sMax, nMax);
    // This warp's pixels have no contributor at or beyond wMax: the warp skips those entries.
    const int wMax = __reduce_max_sync(0xffffffffu, nMax);
    __syncthreads();
    const int jmax = sMax;
    // Entries behind every pixel's last contributor get no gradient (the reference's per-tile
    // accumulators start at zero); their partials are still written, as the chain-rule kernel sums
    // every intersection of a Gaussian.
    for (int j = jmax + tid; j < end - start; j += NT) {
            float *dst = partial + size_t(a.listEmit[start + j]) * kG2d;
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                dst[k] = 0.0f;
        }
    float *myWarp = sWarp + size_t(warp) * NB * kG2d;
    for (int bEnd = jmax; bEnd > 0; bEnd -= NB) {
        const int bStart = max(0, bEnd - NB), cnt = bEnd - bStart;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < BD; ++r) {
            const int slot = r * NT + tid;
            stage<PB, BD>(rec, a.list, start + bStart + slot, slot < cnt, slot, sP, sQ, sR, mask, bx, by);
        }
        {
            float4 *z = reinterpret_cast<float4 *>(sWarp);
            for (int k = tid; k < NW * NB * kG2d / 4; k += NT)
                z[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        __syncthreads();
        for (int k = NG - 1; k >= 0; --k) {
            uint32_t bits = mask[warp][k];
            const int lim = wMax - bStart - 32 * k; // entries of this group below wMax
            if (lim <= 0)
                continue;
            if (lim < 32)
                bits &= (1u << lim) - 1u;
            while (bits) {
                const int hb = 31 - __clz(bits);
                bits &= ~(1u << hb);
                const int jj = 32 * k + hb;
                const int j = bStart + jj;
                float c[kG2d];
#pragma unroll
                for (int q = 0; q < kG2d; ++q)
                    c[q] = 0.0f;
                bool act = false;
                if (j < s0.nC || j < s1.nC) {
                    const float4 P = sP[jj], Q = sQ[jj];
                    const float dx = __fsub_rn(P.x, fx);
                    const ColumnTerms ct = columnTerms(Q, dx);
                    if (j < s0.nC)
                        act |= pairGrad<kBg>(P, Q, sR, jj, dx, ct, minA, s0, c);
                    if (j < s1.nC)
                        act |= pairGrad<kBg>(P, Q, sR, jj, dx, ct, minA, s1, c);
                    c[3] = dx * c[1];
                    c[0] = dx * c[0];
                    c[2] = dx * c[0]; // c[0] already holds dx sum dPow
                }
                if (__any_sync(0xffffffffu, act)) {
                    float v8;
                    const float v = warpReduce9(c, lane, &v8);
                    if ((lane & 3) == 0)
                        myWarp[jj * kG2d + vIdx] = v;
                    if (lane == 1)
                        myWarp[jj * kG2d + 8] = v8;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < BD; ++r) {
            const int e = r * NT + tid;
            if (e >= cnt)
                break;
            float sum[kG2d];
#pragma unroll
            for (int q = 0; q < kG2d; ++q)
                sum[q] = sWarp[e * kG2d + q];
            for (int w = 1; w < NW; ++w)
#pragma unroll
                for (int q = 0; q < kG2d; ++q)
                    sum[q] += sWarp[(size_t(w) * NB + e) * kG2d + q];
            finishEntry(sQ[e], sum);
            float *dst = partial + size_t(a.listEmit[start + bStart + e]) * kG2d;
#pragma unroll
            for (int q = 0; q < kG2d; ++q)
                dst[q] = sum[q];
        }
    }
}

// Resident CTAs per SM the compiler must allow for: caps registers per thread at 65536 / (NT * n)
// (80 at 6 for NT = 128; without a cap ptxas takes 105 and only 4 CTAs fit).
#ifndef U3DG_BWD_MIN_BLOCKS
#define U3DG_BWD_MIN_BLOCKS 6
#endif
// Shared-memory carveout hint in percent of the maximum (negative: the driver's default). More shared
// memory admits more CTAs but leaves less L1 for the record gathers.
#ifndef U3DG_BWD_CARVEOUT
#define U3DG_BWD_CARVEOUT -1
#endif

template <int PB, int BD, bool kBg>
__global__ void __launch_bounds__(RasterShape<PB>::NT, U3DG_BWD_MIN_BLOCKS) compositeBackwardKernel(RasterArgs a, const float *dLdRgb,
                                                                              const float *finalTIn,
                                                                              const int *nContribIn, float *partial)
{
    pdlEntry();
    using S = RasterShape<PB, BD>;
    constexpr int NB = S::NB, NW = S::NW, NG = S::NG;
    __shared__ float4 sP[NB];
    __shared__ float4 sQ[NB];
    __shared__ float4 sR[NB];
    __shared__ uint32_t mask[NW][NG];
    __shared__ int sMax, sNext;
    extern __shared__ float sWarp[]; // NW slots of NB entries x 9 sums
    const int units = a.blocksX * a.blocksY;
    int *counter = a.counters + 2; // backward: counters[2..3]
    for (int b = nextBlock(a, counter, &sNext); b < units; b = nextBlock(a, counter, &sNext))
        backwardBlock<PB, BD, kBg>(a, b % a.blocksX, b / a.blocksX, dLdRgb, finalTIn, nContribIn, partial, sP, sQ, sR,
                              mask, sMax, sWarp);
}

template <class K>
int residentCtas(K kernel, int threads, size_t smem)
{
    int dev = 0, sms = 0, perSm = 0;
    if (U3DG_BWD_CARVEOUT >= 0)
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, U3DG_BWD_CARVEOUT);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, smem);
    return std::max(1, sms * std::max(1, perSm));
}

} // namespace

template <int PB, int BD, bool kBg>
static void launchBackward(const RasterArgs &a, const float *dLdRgb, const float *finalT, const int *nContrib,
                           float *partial, cudaStream_t s)
{
    using S = RasterShape<PB, BD>;
    const size_t smem = size_t(S::NW) * S::NB * kG2d * sizeof(float); // 18 KB (BD 1) or 36 KB (BD 2) at PB 16
    static const int ctas = [&] {
        cudaFuncSetAttribute(compositeBackwardKernel<PB, BD, kBg>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        return residentCtas(compositeBackwardKernel<PB, BD, kBg>, S::NT, smem);
    }();
    const int units = a.blocksX * a.blocksY;
    { launchPdl(compositeBackwardKernel<PB, BD, kBg>, std::min(units, ctas), S::NT, smem, s, a, dLdRgb, finalT, nContrib, partial); countLaunch(); }
}

void launchCompositeBackward(const RasterArgs &a, const float *dLdRgb, const float *finalT, const int *nContrib,
                             float *partial, cudaStream_t s)
{
    if (a.blocksX * a.blocksY <= 0)
        return;
    const bool deep = a.backwardDepth >= 2;
    const bool bg = a.bg[0] != 0.0f || a.bg[1] != 0.0f || a.bg[2] != 0.0f;
    auto run = [&](auto kBg) {
        constexpr bool B = decltype(kBg)::value;
        if (a.tileSize <= 8)
            deep ? launchBackward<8, 2, B>(a, dLdRgb, finalT, nContrib, partial, s)
                 : launchBackward<8, 1, B>(a, dLdRgb, finalT, nContrib, partial, s);
        else
            deep ? launchBackward<16, 2, B>(a, dLdRgb, finalT, nContrib, partial, s)
                 : launchBackward<16, 1, B>(a, dLdRgb, finalT, nContrib, partial, s);
    };
    if (bg)
        run(std::true_type{});
    else
        run(std::false_type{});
}

} // namespace u3dg
