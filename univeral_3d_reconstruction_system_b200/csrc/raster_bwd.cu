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
//
// A thread's two pixels are replayed together in paired FP32 instructions (raster_common.cuh), one
// float2 lane per pixel; the falloff exponents' sums and the divisions stay scalar. A pixel that does
// not contribute at an entry keeps its state (selects) and adds zero to the sums.

#include "raster_common.cuh"

#include <algorithm>
#include <atomic>
#include <type_traits>

namespace u3dg {

namespace {

// Back-to-front replay state of a thread's two pixels (one float2 lane each). The colour behind the
// current entry enters the gradient only through its dot product with dL/dpixel, so the state keeps
// that scalar (the running sum over channels of accum[ch] * dpix[ch], kept negated: nacc) and the last
// contributor's colour dot product (lcd) instead of three channels each: the recurrence accum =
// lastAlpha * lastColour + (1 - lastAlpha) * accum is linear, so the dot products follow it too (the
// sums differ from the per-channel form by rounding only, within the gradient tolerance). lastAlpha is
// kept negated as well (nla), so every update is a paired add or fused multiply-add.
struct PixelPair {
    float2 T, nacc, lcd, nla; // transmittance, -(colour dot behind), last contributor's colour dot, -its alpha
    float2 d0, d1, d2, fy;    // dL/dpixel per channel, pixel row
    float2 fT, bgDot;         // final transmittance, background . dL/dpixel (background term only)
    int nC0, nC1;             // contributor counts
};

// Turns an entry's summed moments (the entry loop) into dL/dmean2d and dL/dconic (Rasterizer.cpp:405-412):
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

__device__ __forceinline__ PixelPair initPair(bool in0, bool in1, size_t pix0, size_t pix1, float fy0, float fy1,
                                              const float *dLdRgb, const float *finalT, const int *nContrib,
                                              const float *bg)
{
    PixelPair p;
    p.nC0 = in0 ? nContrib[pix0] : 0;
    p.nC1 = in1 ? nContrib[pix1] : 0;
    p.fT = make_float2(in0 ? finalT[pix0] : 0.0f, in1 ? finalT[pix1] : 0.0f);
    p.d0 = make_float2(in0 ? dLdRgb[pix0 * 3] : 0.0f, in1 ? dLdRgb[pix1 * 3] : 0.0f);
    p.d1 = make_float2(in0 ? dLdRgb[pix0 * 3 + 1] : 0.0f, in1 ? dLdRgb[pix1 * 3 + 1] : 0.0f);
    p.d2 = make_float2(in0 ? dLdRgb[pix0 * 3 + 2] : 0.0f, in1 ? dLdRgb[pix1 * 3 + 2] : 0.0f);
    p.bgDot = make_float2(bg[0] * p.d0.x + bg[1] * p.d1.x + bg[2] * p.d2.x, bg[0] * p.d0.y + bg[1] * p.d1.y + bg[2] * p.d2.y);
    p.T = p.fT;
    p.nacc = p.lcd = p.nla = make_float2(0.0f, 0.0f);
    p.fy = make_float2(fy0, fy1);
    return p;
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
    PixelPair pp = initPair(in0, in1, in0 ? size_t(wb.py0) * a.width + wb.px : 0,
                            in1 ? size_t(wb.py1) * a.width + wb.px : 0, float(wb.py0), float(wb.py1), dLdRgb,
                            finalTIn, nContribIn, a.bg);
    const float2 one2 = make_float2(1.0f, 1.0f);
    const float fx = float(wb.px);
    const float minA = a.minAlpha;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    const int vIdx = (lane >> 2) & 7; // value held after warpReduce9 (lanes 4v)
    if (tid == 0)
        sMax = 0;
    __syncthreads();
    const int nMax = max(pp.nC0, pp.nC1);
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
            float *dst = partial + size_t(a.entries[start + j].y) * kG2d;
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
            stage<PB, BD>(rec, a.entries, start + bStart + slot, slot < cnt, slot, sP, sQ, sR, mask, bx, by);
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
                if (j < pp.nC0 || j < pp.nC1) {
                    const float4 P = sP[jj], Q = sQ[jj];
                    const float dx = __fsub_rn(P.x, fx);
                    const ColumnTerms ct = columnTerms(Q, dx);
                    // Falloff exponents exactly as the forward decides (powerAt's order; products
                    // paired, sums scalar).
                    const float2 dy = make_float2(__fsub_rn(P.y, pp.fy.x), __fsub_rn(P.y, pp.fy.y));
                    const float2 cdd = mul2rn(mul2rn(make_float2(Q.z, Q.z), dy), dy);
                    const float2 bdy = mul2rn(make_float2(ct.bx, ct.bx), dy);
                    const float2 hq = mul2rn(make_float2(-0.5f, -0.5f), make_float2(__fadd_rn(ct.axx, cdd.x), __fadd_rn(ct.axx, cdd.y)));
                    const float2 pw = make_float2(__fsub_rn(hq.x, bdy.x), __fsub_rn(hq.y, bdy.y));
                    bool v0 = j < pp.nC0 && !(pw.x > 0.0f || pw.x < P.z);
                    bool v1 = j < pp.nC1 && !(pw.y > 0.0f || pw.y < P.z);
                    if (v0 || v1) {
                        // One back-to-front step of Rasterizer.cpp:385-416 for both pixels (a pixel that
                        // is out gets exp(0) and zero weights, and keeps its state).
                        const float2 G = make_float2(rasterExp(v0 ? pw.x : 0.0f), rasterExp(v1 ? pw.y : 0.0f));
                        const float2 raw = mul2rn(make_float2(Q.w, Q.w), G);
                        const float al0 = (raw.x < kMaxAlpha) ? raw.x : kMaxAlpha;
                        const float al1 = (raw.y < kMaxAlpha) ? raw.y : kMaxAlpha;
                        v0 = v0 && !(al0 < minA);
                        v1 = v1 && !(al1 < minA);
                        if (v0 || v1) {
                            act = true;
                            const float4 R = sR[jj];
                            // Transmittance before this entry: T / (1 - alpha), correctly rounded.
                            const float2 om = add2rn(one2, make_float2(-al0, -al1));
                            const float Tn0 = __fdiv_rn(pp.T.x, om.x), Tn1 = __fdiv_rn(pp.T.y, om.y);
                            pp.T = make_float2(v0 ? Tn0 : pp.T.x, v1 ? Tn1 : pp.T.y);
                            const float2 w = mul2rn(make_float2(v0 ? al0 : 0.0f, v1 ? al1 : 0.0f), pp.T);
                            // dAlpha = (colour . dpix - accum . dpix) T (Rasterizer.cpp:393-399), on the
                            // dot products; accum takes the previous contributor's colour first.
                            const float2 rd = fma2rn(make_float2(R.z, R.z), pp.d2,
                                                         fma2rn(make_float2(R.y, R.y), pp.d1,
                                                                    mul2rn(make_float2(R.x, R.x), pp.d0)));
                            const float2 nacc = fma2rn(pp.nla, add2rn(pp.lcd, pp.nacc), pp.nacc);
                            float2 dAl = mul2rn(add2rn(rd, nacc), pp.T);
                            pp.nacc = make_float2(v0 ? nacc.x : pp.nacc.x, v1 ? nacc.y : pp.nacc.y);
                            pp.lcd = make_float2(v0 ? rd.x : pp.lcd.x, v1 ? rd.y : pp.lcd.y);
                            pp.nla = make_float2(v0 ? -al0 : pp.nla.x, v1 ? -al1 : pp.nla.y);
                            const float2 wd0 = mul2rn(w, pp.d0), wd1 = mul2rn(w, pp.d1), wd2 = mul2rn(w, pp.d2);
                            c[5] = wd0.x + wd0.y;
                            c[6] = wd1.x + wd1.y;
                            c[7] = wd2.x + wd2.y;
                            if (kBg) {
                                dAl.x += -pp.fT.x / om.x * pp.bgDot.x;
                                dAl.y += -pp.fT.y / om.y * pp.bgDot.y;
                            }
                            // A clamped alpha has a colour gradient only.
                            const bool m0 = v0 && !(raw.x > kMaxAlpha), m1 = v1 && !(raw.y > kMaxAlpha);
                            float2 t = mul2rn(G, dAl);
                            t = make_float2(m0 ? t.x : 0.0f, m1 ? t.y : 0.0f);
                            c[8] = t.x + t.y;
                            // The mean and conic gradients are linear in the per-pixel moments of dPow
                            // (finishEntry combines them with the conic once per entry); both pixels
                            // share dx, so dx multiplies the thread's sums once.
                            const float2 dPow = mul2rn(make_float2(Q.w, Q.w), t);
                            const float2 pdy = mul2rn(dPow, dy);
                            const float2 pdyy = mul2rn(pdy, dy);
                            c[1] = pdy.x + pdy.y;
                            c[4] = pdyy.x + pdyy.y;
                            c[0] = dx * (dPow.x + dPow.y);
                            c[2] = dx * c[0];
                            c[3] = dx * c[1];
                        }
                    }
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
            float *dst = partial + size_t(a.entries[start + bStart + e].y) * kG2d;
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
