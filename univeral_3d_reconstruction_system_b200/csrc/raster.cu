// raster.cu - tile compositing forward (Rasterizer::forward, Rasterizer.cpp:281-329).
//
// Layout and staging in raster_common.cuh: a CTA per 16x16 or 8x8 pixel block, two pixels per thread,
// 8x8 pixels per warp, batches of one or two list entries per thread staged in shared memory with
// per-warp masks of the entries whose contributing box meets the warp's block. A tile of 16 or 32
// pixels may be covered by several 8x8 CTAs that each walk the whole tile list (RasterArgs::
// forwardBlock): more, shorter CTAs keep the SMs busy while the heaviest tiles finish. Each warp walks its set bits in list
// order and blends both of its pixels' columns, front to back, with the reference's cut-offs
// (alpha <= 0.99, skip alpha < minAlpha, stop when T (1 - alpha) < minTransmittance). A CTA stops when
// every pixel has terminated (__syncthreads_count). Skipped entries are exactly those the reference
// skips for these pixels, so the output is unchanged.
//
// Compiled with -fmad=false: the contribution decisions (power, alpha, the transmittance cut-off) and
// the transmittance round exactly like the reference's, so the same entries contribute. The colour
// sums alone use explicit fused multiply-adds (within 1e-7 of the unfused sums; images are compared
// within 1e-5). A thread's two pixels are blended together in sm_100's paired FP32 instructions
// (add2rn / mul2rn / fma2rn, raster_common.cuh), which round each lane like the scalar operation.

#include "raster_common.cuh"

#include <algorithm>

namespace u3dg {

namespace {

template <int PB, int BD>
__device__ __forceinline__ void forwardBlock(const RasterArgs &a, int bx, int by, float *rgb, float *finalT,
                                             int *nContrib, float4 *sP, float4 *sQ, float4 *sR,
                                             uint32_t (*mask)[RasterShape<PB, BD>::NG])
{
    using S = RasterShape<PB, BD>;
    constexpr int NT = S::NT, NB = S::NB, NG = S::NG;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const WarpBlock<PB> wb(warp, lane, bx, by);
    const int tile = tileOf<PB>(a, bx, by);
    const int start = a.tileOffsets[tile], end = a.tileOffsets[tile + 1];
    const bool in0 = wb.px < a.width && wb.py0 < a.height, in1 = wb.px < a.width && wb.py1 < a.height;
    bool done0 = !in0, done1 = !in1;
    float2 T = make_float2(1.0f, 1.0f), cr = make_float2(0.0f, 0.0f), cg = cr, cb = cr;
    int last0 = 0, last1 = 0;
    const float fx = float(wb.px), fy0 = float(wb.py0), fy1 = float(wb.py1);
    const float2 one = make_float2(1.0f, 1.0f);
    const float minA = a.minAlpha, minT = a.minTransmittance;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    for (int b0 = start; b0 < end; b0 += NB) {
        if (__syncthreads_count(done0 && done1) == NT)
            break;
#pragma unroll
        for (int r = 0; r < BD; ++r) {
            const int slot = r * NT + tid;
            stage<PB, BD>(rec, a.entries, b0 + slot, b0 + slot < end, slot, sP, sQ, sR, mask, bx, by);
        }
        __syncthreads();
        for (int k = 0; k < NG && !(done0 && done1); ++k) {
            uint32_t bits = mask[warp][k];
            while (bits) {
                const int j = 32 * k + __ffs(bits) - 1;
                bits &= bits - 1;
                // One front-to-back blending step of Rasterizer.cpp:305-318 for both of the thread's
                // pixels at once, in paired FP32 instructions where each lane rounds like the scalar
                // operation: the falloff exponent in powerAt's order (products paired, sums scalar),
                // alpha, 1 - alpha, T (1 - alpha) and alpha T, and the colour sums as paired fused
                // multiply-adds; the cut-offs per pixel.
                const float4 P = sP[j], Q = sQ[j];
                const ColumnTerms ct = columnTerms(Q, P.x - fx);
                const float2 dy = make_float2(P.y - fy0, P.y - fy1);
                const float2 cdd = mul2rn(mul2rn(make_float2(Q.z, Q.z), dy), dy);
                const float2 bdy = mul2rn(make_float2(ct.bx, ct.bx), dy);
                const float2 hq = mul2rn(make_float2(-0.5f, -0.5f), make_float2(__fadd_rn(ct.axx, cdd.x), __fadd_rn(ct.axx, cdd.y)));
                const float2 pw = make_float2(__fsub_rn(hq.x, bdy.x), __fsub_rn(hq.y, bdy.y));
                bool v0 = !done0 && !(pw.x > 0.0f || pw.x < P.z);
                bool v1 = !done1 && !(pw.y > 0.0f || pw.y < P.z);
                if (v0 || v1) {
                    // A pixel that is out gets exp(0), whose alpha it never uses.
                    const float2 G = make_float2(rasterExp(v0 ? pw.x : 0.0f), rasterExp(v1 ? pw.y : 0.0f));
                    const float2 raw = mul2rn(make_float2(Q.w, Q.w), G);
                    const float al0 = (raw.x < kMaxAlpha) ? raw.x : kMaxAlpha;
                    const float al1 = (raw.y < kMaxAlpha) ? raw.y : kMaxAlpha;
                    v0 = v0 && !(al0 < minA);
                    v1 = v1 && !(al1 < minA);
                    const float2 nT = mul2rn(T, add2rn(one, make_float2(-al0, -al1)));
                    if (v0 && nT.x < minT) {
                        done0 = true;
                        v0 = false;
                    }
                    if (v1 && nT.y < minT) {
                        done1 = true;
                        v1 = false;
                    }
                    float2 w = mul2rn(make_float2(al0, al1), T);
                    w.x = v0 ? w.x : 0.0f; // a pixel that does not blend adds R * 0 = 0 to its sums
                    w.y = v1 ? w.y : 0.0f;
                    const float4 R = sR[j];
                    cr = fma2rn(make_float2(R.x, R.x), w, cr);
                    cg = fma2rn(make_float2(R.y, R.y), w, cg);
                    cb = fma2rn(make_float2(R.z, R.z), w, cb);
                    const int idx = b0 - start + j + 1;
                    if (v0) {
                        T.x = nT.x;
                        last0 = idx;
                    }
                    if (v1) {
                        T.y = nT.y;
                        last1 = idx;
                    }
                }
                if (done0 && done1)
                    break;
            }
        }
    }
    const float T0 = T.x, T1 = T.y, r0 = cr.x, r1 = cr.y, g0 = cg.x, g1 = cg.y, b0c = cb.x, b1c = cb.y;
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

// Resident CTAs per SM the compiler must allow for: caps registers per thread at 65536 / (NT * n)
// (48 at 10 for NT = 128).
#ifndef U3DG_FWD_MIN_BLOCKS
#define U3DG_FWD_MIN_BLOCKS 10
#endif

template <int PB, int BD>
__global__ void __launch_bounds__(RasterShape<PB>::NT, U3DG_FWD_MIN_BLOCKS) compositeForwardKernel(RasterArgs a, float *rgb, float *finalT,
                                                                              int *nContrib)
{
    pdlEntry();
    using S = RasterShape<PB, BD>;
    constexpr int NB = S::NB, NW = S::NW, NG = S::NG;
    __shared__ float4 sP[NB]; // mx, my, powMin, ey
    __shared__ float4 sQ[NB]; // A, B, C, alpha
    __shared__ float4 sR[NB]; // r, g, b, powMin
    __shared__ uint32_t mask[NW][NG];
    __shared__ int sNext;
    const int units = a.blocksX * a.blocksY;
    if (a.counters == nullptr) { // one CTA per pixel block (every block resident in one wave)
        forwardBlock<PB, BD>(a, int(blockIdx.x) % a.blocksX, int(blockIdx.x) / a.blocksX, rgb, finalT, nContrib, sP,
                             sQ, sR, mask);
        return;
    }
    for (int b = nextBlock(a, a.counters, &sNext); b < units; b = nextBlock(a, a.counters, &sNext))
        forwardBlock<PB, BD>(a, b % a.blocksX, b / a.blocksX, rgb, finalT, nContrib, sP, sQ, sR, mask);
}

// One CTA: the pixel blocks bucketed by the list length of their tile on a log scale (four buckets
// per power of two), longest first. The order only schedules work (every block's result is the same
// whichever CTA computes it when), so blocks within a bucket may come in any order.
constexpr int kOrderBuckets = 132;

__device__ __forceinline__ int lengthBucket(unsigned len)
{
    if (len == 0)
        return kOrderBuckets - 1;
    const int msb = 31 - __clz(len);
    const int sub = msb >= 2 ? int((len >> (msb - 2)) & 3u) : int((len << (2 - msb)) & 3u);
    return kOrderBuckets - 2 - (msb * 4 + sub); // longer lists: smaller bucket index
}

__global__ void __launch_bounds__(1024) blockOrderKernel(const int *tileOffsets, int blocksX, int blocksY, int pb,
                                                         int tileSize, int tilesX, int *order)
{
    pdlEntry();
    __shared__ int count[kOrderBuckets];
    __shared__ int cursor[kOrderBuckets];
    const int units = blocksX * blocksY;
    for (int b = threadIdx.x; b < kOrderBuckets; b += blockDim.x)
        count[b] = 0;
    __syncthreads();
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int bx = u % blocksX, by = u / blocksX;
        const int t = (by * pb / tileSize) * tilesX + bx * pb / tileSize;
        atomicAdd(&count[lengthBucket(unsigned(tileOffsets[t + 1] - tileOffsets[t]))], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) { // exclusive scan of the bucket counts: each lane owns kPer consecutive buckets
        constexpr int kPer = (kOrderBuckets + 31) / 32;
        const int lane = threadIdx.x, b0 = lane * kPer;
        int own = 0;
        for (int b = b0; b < b0 + kPer && b < kOrderBuckets; ++b)
            own += count[b];
        int incl = own;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        int run = incl - own;
        for (int b = b0; b < b0 + kPer && b < kOrderBuckets; ++b) {
            cursor[b] = run;
            run += count[b];
        }
    }
    __syncthreads();
    for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int bx = u % blocksX, by = u / blocksX;
        const int t = (by * pb / tileSize) * tilesX + bx * pb / tileSize;
        const int pos = atomicAdd(&cursor[lengthBucket(unsigned(tileOffsets[t + 1] - tileOffsets[t]))], 1);
        order[pos] = u;
    }
}

// CTAs that can be resident at once for a kernel (cached per kernel and dynamic shared memory size).
template <class K>
int residentCtas(K kernel, int threads, size_t smem)
{
    int dev = 0, sms = 0, perSm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, smem);
    return std::max(1, sms * std::max(1, perSm));
}

} // namespace

void launchBlockOrder(const RasterArgs &a, int *order, cudaStream_t s)
{
    const int units = a.blocksX * a.blocksY;
    if (units <= 0)
        return;
    const int pb = a.tileSize <= 8 ? 8 : 16;
    { launchPdl(blockOrderKernel, 1, 1024, 0, s, a.tileOffsets, a.blocksX, a.blocksY, pb, a.tileSize, a.tilesX, order); countLaunch(); }
}

template <int PB, int BD>
static void launchForward(const RasterArgs &a, float *rgb, float *finalT, int *nContrib, cudaStream_t s)
{
    // When every pixel block fits on the GPU at once, one CTA per block in natural order (no work
    // counter); otherwise the persistent schedule on counters[0..1].
    const int units = a.blocksX * a.blocksY;
    static const int ctas = residentCtas(compositeForwardKernel<PB, BD>, RasterShape<PB>::NT, 0);
    RasterArgs f = a;
    if (units <= ctas)
        f.counters = nullptr;
    { launchPdl(compositeForwardKernel<PB, BD>, std::min(units, ctas), RasterShape<PB>::NT, 0, s, f, rgb, finalT, nContrib); countLaunch(); }
}

// 8x8 CTAs over the lists of larger tiles: one CTA per pixel block in natural order, as many waves as
// it takes (the blocks are short; the persistent order is computed for the backward's blocks).
template <int BD>
static void launchForwardSplit(const RasterArgs &a, float *rgb, float *finalT, int *nContrib, cudaStream_t s)
{
    RasterArgs f = a;
    f.blocksX = (a.width + 7) / 8;
    f.blocksY = (a.height + 7) / 8;
    f.counters = nullptr;
    { launchPdl(compositeForwardKernel<8, BD>, f.blocksX * f.blocksY, RasterShape<8>::NT, 0, s, f, rgb, finalT, nContrib); countLaunch(); }
}

void launchCompositeForward(const RasterArgs &a, float *rgb, float *finalT, int *nContrib, cudaStream_t s)
{
    if (a.blocksX * a.blocksY <= 0)
        return;
    const bool deep = a.forwardDepth >= 2;
    if (a.tileSize > 8 && a.forwardBlock == 8)
        deep ? launchForwardSplit<2>(a, rgb, finalT, nContrib, s) : launchForwardSplit<1>(a, rgb, finalT, nContrib, s);
    else if (a.tileSize <= 8)
        deep ? launchForward<8, 2>(a, rgb, finalT, nContrib, s) : launchForward<8, 1>(a, rgb, finalT, nContrib, s);
    else
        deep ? launchForward<16, 2>(a, rgb, finalT, nContrib, s) : launchForward<16, 1>(a, rgb, finalT, nContrib, s);
}

} // namespace u3dg
