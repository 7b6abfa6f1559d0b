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
// within 1e-5).

#include "raster_common.cuh"

#include <algorithm>

namespace u3dg {

namespace {

// One front-to-back blending step of Rasterizer.cpp:305-318 for one pixel.
__device__ __forceinline__ void blend(const float4 &P, const float4 &Q, const float4 *sR, int j, const ColumnTerms &ct,
                                      float fy, float minA, float minT, int lastIdx, float &T, float &cr, float &cg,
                                      float &cb, int &last, bool &done)
{
    const float dy = P.y - fy;
    const float power = powerAt(Q, ct, dy);
    if (power > 0.0f || power < P.z) // P.z: SplatRec::powMin
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
    cr = __fmaf_rn(R.x, w, cr);
    cg = __fmaf_rn(R.y, w, cg);
    cb = __fmaf_rn(R.z, w, cb);
    T = nextT;
    last = lastIdx;
}

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
    float T0 = 1.0f, r0 = 0.0f, g0 = 0.0f, b0c = 0.0f;
    float T1 = 1.0f, r1 = 0.0f, g1 = 0.0f, b1c = 0.0f;
    int last0 = 0, last1 = 0;
    const float fx = float(wb.px), fy0 = float(wb.py0), fy1 = float(wb.py1);
    const float minA = a.minAlpha, minT = a.minTransmittance;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    for (int b0 = start; b0 < end; b0 += NB) {
        if (__syncthreads_count(done0 && done1) == NT)
            break;
#pragma unroll
        for (int r = 0; r < BD; ++r) {
            const int slot = r * NT + tid;
            stage<PB, BD>(rec, a.list, b0 + slot, b0 + slot < end, slot, sP, sQ, sR, mask, bx, by);
        }
        __syncthreads();
        for (int k = 0; k < NG && !(done0 && done1); ++k) {
            uint32_t bits = mask[warp][k];
            while (bits) {
                const int j = 32 * k + __ffs(bits) - 1;
                bits &= bits - 1;
                const float4 P = sP[j], Q = sQ[j];
                const ColumnTerms ct = columnTerms(Q, P.x - fx);
                const int idx = b0 - start + j + 1;
                if (!done0)
                    blend(P, Q, sR, j, ct, fy0, minA, minT, idx, T0, r0, g0, b0c, last0, done0);
                if (!done1)
                    blend(P, Q, sR, j, ct, fy1, minA, minT, idx, T1, r1, g1, b1c, last1, done1);
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
    if (threadIdx.x == 0) {
        int run = 0;
        for (int b = 0; b < kOrderBuckets; ++b) {
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
