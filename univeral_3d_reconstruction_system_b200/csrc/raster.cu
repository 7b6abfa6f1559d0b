// raster.cu - tile compositing, forward and backward (Rasterizer.cpp:281-329 and 353-427).
//
// One CTA per 16x16 pixel block (8x8 when the tile size is 8), one thread per pixel; each warp owns an
// 8x4 pixel block. A tile's depth-sorted list is walked in batches of one record per thread, staged in
// shared memory. While staging, every warp also votes which of its 32 batch entries meet each warp's
// pixel block: a Gaussian's conservative contributing box (SplatRec::ex, ey) that misses a pixel
// block means alpha < minAlpha for all its pixels, which the reference skips too. Each warp then walks
// only the set bits of its mask, in list order, so most of the pixel-Gaussian pairs of a tile list
// cost nothing while every evaluated pair is computed exactly as the reference does. Forward stops a
// CTA once every pixel has terminated (transmittance cut-off), counted with __syncthreads_count.
//
// Backward walks the same lists back to front from each pixel's contributor count, with the
// reference's per-pixel recurrence. The 9 per-Gaussian 2D gradients of every list entry are summed
// over the warp by a reduce-scatter (14 shuffles for 9 values), then over the warps in shared memory,
// and stored once per (tile, Gaussian) at the entry's emission index: every Gaussian's partials are
// then contiguous for the chain-rule kernel, which sums them in tile order. No global atomics for the
// default tile size 16 (larger tiles span several CTAs and add atomically into zeroed partials).
//
// Compiled with -fmad=false so the per-pixel expressions round exactly like the reference's.

#include "kernels.h"

#include <atomic>

namespace u3dg {

namespace {

__device__ __forceinline__ float rasterExp(float x) { return expf(x); }

// Warp pixel block of 8x4 inside a PB x PB CTA block.
template <int PB>
struct WarpBlock {
    int px, py;           // this thread's pixel
    float x0, x1, y0, y1; // the warp's pixel rectangle (inclusive)
    __device__ explicit WarpBlock(int warp, int lane)
    {
        constexpr int WX = PB / 8;
        const int wx0 = int(blockIdx.x) * PB + (warp % WX) * 8, wy0 = int(blockIdx.y) * PB + (warp / WX) * 4;
        px = wx0 + (lane & 7);
        py = wy0 + (lane >> 3);
        x0 = float(wx0);
        x1 = float(wx0 + 7);
        y0 = float(wy0);
        y1 = float(wy0 + 3);
    }
};

// Does a contributing box (mx, my, ex, ey) meet warp w's pixel block?
template <int PB>
__device__ __forceinline__ bool meets(const float4 &p, int w)
{
    constexpr int WX = PB / 8;
    const float x0 = float(int(blockIdx.x) * PB + (w % WX) * 8), y0 = float(int(blockIdx.y) * PB + (w / WX) * 4);
    return !(p.x + p.z < x0 || p.x - p.z > x0 + 7.0f || p.y + p.w < y0 || p.y - p.w > y0 + 3.0f);
}

template <int PB>
__device__ __forceinline__ int tileOf(const RasterArgs &a)
{
    return (int(blockIdx.y) * PB / a.tileSize) * a.tilesX + int(blockIdx.x) * PB / a.tileSize;
}

// Stages batch entry `slot` (if valid) and builds the per-warp masks: after the call,
// mask[w][k] bit b says batch entry 32k + b meets warp w's pixel block.
template <int PB>
__device__ __forceinline__ void stage(const float4 *rec, const int *list, int idx, bool valid, int slot, float4 *sP,
                                      float4 *sQ, float4 *sR, uint32_t (*mask)[PB * PB / 32])
{
    constexpr int NW = PB * PB / 32;
    float4 p = make_float4(0.0f, 0.0f, -1.0f, -1.0f);
    if (valid) {
        const float4 *r = rec + size_t(list[idx]) * 3;
        p = r[0];
        sP[slot] = p;
        sQ[slot] = r[1];
        sR[slot] = r[2];
    }
    const int warp = slot >> 5, lane = slot & 31;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const uint32_t bits = __ballot_sync(0xffffffffu, valid && meets<PB>(p, w));
        if (lane == 0)
            mask[w][warp] = bits;
    }
}

template <int PB>
__global__ void __launch_bounds__(PB *PB) compositeForwardKernel(RasterArgs a, float *rgb, float *finalT, int *nContrib)
{
    constexpr int NT = PB * PB, NW = NT / 32;
    __shared__ float4 sP[NT]; // mx, my, ex, ey
    __shared__ float4 sQ[NT]; // A, B, C, alpha
    __shared__ float4 sR[NT]; // r, g, b, depth
    __shared__ uint32_t mask[NW][NW];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const WarpBlock<PB> wb(warp, lane);
    const int tile = tileOf<PB>(a);
    const int start = a.tileOffsets[tile], end = a.tileOffsets[tile + 1];
    const bool inside = wb.px < a.width && wb.py < a.height;
    bool done = !inside;
    float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
    int last = 0;
    const float fx = float(wb.px), fy = float(wb.py);
    const float minA = a.minAlpha, minT = a.minTransmittance;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    for (int b0 = start; b0 < end; b0 += NT) {
        if (__syncthreads_count(done) == NT)
            break;
        stage<PB>(rec, a.list, b0 + tid, b0 + tid < end, tid, sP, sQ, sR, mask);
        __syncthreads();
        if (!done) {
            for (int k = 0; k < NW && !done; ++k) {
                uint32_t bits = mask[warp][k];
                while (bits) {
                    const int j = 32 * k + __ffs(bits) - 1;
                    bits &= bits - 1;
                    const float4 P = sP[j], Q = sQ[j];
                    const float dx = P.x - fx, dy = P.y - fy;
                    const float power = -0.5f * (Q.x * dx * dx + Q.z * dy * dy) - Q.y * dx * dy;
                    if (power > 0.0f)
                        continue;
                    const float raw = Q.w * rasterExp(power);
                    const float al = (raw < kMaxAlpha) ? raw : kMaxAlpha;
                    if (al < minA)
                        continue;
                    const float nextT = T * (1.0f - al);
                    if (nextT < minT) {
                        done = true;
                        break;
                    }
                    const float w = al * T;
                    const float4 R = sR[j];
                    cr += R.x * w;
                    cg += R.y * w;
                    cb += R.z * w;
                    T = nextT;
                    last = b0 - start + j + 1;
                }
            }
        }
    }
    if (inside) {
        const size_t pix = size_t(wb.py) * a.width + wb.px;
        rgb[pix * 3] = cr + T * a.bg[0];
        rgb[pix * 3 + 1] = cg + T * a.bg[1];
        rgb[pix * 3 + 2] = cb + T * a.bg[2];
        finalT[pix] = T;
        nContrib[pix] = last;
    }
}

// Sum of c[0..8] over the warp. Values 0..7 by reduce-scatter: after the xor-16/8/4 exchanges lane l
// holds value 4*b4 + 2*b3 + b2 (bits of l) summed over the 8 lanes that share bits 4..2, then xor-2/1
// finish the sum; value 8 by a butterfly. Returns, in lane 4*v (v = 0..7), value v and, in every
// lane, value 8 (as *v8).
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

template <int PB>
__global__ void __launch_bounds__(PB *PB) compositeBackwardKernel(RasterArgs a, const float *dLdRgb,
                                                                   const float *finalTIn, const int *nContribIn,
                                                                   float *partial, int useAtomics)
{
    constexpr int NT = PB * PB, NW = NT / 32;
    __shared__ float4 sP[NT];
    __shared__ float4 sQ[NT];
    __shared__ float4 sR[NT];
    __shared__ uint32_t mask[NW][NW];
    __shared__ int sMax;
    // Per-warp sums of every batch entry, added over the warps in warp order after the batch, so the
    // result does not depend on warp scheduling (dynamic shared memory: NW * NT * 9 floats).
    extern __shared__ float sWarp[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const WarpBlock<PB> wb(warp, lane);
    const int tile = tileOf<PB>(a);
    const int start = a.tileOffsets[tile], end = a.tileOffsets[tile + 1];
    const bool inside = wb.px < a.width && wb.py < a.height;
    const size_t pix = inside ? size_t(wb.py) * a.width + wb.px : 0;
    const int nC = inside ? nContribIn[pix] : 0;
    const float fT = inside ? finalTIn[pix] : 0.0f;
    const float d0 = inside ? dLdRgb[pix * 3] : 0.0f, d1 = inside ? dLdRgb[pix * 3 + 1] : 0.0f,
                d2 = inside ? dLdRgb[pix * 3 + 2] : 0.0f;
    const float bgDot = a.bg[0] * d0 + a.bg[1] * d1 + a.bg[2] * d2;
    const float fx = float(wb.px), fy = float(wb.py);
    const float minA = a.minAlpha;
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    const int vIdx = (lane >> 2) & 7; // value this lane holds after warpReduce9 (lanes 4v)
    float T = fT;
    float acc0 = 0, acc1 = 0, acc2 = 0, lc0 = 0, lc1 = 0, lc2 = 0, lastAlpha = 0;
    if (tid == 0)
        sMax = 0;
    __syncthreads();
    if (nC > 0)
        atomicMax(&sMax, nC);
    __syncthreads();
    const int jmax = sMax;
    // List entries behind every pixel's last contributor get no gradient (the reference's per-tile
    // accumulators start at zero); their partials must still be written, as the chain-rule kernel
    // sums every intersection of a Gaussian.
    if (!useAtomics)
        for (int j = jmax + tid; j < end - start; j += NT) {
            float *dst = partial + size_t(a.listEmit[start + j]) * kG2d;
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                dst[k] = 0.0f;
        }
    for (int bEnd = jmax; bEnd > 0; bEnd -= NT) {
        const int bStart = max(0, bEnd - NT), cnt = bEnd - bStart;
        __syncthreads();
        stage<PB>(rec, a.list, start + bStart + tid, tid < cnt, tid, sP, sQ, sR, mask);
        {
            float4 *z = reinterpret_cast<float4 *>(sWarp);
            for (int k = tid; k < NW * NT * kG2d / 4; k += NT)
                z[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        float *myWarp = sWarp + size_t(warp) * NT * kG2d;
        __syncthreads();
        for (int k = NW - 1; k >= 0; --k) {
            uint32_t bits = mask[warp][k];
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
                if (j < nC) {
                    const float4 P = sP[jj], Q = sQ[jj];
                    const float dx = P.x - fx, dy = P.y - fy;
                    const float power = -0.5f * (Q.x * dx * dx + Q.z * dy * dy) - Q.y * dx * dy;
                    if (!(power > 0.0f)) {
                        const float G = rasterExp(power);
                        const float raw = Q.w * G;
                        const float al = (raw < kMaxAlpha) ? raw : kMaxAlpha;
                        if (!(al < minA)) {
                            const float4 R = sR[jj];
                            act = true;
                            T = T / (1.0f - al);
                            const float w = al * T;
                            float dAl = 0.0f;
                            acc0 = lastAlpha * lc0 + (1.0f - lastAlpha) * acc0;
                            lc0 = R.x;
                            dAl += (R.x - acc0) * d0;
                            c[5] = w * d0;
                            acc1 = lastAlpha * lc1 + (1.0f - lastAlpha) * acc1;
                            lc1 = R.y;
                            dAl += (R.y - acc1) * d1;
                            c[6] = w * d1;
                            acc2 = lastAlpha * lc2 + (1.0f - lastAlpha) * acc2;
                            lc2 = R.z;
                            dAl += (R.z - acc2) * d2;
                            c[7] = w * d2;
                            dAl *= T;
                            lastAlpha = al;
                            dAl += -fT / (1.0f - al) * bgDot;
                            if (!(raw > kMaxAlpha)) {
                                c[8] = G * dAl;
                                const float dPow = Q.w * dAl * G;
                                c[0] = dPow * -(Q.x * dx + Q.y * dy);
                                c[1] = dPow * -(Q.z * dy + Q.y * dx);
                                c[2] = dPow * -0.5f * dx * dx;
                                c[3] = dPow * -dx * dy;
                                c[4] = dPow * -0.5f * dy * dy;
                            }
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
        if (tid < cnt) {
            float s[kG2d];
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                s[k] = sWarp[tid * kG2d + k];
            for (int w = 1; w < NW; ++w)
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    s[k] += sWarp[(size_t(w) * NT + tid) * kG2d + k];
            float *dst = partial + size_t(a.listEmit[start + bStart + tid]) * kG2d;
            if (useAtomics) {
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    atomicAdd(dst + k, s[k]);
            } else {
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    dst[k] = s[k];
            }
        }
    }
}

} // namespace

void launchCompositeForward(const RasterArgs &a, float *rgb, float *finalT, int *nContrib, cudaStream_t s)
{
    if (a.tileSize <= 8) {
        dim3 g((a.width + 7) / 8, (a.height + 7) / 8);
        { compositeForwardKernel<8><<<g, 64, 0, s>>>(a, rgb, finalT, nContrib); countLaunch(); }
    } else {
        dim3 g((a.width + 15) / 16, (a.height + 15) / 16);
        { compositeForwardKernel<16><<<g, 256, 0, s>>>(a, rgb, finalT, nContrib); countLaunch(); }
    }
}

void launchCompositeBackward(const RasterArgs &a, const float *dLdRgb, const float *finalT, const int *nContrib,
                             float *partial, cudaStream_t s)
{
    if (a.tileSize <= 8) {
        dim3 g((a.width + 7) / 8, (a.height + 7) / 8);
        const size_t smem = size_t(2) * 64 * kG2d * sizeof(float);
        { compositeBackwardKernel<8><<<g, 64, smem, s>>>(a, dLdRgb, finalT, nContrib, partial, 0); countLaunch(); }
    } else {
        dim3 g((a.width + 15) / 16, (a.height + 15) / 16);
        const size_t smem = size_t(8) * 256 * kG2d * sizeof(float);
        // Opt in to more than 48 KB of dynamic shared memory, once per device.
        static std::atomic<unsigned long long> optedIn{0};
        int dev = 0;
        cudaGetDevice(&dev);
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(optedIn.load() & bit)) {
            const cudaError_t e = cudaFuncSetAttribute(compositeBackwardKernel<16>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (e != cudaSuccess)
                return; // the launch below is skipped; the caller sees the error via cudaGetLastError
            optedIn.fetch_or(bit);
        }
        { compositeBackwardKernel<16><<<g, 256, smem, s>>>(a, dLdRgb, finalT, nContrib, partial, a.tileSize > 16 ? 1 : 0); countLaunch(); }
    }
}

} // namespace u3dg
