// raster.cu - tile compositing, forward and backward (Rasterizer.cpp:281-329 and 353-427).
//
// One CTA per 16x16 pixel block (8x8 when the tile size is 8), one thread per pixel. The tile's
// depth-sorted list is walked in batches of one record per thread, staged in shared memory; every
// thread then evaluates the batch for its pixel in list order. Forward stops a CTA once every pixel
// has terminated (transmittance cut-off), counted with __syncthreads_count.
//
// Backward walks the same lists back to front from each pixel's contributor count, with the
// reference's per-pixel recurrence. The 9 per-Gaussian 2D gradients of every list entry are summed
// over the tile's pixels inside the CTA (warp butterfly, then shared-memory adds of the warp sums)
// and written once per (tile, Gaussian) - no global atomics for the default tile size 16. The
// per-Gaussian sum over tiles happens later, in tile order, in the chain-rule kernel.
//
// Compiled with -fmad=false so the per-pixel expressions round exactly like the reference's.

#include "kernels.h"

namespace u3dg {

namespace {

__device__ __forceinline__ float rasterExp(float x) { return expf(x); }

template <int PB>
__global__ void __launch_bounds__(PB *PB) compositeForwardKernel(RasterArgs a, float *rgb, float *finalT, int *nContrib)
{
    constexpr int NT = PB * PB;
    __shared__ float4 sA[NT]; // mx, my, A, B
    __shared__ float4 sB[NT]; // C, alpha, r, g
    __shared__ float sC[NT];  // b
    const int tid = threadIdx.x;
    const int px = blockIdx.x * PB + tid % PB, py = blockIdx.y * PB + tid / PB;
    const int tile = (int(blockIdx.y) * PB / a.tileSize) * a.tilesX + int(blockIdx.x) * PB / a.tileSize;
    const int start = a.tileOffsets[tile], end = a.tileOffsets[tile + 1];
    const bool inside = px < a.width && py < a.height;
    bool done = !inside;
    float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
    int last = 0;
    const float fx = float(px), fy = float(py);
    const float minA = a.minAlpha, minT = a.minTransmittance;
    for (int b0 = start; b0 < end; b0 += NT) {
        if (__syncthreads_count(done) == NT)
            break;
        const int idx = b0 + tid;
        if (idx < end) {
            const float4 *r = reinterpret_cast<const float4 *>(a.rec + a.list[idx]);
            const float4 r0 = r[0], r1 = r[1], r2 = r[2];
            sA[tid] = make_float4(r0.x, r0.y, r0.z, r0.w);
            sB[tid] = make_float4(r1.x, r1.y, r1.z, r1.w);
            sC[tid] = r2.x;
        }
        __syncthreads();
        const int cnt = min(NT, end - b0);
        if (!done) {
            for (int j = 0; j < cnt; ++j) {
                const float4 A = sA[j], B = sB[j];
                const float dx = A.x - fx, dy = A.y - fy;
                const float power = -0.5f * (A.z * dx * dx + B.x * dy * dy) - A.w * dx * dy;
                if (power > 0.0f)
                    continue;
                const float raw = B.y * rasterExp(power);
                const float al = (raw < kMaxAlpha) ? raw : kMaxAlpha;
                if (al < minA)
                    continue;
                const float nextT = T * (1.0f - al);
                if (nextT < minT) {
                    done = true;
                    break;
                }
                const float w = al * T;
                cr += B.z * w;
                cg += B.w * w;
                cb += sC[j] * w;
                T = nextT;
                last = b0 - start + j + 1;
            }
        }
    }
    if (inside) {
        const size_t pix = size_t(py) * a.width + px;
        rgb[pix * 3] = cr + T * a.bg[0];
        rgb[pix * 3 + 1] = cg + T * a.bg[1];
        rgb[pix * 3 + 2] = cb + T * a.bg[2];
        finalT[pix] = T;
        nContrib[pix] = last;
    }
}

template <int PB>
__global__ void __launch_bounds__(PB *PB) compositeBackwardKernel(RasterArgs a, const float *dLdRgb,
                                                                   const float *finalTIn, const int *nContribIn,
                                                                   float *partial, int useAtomics)
{
    constexpr int NT = PB * PB;
    __shared__ float4 sA[NT];
    __shared__ float4 sB[NT];
    __shared__ float sC[NT];
    __shared__ float sAcc[NT][kG2d];
    __shared__ int sMax;
    const int tid = threadIdx.x, lane = tid & 31;
    const int px = blockIdx.x * PB + tid % PB, py = blockIdx.y * PB + tid / PB;
    const int tile = (int(blockIdx.y) * PB / a.tileSize) * a.tilesX + int(blockIdx.x) * PB / a.tileSize;
    const int start = a.tileOffsets[tile];
    const bool inside = px < a.width && py < a.height;
    const size_t pix = inside ? size_t(py) * a.width + px : 0;
    const int nC = inside ? nContribIn[pix] : 0;
    const float fT = inside ? finalTIn[pix] : 0.0f;
    const float d0 = inside ? dLdRgb[pix * 3] : 0.0f, d1 = inside ? dLdRgb[pix * 3 + 1] : 0.0f,
                d2 = inside ? dLdRgb[pix * 3 + 2] : 0.0f;
    const float bgDot = a.bg[0] * d0 + a.bg[1] * d1 + a.bg[2] * d2;
    const float fx = float(px), fy = float(py);
    const float minA = a.minAlpha;
    float T = fT;
    float acc0 = 0, acc1 = 0, acc2 = 0, lc0 = 0, lc1 = 0, lc2 = 0, lastAlpha = 0;
    if (tid == 0)
        sMax = 0;
    __syncthreads();
    if (nC > 0)
        atomicMax(&sMax, nC);
    __syncthreads();
    const int jmax = sMax;
    for (int bEnd = jmax; bEnd > 0; bEnd -= NT) {
        const int bStart = max(0, bEnd - NT), cnt = bEnd - bStart;
        __syncthreads();
        if (tid < cnt) {
            const float4 *r = reinterpret_cast<const float4 *>(a.rec + a.list[start + bStart + tid]);
            const float4 r0 = r[0], r1 = r[1], r2 = r[2];
            sA[tid] = r0;
            sB[tid] = r1;
            sC[tid] = r2.x;
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                sAcc[tid][k] = 0.0f;
        }
        __syncthreads();
        for (int jj = cnt - 1; jj >= 0; --jj) {
            const int j = bStart + jj;
            float c[kG2d];
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                c[k] = 0.0f;
            bool act = false;
            if (j < nC) {
                const float4 A = sA[jj], B = sB[jj];
                const float colB = sC[jj];
                const float dx = A.x - fx, dy = A.y - fy;
                const float power = -0.5f * (A.z * dx * dx + B.x * dy * dy) - A.w * dx * dy;
                if (!(power > 0.0f)) {
                    const float G = rasterExp(power);
                    const float raw = B.y * G;
                    const float al = (raw < kMaxAlpha) ? raw : kMaxAlpha;
                    if (!(al < minA)) {
                        act = true;
                        T = T / (1.0f - al);
                        const float w = al * T;
                        float dAl = 0.0f;
                        acc0 = lastAlpha * lc0 + (1.0f - lastAlpha) * acc0;
                        lc0 = B.z;
                        dAl += (B.z - acc0) * d0;
                        c[5] = w * d0;
                        acc1 = lastAlpha * lc1 + (1.0f - lastAlpha) * acc1;
                        lc1 = B.w;
                        dAl += (B.w - acc1) * d1;
                        c[6] = w * d1;
                        acc2 = lastAlpha * lc2 + (1.0f - lastAlpha) * acc2;
                        lc2 = colB;
                        dAl += (colB - acc2) * d2;
                        c[7] = w * d2;
                        dAl *= T;
                        lastAlpha = al;
                        dAl += -fT / (1.0f - al) * bgDot;
                        if (!(raw > kMaxAlpha)) {
                            c[8] = G * dAl;
                            const float dPow = B.y * dAl * G;
                            c[0] = dPow * -(A.z * dx + A.w * dy);
                            c[1] = dPow * -(B.x * dy + A.w * dx);
                            c[2] = dPow * -0.5f * dx * dx;
                            c[3] = dPow * -dx * dy;
                            c[4] = dPow * -0.5f * dy * dy;
                        }
                    }
                }
            }
            if (__any_sync(0xffffffffu, act)) {
#pragma unroll
                for (int k = 0; k < kG2d; ++k) {
                    float v = c[k];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1)
                        v += __shfl_xor_sync(0xffffffffu, v, o);
                    c[k] = v;
                }
                float mine = 0.0f;
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    if (lane == k)
                        mine = c[k];
                if (lane < kG2d)
                    atomicAdd(&sAcc[jj][lane], mine);
            }
        }
        __syncthreads();
        if (tid < cnt) {
            float *dst = partial + size_t(start + bStart + tid) * kG2d;
            if (useAtomics) {
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    atomicAdd(dst + k, sAcc[tid][k]);
            } else {
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    dst[k] = sAcc[tid][k];
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
        { compositeBackwardKernel<8><<<g, 64, 0, s>>>(a, dLdRgb, finalT, nContrib, partial, 0); countLaunch(); }
    } else {
        dim3 g((a.width + 15) / 16, (a.height + 15) / 16);
        { compositeBackwardKernel<16><<<g, 256, 0, s>>>(a, dLdRgb, finalT, nContrib, partial, a.tileSize > 16 ? 1 : 0); countLaunch(); }
    }
}

} // namespace u3dg
