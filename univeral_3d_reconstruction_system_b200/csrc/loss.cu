// loss.cu - (1 - lambda) L1 + lambda (1 - SSIM) and its gradient (photometricLoss, Loss.cpp:47-184).
//
// The reference runs four separable passes over (channel, row) pairs with full-image scratch maps.
// Here two tiled kernels do the same arithmetic with the blurs staged in shared memory, one CTA per
// 32x16 tile and colour channel (the three channels in parallel CTAs: the kernels are latency-bound,
// and a CTA per tile walking the channels in turn was 11 % slower):
//   lossForwardKernel : L1 term + horizontal blur of x, y, x^2, y^2, xy + vertical blur + SSIM and
//                       its three per-pixel partials (passes 1 and 2), block partial sums in double;
//   lossBackwardKernel: horizontal + vertical blur of the partials and the chain rule into
//                       dL/drender (passes 3 and 4; the Gaussian blur is self-adjoint).
// Zero padding is reproduced by loading zeros outside the image: the reference skips out-of-image
// taps, and adding w * 0 to the running sums leaves every intermediate value unchanged, so each
// per-pixel value keeps the reference's rounding (the file is compiled with -fmad=false). The
// block sums are reduced in a fixed order, so the loss is deterministic.

#include "kernels.h"

#include <cmath>

namespace u3dg {

namespace {

constexpr int kR = 5;                    // 11x11 window (Loss.cpp:11)
constexpr int kTW = 32, kTH = 16;        // output tile
constexpr int kIW = kTW + 2 * kR, kIH = kTH + 2 * kR;
constexpr int kThreads = 256;

// The 11 blur weights, passed to the loss kernels by value: kernel parameters sit in the constant
// bank like a __constant__ array, but need no upload into each device context (no synchronous copy
// before the first launch, nothing to redo after a context is recreated, nothing shared between host
// threads), and a captured graph keeps them with the launch.
struct SsimWindow {
    float w[2 * kR + 1];
};

// The window exactly as Loss.cpp:15-27 builds it (host float arithmetic with glibc expf).
struct HostWindow : SsimWindow {
    HostWindow()
    {
        float sum = 0;
        for (int k = -kR; k <= kR; ++k) {
            w[k + kR] = std::exp(-float(k * k) / (2.0f * 1.5f * 1.5f));
            sum += w[k + kR];
        }
        for (float &v : w)
            v /= sum;
    }
};

__device__ __forceinline__ double blockSumDouble(double v)
{
    __shared__ double warpSums[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
        warpSums[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w)
            t += warpSums[w];
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kThreads) lossForwardKernel(const float *render, const float *targetF,
                                                              const uint8_t *targetU8, int W, int H, float lambda,
                                                              float *grad, float *abc, double *blockSums,
                                                              const StepDesc *desc, const SsimWindow cWin)
{
    pdlEntry();
    if (desc)
        targetU8 = desc->target;
    __shared__ float sx[kIH][kIW], sy[kIH][kIW];
    __shared__ float hm[5][kIH][kTW];
    const int x0 = blockIdx.x * kTW, y0 = blockIdx.y * kTH;
    const size_t P = size_t(W) * H;
    const float invCount = 1.0f / float(P * 3);
    const float l1Scale = (1.0f - lambda) * invCount;
    const float dLds = -lambda * invCount;
    const float kC1 = 0.01f * 0.01f, kC2 = 0.03f * 0.03f;
    const float inv255 = 1.0f / 255.0f;
    double l1 = 0.0, ssim = 0.0, sq = 0.0;
    {
        const int c = blockIdx.z; // one colour channel per block
        for (int k = threadIdx.x; k < kIW * kIH; k += kThreads) {
            const int ix = k % kIW, iy = k / kIW;
            const int gx = x0 + ix - kR, gy = y0 + iy - kR;
            float a = 0.0f, b = 0.0f;
            if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
                const size_t idx = (size_t(gy) * W + gx) * 3 + c;
                a = render[idx];
                b = targetU8 ? float(targetU8[idx]) * inv255 : targetF[idx];
            }
            sx[iy][ix] = a;
            sy[iy][ix] = b;
        }
        __syncthreads();
        // L1 term for this tile's pixels (Loss.cpp:68-74).
        for (int k = threadIdx.x; k < kTW * kTH; k += kThreads) {
            const int ox = k % kTW, oy = k / kTW;
            const int gx = x0 + ox, gy = y0 + oy;
            if (gx < W && gy < H) {
                const float d = sx[oy + kR][ox + kR] - sy[oy + kR][ox + kR];
                l1 += fabs(double(d));
                const double dd = double(sx[oy + kR][ox + kR]) - double(sy[oy + kR][ox + kR]);
                sq += dd * dd;
                grad[(size_t(gy) * W + gx) * 3 + c] = l1Scale * (d > 0 ? 1.0f : (d < 0 ? -1.0f : 0.0f));
            }
        }
        if (lambda > 0.0f) {
            // Horizontal blur of x, y, x^2, y^2, xy (Loss.cpp:77-94).
            for (int k = threadIdx.x; k < kTW * kIH; k += kThreads) {
                const int ox = k % kTW, iy = k / kTW;
                float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
#pragma unroll
                for (int t = 0; t <= 2 * kR; ++t) {
                    const float a = sx[iy][ox + t], b = sy[iy][ox + t], w = cWin.w[t];
                    s0 += w * a;
                    s1 += w * b;
                    s2 += w * a * a;
                    s3 += w * b * b;
                    s4 += w * a * b;
                }
                hm[0][iy][ox] = s0;
                hm[1][iy][ox] = s1;
                hm[2][iy][ox] = s2;
                hm[3][iy][ox] = s3;
                hm[4][iy][ox] = s4;
            }
            __syncthreads();
            // Vertical blur, SSIM and its partials (Loss.cpp:113-137).
            for (int k = threadIdx.x; k < kTW * kTH; k += kThreads) {
                const int ox = k % kTW, oy = k / kTW;
                const int gx = x0 + ox, gy = y0 + oy;
                if (gx >= W || gy >= H)
                    continue;
                float m[5] = {0, 0, 0, 0, 0};
#pragma unroll
                for (int t = 0; t <= 2 * kR; ++t) {
                    const float w = cWin.w[t];
#pragma unroll
                    for (int j = 0; j < 5; ++j)
                        m[j] += w * hm[j][oy + t][ox];
                }
                const float mx = m[0], my = m[1];
                const float vx = m[2] - mx * mx, vy = m[3] - my * my, vxy = m[4] - mx * my;
                const float a1 = 2 * mx * my + kC1, a2 = 2 * vxy + kC2;
                const float b1 = mx * mx + my * my + kC1, b2 = vx + vy + kC2;
                const float v = (a1 * a2) / (b1 * b2);
                ssim += double(v);
                const float dmu = (2 * my * a2 - 2 * my * a1) / (b1 * b2) - v * (2 * mx / b1 - 2 * mx / b2);
                const size_t o = size_t(c) * P + size_t(gy) * W + gx;
                abc[o] = dLds * dmu;
                abc[3 * P + o] = dLds * (-v / b2);
                abc[6 * P + o] = dLds * (2 * a1 / (b1 * b2));
            }
        }
        __syncthreads();
    }
    const double t0 = blockSumDouble(l1);
    const double t1 = blockSumDouble(ssim);
    const double t2 = blockSumDouble(sq);
    if (threadIdx.x == 0) {
        const int b = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        blockSums[3 * b] = t0;
        blockSums[3 * b + 1] = t1;
        blockSums[3 * b + 2] = t2;
    }
}

__global__ void __launch_bounds__(kThreads) lossBackwardKernel(const float *render, const float *targetF,
                                                               const uint8_t *targetU8, int W, int H, const float *abc,
                                                               float *grad, const StepDesc *desc,
                                                               const SsimWindow cWin)
{
    pdlEntry();
    if (desc)
        targetU8 = desc->target;
    __shared__ float sm[3][kIH][kIW];
    __shared__ float hm[3][kIH][kTW];
    const int x0 = blockIdx.x * kTW, y0 = blockIdx.y * kTH;
    const size_t P = size_t(W) * H;
    const float inv255 = 1.0f / 255.0f;
    {
        const int c = blockIdx.z; // one colour channel per block
        for (int k = threadIdx.x; k < kIW * kIH; k += kThreads) {
            const int ix = k % kIW, iy = k / kIW;
            const int gx = x0 + ix - kR, gy = y0 + iy - kR;
            const bool in = gx >= 0 && gx < W && gy >= 0 && gy < H;
            const size_t o = size_t(c) * P + (in ? size_t(gy) * W + gx : 0);
            sm[0][iy][ix] = in ? abc[o] : 0.0f;
            sm[1][iy][ix] = in ? abc[3 * P + o] : 0.0f;
            sm[2][iy][ix] = in ? abc[6 * P + o] : 0.0f;
        }
        __syncthreads();
        // Pass 3: horizontal blur of the partials (Loss.cpp:142-157).
        for (int k = threadIdx.x; k < kTW * kIH; k += kThreads) {
            const int ox = k % kTW, iy = k / kTW;
            float a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
            for (int t = 0; t <= 2 * kR; ++t) {
                const float w = cWin.w[t];
                a0 += w * sm[0][iy][ox + t];
                a1 += w * sm[1][iy][ox + t];
                a2 += w * sm[2][iy][ox + t];
            }
            hm[0][iy][ox] = a0;
            hm[1][iy][ox] = a1;
            hm[2][iy][ox] = a2;
        }
        __syncthreads();
        // Pass 4: vertical blur + chain rule (Loss.cpp:160-177).
        for (int k = threadIdx.x; k < kTW * kTH; k += kThreads) {
            const int ox = k % kTW, oy = k / kTW;
            const int gx = x0 + ox, gy = y0 + oy;
            if (gx >= W || gy >= H)
                continue;
            float g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
            for (int t = 0; t <= 2 * kR; ++t) {
                const float w = cWin.w[t];
                g0 += w * hm[0][oy + t][ox];
                g1 += w * hm[1][oy + t][ox];
                g2 += w * hm[2][oy + t][ox];
            }
            const size_t idx = (size_t(gy) * W + gx) * 3 + c;
            const float tg = targetU8 ? float(targetU8[idx]) * inv255 : targetF[idx];
            grad[idx] += g0 + 2.0f * render[idx] * g1 + tg * g2;
        }
        __syncthreads();
    }
}

// Single block: fixed-order sum of the block partials, LossValue, PSNR and the EMA stats.
constexpr int kFinalThreads = 1024;

__global__ void __launch_bounds__(kFinalThreads) lossFinalizeKernel(const double *blockSums, int blocks, int W, int H,
                                                               float lambda, DevStats *stats, int iteration,
                                                               const BinCounts *counts, float *out3, float *psnrOut,
                                                               const StepDesc *desc)
{
    pdlEntry();
    if (desc)
        iteration = desc->iteration + 1;
    if (counts != nullptr && counts->abortIter >= 0)
        stats = nullptr; // an aborted step leaves the statistics alone (it is replayed)
    // The three sums over the loss blocks in a fixed order: strided per thread, a butterfly per warp,
    // then the warps' sums in warp order (one barrier for all three).
    __shared__ double warpSums[kFinalThreads / 32][3];
    double s0 = 0, s1 = 0, s2 = 0;
    for (int b = threadIdx.x; b < blocks; b += kFinalThreads) {
        s0 += blockSums[3 * b];
        s1 += blockSums[3 * b + 1];
        s2 += blockSums[3 * b + 2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        warpSums[threadIdx.x >> 5][0] = s0;
        warpSums[threadIdx.x >> 5][1] = s1;
        warpSums[threadIdx.x >> 5][2] = s2;
    }
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    s0 = s1 = s2 = 0.0;
    for (int w = 0; w < kFinalThreads / 32; ++w) {
        s0 += warpSums[w][0];
        s1 += warpSums[w][1];
        s2 += warpSums[w][2];
    }
    const size_t P = size_t(W) * H;
    const float invCount = 1.0f / float(P * 3);
    const float l1 = float(s0 * invCount);
    float ssim = 0.0f, total = l1;
    if (lambda > 0.0f) {
        ssim = float(s1 * invCount);
        total = (1.0f - lambda) * l1 + lambda * (1.0f - ssim);
    }
    double mse = s2 / double(P * 3 > 0 ? P * 3 : 1);
    const float psnr = mse <= 1e-12 ? 99.0f : float(-10.0 * log10(mse));
    if (out3) {
        out3[0] = total;
        out3[1] = l1;
        out3[2] = ssim;
    }
    if (psnrOut)
        *psnrOut = psnr;
    if (stats) {
        const float k = stats->iteration == 0 ? 1.0f : 0.05f;
        stats->loss += k * (total - stats->loss);
        stats->psnr += k * (psnr - stats->psnr);
        stats->iteration = iteration;
        stats->lastLoss = total;
        stats->lastL1 = l1;
        stats->lastSsim = ssim;
        stats->lastPsnr = psnr;
    }
}

// Sum of squared differences in double, one partial per block, then a fixed-order final sum.
__global__ void __launch_bounds__(kThreads) sqDiffKernel(const float *a, const float *bF, const uint8_t *bU8,
                                                         size_t count, double *partial)
{
    const float inv255 = 1.0f / 255.0f;
    double s = 0.0;
    for (size_t k = size_t(blockIdx.x) * kThreads + threadIdx.x; k < count; k += size_t(gridDim.x) * kThreads) {
        const float b = bU8 ? float(bU8[k]) * inv255 : bF[k];
        const double d = double(a[k]) - double(b);
        s += d * d;
    }
    s = blockSumDouble(s);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) sumPartialsKernel(const double *partial, int n, double *out)
{
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += kThreads)
        s += partial[k];
    s = blockSumDouble(s);
    if (threadIdx.x == 0)
        *out = s;
}

__global__ void quantizeKernel(const float *rgb, size_t count, uint8_t *out)
{
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count)
        return;
    const float v = rgb[k];
    const float c = (v < 0.0f) ? 0.0f : v;            // std::max(0.0f, v)
    const float y = ((1.0f < c) ? 1.0f : c) * 255.0f; // std::min(1.0f, c) * 255.0f
    int r = int(y);                                   // y >= 0: truncation, then round half up = lround
    if (y - float(r) >= 0.5f)
        ++r;
    out[k] = uint8_t(r);
}

const SsimWindow &window()
{
    static const HostWindow w; // thread-safe one-time initialisation
    return w;
}

constexpr int kSqBlocks = 296; // 2 x 148 SMs

} // namespace

int lossBlocks(int width, int height) { return 3 * ((width + kTW - 1) / kTW) * ((height + kTH - 1) / kTH); }

void launchLoss(const float *render, const float *targetF, const uint8_t *targetU8, int width, int height, float lambda,
                float *grad, const LossScratch &ls, cudaStream_t s, const StepDesc *desc)
{
    const SsimWindow &win = window();
    dim3 g((width + kTW - 1) / kTW, (height + kTH - 1) / kTH, 3);
    { launchPdl(lossForwardKernel, g, kThreads, 0, s, render, targetF, targetU8, width, height, lambda, grad, ls.abc,
                                             ls.blockSums, desc, win); countLaunch(); }
    if (lambda > 0.0f)
        { launchPdl(lossBackwardKernel, g, kThreads, 0, s, render, targetF, targetU8, width, height, ls.abc, grad, desc, win); countLaunch(); }
}

void launchLossFinalize(const LossScratch &ls, int width, int height, float lambda, DevStats *stats, int iteration,
                        const BinCounts *counts, float *out3, float *psnrOut, cudaStream_t s, const StepDesc *desc)
{
    { launchPdl(lossFinalizeKernel, 1, kFinalThreads, 0, s, ls.blockSums, ls.blocks, width, height, lambda, stats, iteration,
                                              counts, out3, psnrOut, desc); countLaunch(); }
}

void launchPsnrU8(const float *render, const uint8_t *target, size_t count, double *sumOut, cudaStream_t s)
{
    // sumOut must hold kSqBlocks + 1 doubles; the total lands in sumOut[kSqBlocks].
    { sqDiffKernel<<<kSqBlocks, kThreads, 0, s>>>(render, nullptr, target, count, sumOut); countLaunch(); }
    { sumPartialsKernel<<<1, kThreads, 0, s>>>(sumOut, kSqBlocks, sumOut + kSqBlocks); countLaunch(); }
}

void launchQuantize(const float *rgb, size_t count, uint8_t *out, cudaStream_t s)
{
    if (count)
        { quantizeKernel<<<unsigned((count + 255) / 256), 256, 0, s>>>(rgb, count, out); countLaunch(); }
}

void launchPsnrF(const float *a, const float *b, size_t count, double *sumOut, cudaStream_t s)
{
    { sqDiffKernel<<<kSqBlocks, kThreads, 0, s>>>(a, b, nullptr, count, sumOut); countLaunch(); }
    { sumPartialsKernel<<<1, kThreads, 0, s>>>(sumOut, kSqBlocks, sumOut + kSqBlocks); countLaunch(); }
}

} // namespace u3dg
