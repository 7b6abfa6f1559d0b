// loss.cu - (1 - lambda) L1 + lambda (1 - SSIM) and its gradient (photometricLoss, Loss.cpp:47-184).
//
// The reference runs four separable passes over (channel, row) pairs with full-image scratch maps.
// Here one tiled kernel (lossKernel) does all four passes for a 32x16 tile with the blurs staged in
// shared memory: L1 term, horizontal + vertical blur of x, y, x^2, y^2, xy, SSIM and its three
// per-pixel partials (passes 1 and 2) over the tile and a 5-pixel halo, then the blur of the partials
// and the chain rule into dL/drender (passes 3 and 4; the Gaussian blur is self-adjoint), with block
// partial sums in double.
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

// The whole loss of one 32x16 output tile and one channel at a time, in one kernel. The gradient of
// the D-SSIM term at a pixel needs the three SSIM partials (abc) of the 11x11 window around it, and
// each of those needs the blurred statistics of the window around that pixel: the tile stages its
// inputs with a 10-pixel halo, computes the statistics and the partials for the tile plus a 5-pixel
// halo, and blurs the partials back onto the tile. The halo partials are the ones the neighbouring
// tiles compute for their own pixels (same inputs, same operations in the same order), so every value
// is what the two-pass formulation of Loss.cpp:47-184 gives, without the partials' round trip through
// global memory. The L1 and SSIM sums of a block cover its own pixels only, in a fixed per-thread
// order.
constexpr int kH = 2 * kR;                    // input halo: 10 pixels
constexpr int kSW = kTW + 2 * kH, kSH = kTH + 2 * kH; // staged inputs: 52 x 36
constexpr int kAW = kTW + 2 * kR, kAH = kTH + 2 * kR; // statistics / partials region: 42 x 26

struct LossSmem {
    float x[kSH][kSW], y[kSH][kSW];   // render and target of one channel
    float hm[5][kSH][kAW];           // horizontal blurs of x, y, x^2, y^2, xy (then of the partials)
    float abc[3][kAH][kAW];          // SSIM partials over the tile and its 5-pixel halo
    float v[kTH][kTW];               // SSIM of the tile's pixels
};

__global__ void __launch_bounds__(kThreads) lossKernel(const float *render, const float *targetF,
                                                       const uint8_t *targetU8, int W, int H, float lambda,
                                                       float *grad, double *blockSums, const StepDesc *desc,
                                                       const SsimWindow cWin)
{
    if (desc)
        targetU8 = desc->target;
    extern __shared__ __align__(16) unsigned char lossSmemRaw[];
    LossSmem &sm = *reinterpret_cast<LossSmem *>(lossSmemRaw);
    float(*h2)[kAH][kTW] = reinterpret_cast<float(*)[kAH][kTW]>(&sm.hm[0][0][0]); // blurred partials
    const int x0 = blockIdx.x * kTW, y0 = blockIdx.y * kTH;
    const size_t P = size_t(W) * H;
    const float invCount = 1.0f / float(P * 3);
    const float l1Scale = (1.0f - lambda) * invCount;
    const float dLds = -lambda * invCount;
    const float kC1 = 0.01f * 0.01f, kC2 = 0.03f * 0.03f;
    const float inv255 = 1.0f / 255.0f;
    double l1 = 0.0, ssim = 0.0, sq = 0.0;
    constexpr int kPix = kTW * kTH / kThreads; // tile pixels per thread (2)
    for (int c = 0; c < 3; ++c) {
        for (int k = threadIdx.x; k < kSW * kSH; k += kThreads) {
            const int ix = k % kSW, iy = k / kSW;
            const int gx = x0 + ix - kH, gy = y0 + iy - kH;
            float a = 0.0f, b = 0.0f;
            if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
                const size_t idx = (size_t(gy) * W + gx) * 3 + c;
                a = render[idx];
                b = targetU8 ? float(targetU8[idx]) * inv255 : targetF[idx];
            }
            sm.x[iy][ix] = a;
            sm.y[iy][ix] = b;
        }
        __syncthreads();
        // L1 term for this tile's pixels (Loss.cpp:68-74).
        float l1grad[kPix];
#pragma unroll
        for (int r = 0; r < kPix; ++r) {
            const int k = threadIdx.x + r * kThreads;
            const int ox = k % kTW, oy = k / kTW;
            const int gx = x0 + ox, gy = y0 + oy;
            l1grad[r] = 0.0f;
            if (gx < W && gy < H) {
                const float d = sm.x[oy + kH][ox + kH] - sm.y[oy + kH][ox + kH];
                l1 += fabs(double(d));
                const double dd = double(sm.x[oy + kH][ox + kH]) - double(sm.y[oy + kH][ox + kH]);
                sq += dd * dd;
                l1grad[r] = l1Scale * (d > 0 ? 1.0f : (d < 0 ? -1.0f : 0.0f));
            }
        }
        if (lambda > 0.0f) {
            // Horizontal blur of x, y, x^2, y^2, xy (Loss.cpp:77-94) for every staged row, over the
            // columns of the tile and its 5-pixel halo.
            for (int k = threadIdx.x; k < kAW * kSH; k += kThreads) {
                const int ox = k % kAW, iy = k / kAW;
                float s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
#pragma unroll
                for (int t = 0; t <= 2 * kR; ++t) {
                    const float a = sm.x[iy][ox + t], b = sm.y[iy][ox + t], w = cWin.w[t];
                    s0 += w * a;
                    s1 += w * b;
                    s2 += w * a * a;
                    s3 += w * b * b;
                    s4 += w * a * b;
                }
                sm.hm[0][iy][ox] = s0;
                sm.hm[1][iy][ox] = s1;
                sm.hm[2][iy][ox] = s2;
                sm.hm[3][iy][ox] = s3;
                sm.hm[4][iy][ox] = s4;
            }
            __syncthreads();
            // Vertical blur, SSIM and its partials (Loss.cpp:113-137) over the tile and its halo;
            // partials outside the image are zero (the blur of pass 3 pads with zeros).
            for (int k = threadIdx.x; k < kAW * kAH; k += kThreads) {
                const int ox = k % kAW, oy = k / kAW;
                const int gx = x0 + ox - kR, gy = y0 + oy - kR;
                float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
                if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
                    float m[5] = {0, 0, 0, 0, 0};
#pragma unroll
                    for (int t = 0; t <= 2 * kR; ++t) {
                        const float w = cWin.w[t];
#pragma unroll
                        for (int j = 0; j < 5; ++j)
                            m[j] += w * sm.hm[j][oy + t][ox];
                    }
                    const float mx = m[0], my = m[1];
                    const float vx = m[2] - mx * mx, vy = m[3] - my * my, vxy = m[4] - mx * my;
                    const float A1 = 2 * mx * my + kC1, A2 = 2 * vxy + kC2;
                    const float B1 = mx * mx + my * my + kC1, B2 = vx + vy + kC2;
                    const float v = (A1 * A2) / (B1 * B2);
                    const float dmu = (2 * my * A2 - 2 * my * A1) / (B1 * B2) - v * (2 * mx / B1 - 2 * mx / B2);
                    a0 = dLds * dmu;
                    a1 = dLds * (-v / B2);
                    a2 = dLds * (2 * A1 / (B1 * B2));
                    if (ox >= kR && ox < kR + kTW && oy >= kR && oy < kR + kTH)
                        sm.v[oy - kR][ox - kR] = v;
                }
                sm.abc[0][oy][ox] = a0;
                sm.abc[1][oy][ox] = a1;
                sm.abc[2][oy][ox] = a2;
            }
            __syncthreads();
            // SSIM sum over the tile's own pixels, in the order each thread owns them.
#pragma unroll
            for (int r = 0; r < kPix; ++r) {
                const int k = threadIdx.x + r * kThreads;
                const int ox = k % kTW, oy = k / kTW;
                if (x0 + ox < W && y0 + oy < H)
                    ssim += double(sm.v[oy][ox]);
            }
            // Horizontal blur of the partials (pass 3, Loss.cpp:142-157), into the first maps' space.
            for (int k = threadIdx.x; k < kTW * kAH; k += kThreads) {
                const int ox = k % kTW, iy = k / kTW;
                float b0 = 0, b1 = 0, b2 = 0;
#pragma unroll
                for (int t = 0; t <= 2 * kR; ++t) {
                    const float w = cWin.w[t];
                    b0 += w * sm.abc[0][iy][ox + t];
                    b1 += w * sm.abc[1][iy][ox + t];
                    b2 += w * sm.abc[2][iy][ox + t];
                }
                h2[0][iy][ox] = b0;
                h2[1][iy][ox] = b1;
                h2[2][iy][ox] = b2;
            }
            __syncthreads();
        }
        // Vertical blur of the partials and the chain rule into dL/drender (pass 4, Loss.cpp:160-177),
        // added to the L1 term.
#pragma unroll
        for (int r = 0; r < kPix; ++r) {
            const int k = threadIdx.x + r * kThreads;
            const int ox = k % kTW, oy = k / kTW;
            const int gx = x0 + ox, gy = y0 + oy;
            if (gx >= W || gy >= H)
                continue;
            const size_t idx = (size_t(gy) * W + gx) * 3 + c;
            if (lambda > 0.0f) {
                float g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
                for (int t = 0; t <= 2 * kR; ++t) {
                    const float w = cWin.w[t];
                    g0 += w * h2[0][oy + t][ox];
                    g1 += w * h2[1][oy + t][ox];
                    g2 += w * h2[2][oy + t][ox];
                }
                const float rv = sm.x[oy + kH][ox + kH], tg = sm.y[oy + kH][ox + kH];
                grad[idx] = l1grad[r] + (g0 + 2.0f * rv * g1 + tg * g2);
            } else {
                grad[idx] = l1grad[r];
            }
        }
        __syncthreads();
    }
    const double t0 = blockSumDouble(l1);
    const double t1 = blockSumDouble(ssim);
    const double t2 = blockSumDouble(sq);
    if (threadIdx.x == 0) {
        const int b = blockIdx.y * gridDim.x + blockIdx.x;
        blockSums[3 * b] = t0;
        blockSums[3 * b + 1] = t1;
        blockSums[3 * b + 2] = t2;
    }
}

// Single block: fixed-order sum of the block partials, LossValue, PSNR and the EMA stats.
__global__ void __launch_bounds__(kThreads) lossFinalizeKernel(const double *blockSums, int blocks, int W, int H,
                                                               float lambda, DevStats *stats, int iteration,
                                                               const BinCounts *counts, float *out3, float *psnrOut,
                                                               const StepDesc *desc)
{
    if (desc)
        iteration = desc->iteration + 1;
    if (counts != nullptr && counts->abortIter >= 0)
        stats = nullptr; // an aborted step leaves the statistics alone (it is replayed)
    double s0 = 0, s1 = 0, s2 = 0;
    for (int b = threadIdx.x; b < blocks; b += kThreads) {
        s0 += blockSums[3 * b];
        s1 += blockSums[3 * b + 1];
        s2 += blockSums[3 * b + 2];
    }
    s0 = blockSumDouble(s0);
    s1 = blockSumDouble(s1);
    s2 = blockSumDouble(s2);
    if (threadIdx.x != 0)
        return;
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

int lossBlocks(int width, int height) { return ((width + kTW - 1) / kTW) * ((height + kTH - 1) / kTH); }

void launchLoss(const float *render, const float *targetF, const uint8_t *targetU8, int width, int height, float lambda,
                float *grad, const LossScratch &ls, cudaStream_t s, const StepDesc *desc)
{
    const SsimWindow &win = window();
    static const bool sized = [] {
        cudaFuncSetAttribute(lossKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(LossSmem)));
        return true;
    }();
    (void)sized;
    dim3 g((width + kTW - 1) / kTW, (height + kTH - 1) / kTH);
    { lossKernel<<<g, kThreads, sizeof(LossSmem), s>>>(render, targetF, targetU8, width, height, lambda, grad,
                                                      ls.blockSums, desc, win); countLaunch(); }
}

void launchLossFinalize(const LossScratch &ls, int width, int height, float lambda, DevStats *stats, int iteration,
                        const BinCounts *counts, float *out3, float *psnrOut, cudaStream_t s, const StepDesc *desc)
{
    { lossFinalizeKernel<<<1, kThreads, 0, s>>>(ls.blockSums, ls.blocks, width, height, lambda, stats, iteration,
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
