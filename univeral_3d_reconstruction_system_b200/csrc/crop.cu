// crop.cu - cropModel, suggestCropBox and modelBounds (engine/src/splat/Crop.cpp:12-62) on the GPU.
//
// cropModel keeps the Gaussians whose centre lies in an axis-aligned box and whose opacity reaches a
// floor: a keep flag per Gaussian, an exclusive scan of the flags, and a scatter of the kept rows
// (parameters, and the Adam moments when a trainer's model is cropped) in their original order.
//
// The crop boxes are per-axis quantiles of the centres of the opaque Gaussians. The reference takes
// them with std::nth_element on a host copy of each axis; here the axis values of the selected
// Gaussians are gathered as order-preserving 32-bit keys (sign bit flipped for positive floats, all
// bits inverted for negative ones), sorted with the binning's device radix sort, and the two
// quantile positions are read back. The k-th smallest value does not depend on how it was found, so
// the box is the reference's, given the same selection. The selection uses a sigmoid rounded from
// double precision, which agrees with the reference's float sigmoid except within an ulp of the
// floor.

#include "engine.h"

#include <algorithm>
#include <cstring>

namespace u3dg {

namespace {

__device__ __forceinline__ bool inBox(const u3dg_crop_box &b, float x, float y, float z)
{
    return x >= b.min[0] && x <= b.max[0] && y >= b.min[1] && y <= b.max[1] && z >= b.min[2] && z <= b.max[2];
}

// keep[i] = centre in the box and sigmoid(opacity) >= floor (CropBox::contains, Crop.cpp:44-52).
__global__ void cropKeepKernel(Params P, int n, u3dg_crop_box box, float minOpacity, int *keep)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float *m = P.means + size_t(i) * 3;
    keep[i] = (inBox(box, m[0], m[1], m[2]) && sigmoidCR(P.opac[i]) >= minOpacity) ? 1 : 0;
}

// Copies the kept rows of `arenas` consecutive group-major arenas (14 floats per Gaussian each,
// src strided by srcCap, dst by dstCap) to their compacted positions.
__global__ void cropWriteKernel(const float *src, size_t srcCap, float *dst, size_t dstCap, int arenas, int n,
                                const int *keep, const int *pos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !keep[i])
        return;
    const size_t j = size_t(pos[i]);
    // Group offsets of an arena in units of its capacity: means 0, scales 3, quats 6, opacities 10,
    // colours 11 (paramsAt).
    for (int a = 0; a < arenas; ++a) {
        const float *S = src + size_t(a) * 14 * srcCap;
        float *D = dst + size_t(a) * 14 * dstCap;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            D[j * 3 + k] = S[size_t(i) * 3 + k];
            D[3 * dstCap + j * 3 + k] = S[3 * srcCap + size_t(i) * 3 + k];
            D[11 * dstCap + j * 3 + k] = S[11 * srcCap + size_t(i) * 3 + k];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            D[6 * dstCap + j * 4 + k] = S[6 * srcCap + size_t(i) * 4 + k];
        D[10 * dstCap + j] = S[10 * srcCap + i];
    }
}

__global__ void opaqueKernel(const float *opac, int n, float minOpacity, int *flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        flag[i] = sigmoidCR(opac[i]) >= minOpacity ? 1 : 0;
}

__device__ __forceinline__ uint32_t orderKey(float v)
{
    const uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// keys[pos[i]] = order key of axis `axis` of every selected Gaussian (flag[i], or all when useAll).
__global__ void axisKeysKernel(const float *means, int n, int axis, const int *flag, const int *pos, int useAll,
                               uint32_t *keys)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    if (useAll)
        keys[i] = orderKey(means[size_t(i) * 3 + axis]);
    else if (flag[i])
        keys[pos[i]] = orderKey(means[size_t(i) * 3 + axis]);
}

__global__ void setIntKernel(int *p, int v) { *p = v; }

inline int grid(int n) { return (n + 255) / 256; }

float keyValue(uint32_t k)
{
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

} // namespace

size_t cropKeep(const Params &P, int n, const u3dg_crop_box &box, float minOpacity, DevBuf<int> &keep,
                DevBuf<int> &pos, DevBuf<int> &scratch, cudaStream_t s)
{
    keep.reserve(size_t(n) + 1);
    pos.reserve(size_t(n) + 1);
    scratch.reserve(scanPartialEntries(n) + 1);
    if (n > 0)
        { cropKeepKernel<<<grid(n), 256, 0, s>>>(P, n, box, minOpacity, keep.p); countLaunch(); }
    exclusiveScan(keep.p, pos.p, n, scratch.p, s);
    int kept = 0;
    U3DG_CUDA(cudaMemcpyAsync(&kept, pos.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaStreamSynchronize(s));
    return size_t(kept);
}

void launchCropWrite(const float *src, size_t srcCap, float *dst, size_t dstCap, int arenas, int n, const int *keep,
                     const int *pos, cudaStream_t s)
{
    if (n > 0)
        { cropWriteKernel<<<grid(n), 256, 0, s>>>(src, srcCap, dst, dstCap, arenas, n, keep, pos); countLaunch(); }
}

u3dg_crop_box quantileBoxOnDevice(const Params &P, int n, float lo, float hi, float margin, float minOpacity,
                                  cudaStream_t s)
{
    u3dg_crop_box box{};
    if (n <= 0) { // no centres at all (Crop.cpp:28-32)
        for (int k = 0; k < 3; ++k) {
            box.min[k] = -1.0f;
            box.max[k] = 1.0f;
        }
        return box;
    }
    DevBuf<int> flag, pos, scratch, count;
    DevBuf<uint32_t> keysA, keysB, valsA, valsB;
    DevBuf<int> hist, rowTotals;
    flag.reserve(size_t(n) + 1);
    pos.reserve(size_t(n) + 1);
    scratch.reserve(scanPartialEntries(n) + 1);
    count.reserve(1);
    for (DevBuf<uint32_t> *b : {&keysA, &keysB, &valsA, &valsB})
        b->reserve(size_t(n));
    hist.reserve(radixHistEntries(n));
    rowTotals.reserve(size_t(radixDigits()));
    { opaqueKernel<<<grid(n), 256, 0, s>>>(P.opac, n, minOpacity, flag.p); countLaunch(); }
    exclusiveScan(flag.p, pos.p, n, scratch.p, s);
    int selected = 0;
    U3DG_CUDA(cudaMemcpyAsync(&selected, pos.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaStreamSynchronize(s));
    const bool useAll = selected == 0; // everything faint: all centres (Crop.cpp:24-26)
    const int m = useAll ? n : selected;
    // Quantile positions exactly as the reference computes them in float (Crop.cpp:33-36).
    auto at = [m](float q) { return std::min(size_t(m) - 1, size_t(q * float(m - 1) + 0.5f)); };
    const size_t ia = at(lo), ib = at(hi);
    for (int k = 0; k < 3; ++k) {
        { axisKeysKernel<<<grid(n), 256, 0, s>>>(P.means, n, k, flag.p, pos.p, useAll ? 1 : 0, keysA.p); countLaunch(); }
        { setIntKernel<<<1, 1, 0, s>>>(count.p, m); countLaunch(); }
        uint32_t *kout = nullptr, *vout = nullptr;
        radixSortPairs(keysA.p, keysB.p, valsA.p, valsB.p, count.p, m, 32, hist.p, rowTotals.p, &kout, &vout, s);
        uint32_t a = 0, b = 0;
        U3DG_CUDA(cudaMemcpyAsync(&a, kout + ia, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(&b, kout + ib, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaStreamSynchronize(s));
        const float fa = keyValue(a), fb = keyValue(b);
        const float pad = std::max((fb - fa) * margin, 1e-4f);
        box.min[k] = fa - pad;
        box.max[k] = fb + pad;
    }
    return box;
}

} // namespace u3dg
