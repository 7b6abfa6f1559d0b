// warmstart.h - learned warm-start network: sizes and launch interface (see warmstart.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/u3dg.h"

namespace u3dg {

constexpr int kWarmInputs = 134;
constexpr int kWarmHidden = 128;
constexpr int kWarmOutputs = 11;
constexpr int kWarmNeighbours = 16;
constexpr int kWarmViews = 7;
// Layer l maps kWarmIn[l] -> kWarmOut[l]; parameters are W (out x in) then b, layer after layer.
constexpr int kWarmLayers = 4;
constexpr int kWarmIn[kWarmLayers] = {kWarmInputs, kWarmHidden, kWarmHidden, kWarmHidden};
constexpr int kWarmOut[kWarmLayers] = {kWarmHidden, kWarmHidden, kWarmHidden, kWarmOutputs};
constexpr int kWarmParams = kWarmInputs * kWarmHidden + kWarmHidden + 2 * (kWarmHidden * kWarmHidden + kWarmHidden) +
                            kWarmHidden * kWarmOutputs + kWarmOutputs; // 51,723

void launchKnn(const float *queries, int nq, const float *points, int np, int k, int excludeSelf, int *idx, float *d2,
               cudaStream_t s);
size_t warmViewRefBytes();
void fillWarmViewRef(void *dst, const u3dg_camera &cam, const uint8_t *rgbDev);
void launchWarmFeatures(const float *xyz, const float *rgb, int n, const int *nbr, const float *nd2,
                        const float *baseScale, const void *views, int nViews, float *feat, cudaStream_t s);
void launchGemm(const float *A, int sAm, int sAk, const float *B, int sBk, int sBn, float *C, int ldc, int M, int N,
                int K, const float *bias, bool relu, cudaStream_t s);
void launchReluBackward(float *d, const float *y, size_t count, cudaStream_t s);
void launchColumnSum(const float *d, int n, int out, float *db, cudaStream_t s);
int mseBlocks();
void launchMse(const float *y, const float *t, const float *w, int n, float *dy, double *partial, float *lossOut,
               cudaStream_t s);
void launchAdamFlat(float *p, const float *g, float *m, float *v, int n, float stepSize, float invSqrtBc2, float eps,
                    cudaStream_t s);
void launchGatherRows(const float *src, int width, const int *rows, int n, float *dst, cudaStream_t s);
void launchWarmCombine(const float *pred, int n, float *scales, float *quats, float *opac, float *colors,
                       cudaStream_t s);

} // namespace u3dg
