// common.cuh - shared device definitions of the sm_100a splat trainer.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/u3dg.h"

namespace u3dg {

// Host-side count of the kernels this library has launched (read by u3dg_launch_count).
void countLaunch();

constexpr float kShC0 = 0.28209479177387814f; // degree-0 SH (GaussianModel.h:10)
constexpr float kMaxAlpha = 0.99f;            // Rasterizer.cpp:13
constexpr int kG2d = 9;                       // per-Gaussian 2D gradient: dmx dmy dA dB dC dr dg db dalpha

// Device view of a GaussianModel arena: the five groups one after the other, each strided by the
// arena's capacity, so one allocation of 14 * capacity floats holds a whole model.
struct Params {
    float *means;  // 3 per Gaussian
    float *scales; // 3
    float *quats;  // 4
    float *opac;   // 1
    float *colors; // 3
};

inline Params paramsAt(float *base, size_t capacity)
{
    Params p;
    p.means = base;
    p.scales = base + 3 * capacity;
    p.quats = base + 6 * capacity;
    p.opac = base + 10 * capacity;
    p.colors = base + 11 * capacity;
    return p;
}

// Raster record of one projected Gaussian (48 bytes = 3 x float4): what the compositing kernels
// gather per tile-list entry. (ex, ey) are the half-extents of a conservative axis-aligned box around
// every pixel whose alpha can reach the minimum alpha; compositing warps skip the Gaussian when their
// pixel block lies outside it (the tile lists themselves stay exactly the reference's).
struct __align__(16) SplatRec {
    float mx, my;  // projected mean (pixels)
    float ex, ey;  // contributing half-extents (pixels); +inf = no culling
    float A, B, C; // conic = inverse 2D covariance
    float alpha;   // sigmoid(opacity)
    float r, g, b; // clamped DC colour
    // Lowest Gaussian exponent whose alpha can reach the minimum alpha: ln(minAlpha / alpha) - 1e-4
    // (-inf when minAlpha <= 0). Below it, alpha * expf(power) < minAlpha whatever expf's rounding
    // (at most a few ulps, far inside the 1e-4 margin), so the compositing kernels skip the exponential
    // for those pixels and still decide exactly as the reference does.
    float powMin;
};

// Per-step scalars the device computes and the host reads lazily.
struct DevStats {
    int iteration;
    float loss;       // EMA (Trainer.cpp:88-92)
    float psnr;       // EMA
    float lastLoss;   // this step's LossValue::total
    float lastL1;
    float lastSsim;
    float lastPsnr;
    int pad;
};

// exp rounded from double precision: the correctly rounded float result for all practical inputs.
// glibc's expf (what the reference calls) agrees with it on all but ~7e-5 of float inputs.
__device__ __forceinline__ float expCR(float x) { return (float)exp((double)x); }
__device__ __forceinline__ float sigmoidCR(float x) { return 1.0f / (1.0f + expCR(-x)); }

// Rotation matrix (row-major) of a normalised quaternion (w, x, y, z) (Rasterizer.cpp:24-29).
__device__ __forceinline__ void quatToRot(float w, float x, float y, float z, float R[9])
{
    R[0] = 1 - 2 * (y * y + z * z);
    R[1] = 2 * (x * y - w * z);
    R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);
    R[4] = 1 - 2 * (x * x + z * z);
    R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);
    R[7] = 2 * (y * z + w * x);
    R[8] = 1 - 2 * (x * x + y * y);
}

// Intermediate quantities of one Gaussian's EWA projection (Rasterizer.cpp:32-45).
struct Ewa {
    float pc[3], q[4], qNorm, Rq[9], s[3], M[9], Sigma[9];
    float tx, ty, limTx, limTy;
    bool clampX, clampY;
    float T0[3], T1[3];
    float a, b, c;
};

// EWA projection of Gaussian i (computeProjection, Rasterizer.cpp:48-110), same operation order;
// files including this are compiled with -fmad=false so no multiply-add is contracted.
__device__ __forceinline__ bool ewaProject(const float mu[3], const float qr[4], const float ls[3],
                                           const u3dg_camera &cam, const u3dg_raster_settings &st, Ewa &p)
{
    const float *R = cam.R;
    p.pc[0] = R[0] * mu[0] + R[1] * mu[1] + R[2] * mu[2] + cam.t[0];
    p.pc[1] = R[3] * mu[0] + R[4] * mu[1] + R[5] * mu[2] + cam.t[1];
    p.pc[2] = R[6] * mu[0] + R[7] * mu[1] + R[8] * mu[2] + cam.t[2];
    const float z = p.pc[2];
    if (z < st.near_plane)
        return false;
    p.qNorm = sqrtf(qr[0] * qr[0] + qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
    if (p.qNorm < 1e-12f) {
        p.qNorm = 1.0f;
        p.q[0] = 1;
        p.q[1] = p.q[2] = p.q[3] = 0;
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            p.q[k] = qr[k] / p.qNorm;
    }
    quatToRot(p.q[0], p.q[1], p.q[2], p.q[3], p.Rq);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        p.s[k] = expCR(ls[k]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            p.M[r * 3 + c] = p.Rq[r * 3 + c] * p.s[c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            p.Sigma[r * 3 + c] = p.M[r * 3] * p.M[c * 3] + p.M[r * 3 + 1] * p.M[c * 3 + 1] + p.M[r * 3 + 2] * p.M[c * 3 + 2];
    const float W = float(cam.width), H = float(cam.height);
    const float limXPos = (W - cam.cx) / cam.fx + 0.3f * 0.5f * W / cam.fx;
    const float limXNeg = cam.cx / cam.fx + 0.3f * 0.5f * W / cam.fx;
    const float limYPos = (H - cam.cy) / cam.fy + 0.3f * 0.5f * H / cam.fy;
    const float limYNeg = cam.cy / cam.fy + 0.3f * 0.5f * H / cam.fy;
    const float xz = p.pc[0] / z, yz = p.pc[1] / z;
    // std::min(a, b) = (b < a) ? b : a and std::max(a, b) = (a < b) ? b : a, kept literally.
    const float mxz = (-limXNeg < xz) ? xz : -limXNeg;
    const float cxz = (mxz < limXPos) ? mxz : limXPos;
    const float myz = (-limYNeg < yz) ? yz : -limYNeg;
    const float cyz = (myz < limYPos) ? myz : limYPos;
    p.clampX = cxz != xz;
    p.clampY = cyz != yz;
    p.limTx = cxz;
    p.limTy = cyz;
    p.tx = z * cxz;
    p.ty = z * cyz;
    const float J00 = cam.fx / z, J02 = -cam.fx * p.tx / (z * z);
    const float J11 = cam.fy / z, J12 = -cam.fy * p.ty / (z * z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p.T0[k] = J00 * R[k] + J02 * R[6 + k];
        p.T1[k] = J11 * R[3 + k] + J12 * R[6 + k];
    }
    float S0[3], S1[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        S0[r] = p.Sigma[r * 3] * p.T0[0] + p.Sigma[r * 3 + 1] * p.T0[1] + p.Sigma[r * 3 + 2] * p.T0[2];
        S1[r] = p.Sigma[r * 3] * p.T1[0] + p.Sigma[r * 3 + 1] * p.T1[1] + p.Sigma[r * 3 + 2] * p.T1[2];
    }
    p.a = p.T0[0] * S0[0] + p.T0[1] * S0[1] + p.T0[2] * S0[2] + st.eps2d;
    p.b = p.T0[0] * S1[0] + p.T0[1] * S1[1] + p.T0[2] * S1[2];
    p.c = p.T1[0] * S1[0] + p.T1[1] * S1[1] + p.T1[2] * S1[2] + st.eps2d;
    return true;
}

} // namespace u3dg
