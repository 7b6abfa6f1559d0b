// gaussian.cu - per-Gaussian kernels: EWA projection, chain rule fused with Adam, standalone Adam,
// densification (clone / split / prune with the greedy budget) and opacity reset.
//
// Compiled with -fmad=false: every float expression keeps the reference's operation order without
// multiply-add contraction, so that for the same inputs these kernels give the reference's bits
// except where glibc's expf differs from the correctly rounded exp used here (expCR).
// All of these kernels stream over Gaussians and are HBM-bound.

#include "tile_cull.cuh"

#include <cfloat>
#include <climits>

namespace u3dg {

namespace {

__device__ __forceinline__ float stdMax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float mid2(const Ewa &p) { return 0.5f * (p.a + p.c); }

// Degree 1..3 real-SH colour terms, 3DGS sign convention; coef points at 15 * 3 floats.
__device__ float shRest(const float *coef, int degree, int ch, const float d[3])
{
    const float x = d[0], y = d[1], z = d[2];
    auto c = [&](int k) { return coef[(k - 1) * 3 + ch]; };
    float sum = 0.0f;
    if (degree >= 1) {
        const float C1 = 0.4886025119029199f;
        sum += -C1 * y * c(1);
        sum += C1 * z * c(2);
        sum += -C1 * x * c(3);
    }
    if (degree >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        sum += 1.0925484305920792f * (x * y) * c(4);
        sum += -1.0925484305920792f * (y * z) * c(5);
        sum += 0.31539156525252005f * (2.0f * zz - xx - yy) * c(6);
        sum += -1.0925484305920792f * (x * z) * c(7);
        sum += 0.5462742152960396f * (xx - yy) * c(8);
        if (degree >= 3) {
            sum += -0.5900435899266435f * y * (3.0f * xx - yy) * c(9);
            sum += 2.890611442640554f * (x * y) * z * c(10);
            sum += -0.4570457994644658f * y * (4.0f * zz - xx - yy) * c(11);
            sum += 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * c(12);
            sum += -0.4570457994644658f * x * (4.0f * zz - xx - yy) * c(13);
            sum += 1.445305721320277f * z * (xx - yy) * c(14);
            sum += -0.5900435899266435f * x * (xx - 3.0f * yy) * c(15);
        }
    }
    return sum;
}

// Rasterizer::project (Rasterizer.cpp:137-204) for one Gaussian per thread.
__global__ void __launch_bounds__(256) projectKernel(Params P, int n, u3dg_camera camArg, u3dg_raster_settings st,
                                                     int tilesX, int tilesY, const float *shRestCoef, int shDegree,
                                                     float3 camPos, ProjOut out, const StepDesc *desc)
{
    pdlEntry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const u3dg_camera cam = desc ? desc->cam : camArg;
    const float mu[3] = {P.means[3 * i], P.means[3 * i + 1], P.means[3 * i + 2]};
    const float qr[4] = {P.quats[4 * i], P.quats[4 * i + 1], P.quats[4 * i + 2], P.quats[4 * i + 3]};
    const float ls[3] = {P.scales[3 * i], P.scales[3 * i + 1], P.scales[3 * i + 2]};
    const int ts = st.tile_size;
    Ewa p;
    int radius = 0;
    int4 rect = make_int4(0, 0, 0, 0);
    bool visible = ewaProject(mu, qr, ls, cam, st, p);
    float det = 0.0f, u = 0.0f, v = 0.0f;
    if (visible) {
        det = p.a * p.c - p.b * p.b;
        visible = det > 0.0f;
    }
    if (visible) {
        const float z = p.pc[2];
        u = cam.fx * p.pc[0] / z + cam.cx;
        v = cam.fy * p.pc[1] / z + cam.cy;
        const float mid = 0.5f * (p.a + p.c);
        const float lambda = mid + sqrtf(stdMax(0.1f, mid * mid - det));
        const float rf = ceilf(3.0f * sqrtf(lambda));
        // int(float) of values outside int range gives INT_MIN on x86-64 (cvttss2si), which the
        // reference's visibility test below then rejects; reproduce that instead of saturating.
        radius = (rf < 2147483648.0f) ? int(rf) : INT_MIN;
        const float fr = float(radius);
        if (u + fr < 0 || v + fr < 0 || u - fr >= float(cam.width) || v - fr >= float(cam.height)) {
            visible = false;
        } else {
            const int tx0 = max(0, int(floorf((u - fr) / float(ts))));
            const int ty0 = max(0, int(floorf((v - fr) / float(ts))));
            const int tx1 = min(tilesX, int(floorf((u + fr) / float(ts))) + 1);
            const int ty1 = min(tilesY, int(floorf((v + fr) / float(ts))) + 1);
            if (tx0 >= tx1 || ty0 >= ty1)
                visible = false;
            else
                rect = make_int4(tx0, ty0, tx1, ty1);
        }
    }
    if (!visible) {
        out.radius[i] = 0;
        out.rect[i] = make_int4(0, 0, 0, 0);
        out.depthKey[i] = 0xFFFFFFFFu;
        out.flags[i] = 0;
        out.tileCount[i] = 0;
        return;
    }
    const float invDet = 1.0f / det;
    SplatRec r;
    r.mx = u;
    r.my = v;
    r.A = p.c * invDet;
    r.B = -p.b * invDet;
    r.C = p.a * invDet;
    uint8_t f = uint8_t((p.clampX ? 1 : 0) | (p.clampY ? 2 : 0));
    float dir[3] = {0.0f, 0.0f, 0.0f};
    const int K = (shDegree + 1) * (shDegree + 1) - 1;
    if (shRestCoef != nullptr && shDegree > 0) {
        const float dd[3] = {mu[0] - camPos.x, mu[1] - camPos.y, mu[2] - camPos.z};
        float nrm = 0.0f;
        for (int k = 0; k < 3; ++k)
            nrm += dd[k] * dd[k];
        nrm = sqrtf(nrm);
        for (int k = 0; k < 3; ++k)
            dir[k] = dd[k] / nrm;
    }
    float col3[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float term = kShC0 * P.colors[3 * i + ch];
        if (shRestCoef != nullptr && shDegree > 0)
            term = term + shRest(shRestCoef + size_t(i) * size_t(K) * 3, shDegree, ch, dir);
        const float col = 0.5f + term;
        if (col < 0.0f)
            f |= uint8_t(4 << ch);
        col3[ch] = stdMax(col, 0.0f);
    }
    r.r = col3[0];
    r.g = col3[1];
    r.b = col3[2];
    r.alpha = sigmoidCR(P.opac[i]);
    r.powMin = st.min_alpha > 0.0f ? logf(st.min_alpha / r.alpha) - 1e-4f : -__int_as_float(0x7f800000);
    // Contributing box: alpha = min(0.99, a exp(-q/2)) >= minAlpha  <=>  q <= t = 2 ln(a / minAlpha), and
    // {q <= t} lies within |dx| <= sqrt(t Sxx), |dy| <= sqrt(t Syy). The float evaluation of q in the
    // compositing kernels may differ from the exact q by a few ulps times the covariance condition
    // number, so t is widened by 2% (enough up to a condition number of 1e4; beyond that, no culling)
    // and the box by one pixel.
    {
        const float disc = stdMax(0.0f, mid2(p) * mid2(p) - det);
        const float lmax = mid2(p) + sqrtf(disc), lmin = mid2(p) - sqrtf(disc);
        const float minA = st.min_alpha;
        if (minA > 0.0f && lmin > 0.0f && lmax <= 1e4f * lmin) {
            const float t = 2.0f * logf(r.alpha / minA);
            const float tt = stdMax(t, 0.0f) * 1.02f + 1e-5f;
            r.ex = sqrtf(tt * p.a) + 1.0f;
            r.ey = sqrtf(tt * p.c) + 1.0f;
        } else {
            r.ex = r.ey = __int_as_float(0x7f800000);
        }
    }
    out.rec[i] = r;
    out.cov2d[i] = make_float4(p.a, p.b, p.c, 0.0f);
    out.flags[i] = f;
    out.rect[i] = rect;
    out.radius[i] = radius;
    out.depth[i] = p.pc[2];
    out.depthKey[i] = __float_as_uint(p.pc[2]);
    // The tiles it is listed in (Rasterizer.cpp:206-261 lists the whole rectangle; the trainers only the
    // tiles its contributing ellipse reaches), counted here where the record is in registers; the
    // binning scans the counts in depth order.
    int tiles = 0;
    if (radius > 0) {
        const bool cull = out.cullTiles != 0;
        const CullShape cs = cull ? cullShapeOf(make_float4(r.mx, r.my, r.ex, r.ey), make_float4(r.A, r.B, r.C, r.alpha),
                                                r.powMin)
                                  : CullShape{};
        tiles = listedTiles(cs, cull, rect, ts, cull ? out.rowTab + size_t(i) * kCullRows : nullptr);
    }
    out.tileCount[i] = tiles;
}

// One Adam element update (adamArray, Adam.cpp:13-28), same order as the reference.
__device__ __forceinline__ void adamOne(float &p, float &m, float &v, float g, float stepSize, float invSqrtBc2)
{
    m = 0.9f * m + (1.0f - 0.9f) * g;
    v = 0.999f * v + (1.0f - 0.999f) * g * g;
    p -= stepSize * m / (sqrtf(v) * invSqrtBc2 + 1e-15f);
}

// The 9 summed 2D gradients of every Gaussian from the per-(tile, Gaussian) partials of the
// compositing backward. Emission order is depth-rank order, so a rank's partials are contiguous: one
// warp per 32 consecutive ranks walks their partials 32 entries at a time (coalesced), lane j holding
// entry j of the chunk; a segmented inclusive scan over the lanes (segments = ranks) adds the entries
// of each rank in lane order, and each rank's lane adds the scan value at its last entry in the chunk.
// The order of the additions is fixed, so the sums are deterministic. Written per Gaussian id.
__global__ void __launch_bounds__(256) partialSumKernel(const float *partial, int subSlots, size_t subStride,
                                                        const int *offs, const uint32_t *sortedIds, int n,
                                                        const BinCounts *counts, float *g2d)
{
    pdlEntry();
    if (counts != nullptr && counts->abortIter >= 0)
        return;
    const int lane = threadIdx.x & 31;
    const int warps = int((gridDim.x * blockDim.x) >> 5);
    for (int w = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w * 32 < n; w += warps) {
        const int r = w * 32 + lane;
        const bool valid = r < n;
        const int o = valid ? offs[r] : INT_MAX;
        const int oEnd = valid ? offs[r + 1] : INT_MAX;
        const int first = offs[w * 32], last = offs[min(w * 32 + 32, n)];
        float acc[kG2d];
#pragma unroll
        for (int k = 0; k < kG2d; ++k)
            acc[k] = 0.0f;
        for (int c0 = first; c0 < last; c0 += 32) {
            const int e = c0 + lane;
            const bool in = e < last;
            // Owner of entry e: the last lane whose start offset is not above e.
            int owner = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int oc = __shfl_sync(0xffffffffu, o, owner + step);
                if (oc <= e)
                    owner += step;
            }
            float v[kG2d];
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                v[k] = in ? partial[size_t(e) * kG2d + k] : 0.0f;
            // Tiles covered by several CTAs: their slots, added in slot order.
            for (int sl = 1; sl < subSlots; ++sl) {
                const float *p = partial + size_t(sl) * subStride;
#pragma unroll
                for (int k = 0; k < kG2d; ++k)
                    v[k] = __fadd_rn(v[k], in ? p[size_t(e) * kG2d + k] : 0.0f);
            }
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int ownerUp = __shfl_up_sync(0xffffffffu, owner, d);
                const bool same = lane >= d && ownerUp == owner;
#pragma unroll
                for (int k = 0; k < kG2d; ++k) {
                    const float up = __shfl_up_sync(0xffffffffu, v[k], d);
                    if (same)
                        v[k] = __fadd_rn(v[k], up);
                }
            }
            // This lane's rank: its last entry inside the chunk, if any.
            const int lastE = min(min(oEnd, last), c0 + 32) - 1;
            const bool has = valid && o < c0 + 32 && oEnd > c0 && lastE >= max(o, c0);
            const int src = has ? lastE - c0 : lane;
#pragma unroll
            for (int k = 0; k < kG2d; ++k) {
                const float got = __shfl_sync(0xffffffffu, v[k], src);
                if (has)
                    acc[k] = __fadd_rn(acc[k], got);
            }
        }
        if (valid) {
            float *dst = g2d + size_t(sortedIds[r]) * kG2d;
#pragma unroll
            for (int k = 0; k < kG2d; ++k)
                dst[k] = acc[k];
        }
    }
}

// Rasterizer::backward pass 2 (Rasterizer.cpp:432-544) for one Gaussian per thread, fused either with
// Adam::step (kAdam: the trainer; gradients never leave registers) or with adding the gradients into
// caller arrays (the unit entry point). The per-Gaussian 2D gradient comes from partialSumKernel.
// Resident CTAs per SM the compiler must allow for: caps registers per thread at 65536 / (256 * n)
// (64 at 4; the kernel is latency-bound, and 4 CTAs per SM beat fewer with more registers).
#ifndef U3DG_CHAIN_MIN_BLOCKS
#define U3DG_CHAIN_MIN_BLOCKS 4
#endif

template <bool kAdam>
__global__ void __launch_bounds__(256, U3DG_CHAIN_MIN_BLOCKS) chainKernel(ChainArgs a)
{
    pdlEntry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n || (a.counts != nullptr && a.counts->abortIter >= 0))
        return;
    const Params &P = a.params;
    float gMeans[3] = {0, 0, 0}, gScales[3] = {0, 0, 0}, gQuats[4] = {0, 0, 0, 0}, gOpac = 0, gColors[3] = {0, 0, 0};
    if (a.radius[i] > 0) {
        float g[kG2d];
#pragma unroll
        for (int k = 0; k < kG2d; ++k)
            g[k] = a.g2d[size_t(i) * kG2d + k];
        const u3dg_camera &cam = a.desc ? a.desc->cam : a.cam;
        const float dmx = g[0], dmy = g[1], dA = g[2], dB = g[3], dC = g[4];
        if (a.gradAccum != nullptr) {
            const float nx = dmx * 0.5f * float(cam.width), ny = dmy * 0.5f * float(cam.height);
            a.gradAccum[i] += sqrtf(nx * nx + ny * ny);
        }
        if (a.gradCount != nullptr)
            a.gradCount[i] += 1;
        const uint8_t fl = a.flags[i];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
            if (!(fl & (4 << ch)))
                gColors[ch] = kShC0 * g[5 + ch];
        const float op = a.rec[i].alpha;
        gOpac = g[8] * op * (1.0f - op);

        const float mu[3] = {P.means[3 * i], P.means[3 * i + 1], P.means[3 * i + 2]};
        const float qr[4] = {P.quats[4 * i], P.quats[4 * i + 1], P.quats[4 * i + 2], P.quats[4 * i + 3]};
        const float ls[3] = {P.scales[3 * i], P.scales[3 * i + 1], P.scales[3 * i + 2]};
        Ewa p;
        ewaProject(mu, qr, ls, cam, a.st, p);
        const float z = p.pc[2];
        const float aa = p.a, bb = p.b, cc = p.c;
        const float det = aa * cc - bb * bb;
        const float det2 = det * det;
        const float da = (dA * -cc * cc + dB * bb * cc + dC * -bb * bb) / det2;
        const float db = (dA * 2 * bb * cc + dC * 2 * aa * bb) / det2 + dB * (-1.0f / det - 2 * bb * bb / det2);
        const float dc = (dA * -bb * bb + dB * aa * bb + dC * -aa * aa) / det2;
        const float G00 = da, G01 = 0.5f * db, G11 = dc;
        float dSigma[9];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int l = 0; l < 3; ++l)
                dSigma[k * 3 + l] = p.T0[k] * (G00 * p.T0[l] + G01 * p.T1[l]) + p.T1[k] * (G01 * p.T0[l] + G11 * p.T1[l]);
        float TS0[3], TS1[3];
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            TS0[col] = p.T0[0] * p.Sigma[col] + p.T0[1] * p.Sigma[3 + col] + p.T0[2] * p.Sigma[6 + col];
            TS1[col] = p.T1[0] * p.Sigma[col] + p.T1[1] * p.Sigma[3 + col] + p.T1[2] * p.Sigma[6 + col];
        }
        float dT0[3], dT1[3];
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            dT0[col] = 2.0f * (G00 * TS0[col] + G01 * TS1[col]);
            dT1[col] = 2.0f * (G01 * TS0[col] + G11 * TS1[col]);
        }
        float dM[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int col = 0; col < 3; ++col)
                dM[r * 3 + col] = 2.0f * (dSigma[r * 3] * p.M[col] + dSigma[r * 3 + 1] * p.M[3 + col] + dSigma[r * 3 + 2] * p.M[6 + col]);
        float dRq[9];
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            float ds = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                ds += dM[r * 3 + col] * p.Rq[r * 3 + col];
                dRq[r * 3 + col] = dM[r * 3 + col] * p.s[col];
            }
            gScales[col] = ds * p.s[col];
        }
        const float w = p.q[0], x = p.q[1], y = p.q[2], zq = p.q[3];
        const float dw = 2 * (-zq * dRq[1] + y * dRq[2] + zq * dRq[3] - x * dRq[5] - y * dRq[6] + x * dRq[7]);
        const float dx = 2 * (y * dRq[1] + zq * dRq[2] + y * dRq[3] - 2 * x * dRq[4] - w * dRq[5] + zq * dRq[6] + w * dRq[7] - 2 * x * dRq[8]);
        const float dy = 2 * (-2 * y * dRq[0] + x * dRq[1] + w * dRq[2] + x * dRq[3] + zq * dRq[5] - w * dRq[6] + zq * dRq[7] - 2 * y * dRq[8]);
        const float dz = 2 * (-2 * zq * dRq[0] - w * dRq[1] + x * dRq[2] + w * dRq[3] - 2 * zq * dRq[4] + y * dRq[5] + x * dRq[6] + y * dRq[7]);
        const float dq[4] = {dw, dx, dy, dz};
        const float qdot = dq[0] * p.q[0] + dq[1] * p.q[1] + dq[2] * p.q[2] + dq[3] * p.q[3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            gQuats[k] = (dq[k] - qdot * p.q[k]) / p.qNorm;
        const float *R = cam.R;
        const float dJ00 = dT0[0] * R[0] + dT0[1] * R[1] + dT0[2] * R[2];
        const float dJ02 = dT0[0] * R[6] + dT0[1] * R[7] + dT0[2] * R[8];
        const float dJ11 = dT1[0] * R[3] + dT1[1] * R[4] + dT1[2] * R[5];
        const float dJ12 = dT1[0] * R[6] + dT1[1] * R[7] + dT1[2] * R[8];
        const float z2 = z * z, z3 = z2 * z;
        float dpc[3] = {0, 0, 0};
        dpc[2] += dJ00 * -cam.fx / z2 + dJ02 * 2 * cam.fx * p.tx / z3 + dJ11 * -cam.fy / z2 + dJ12 * 2 * cam.fy * p.ty / z3;
        const float dtx = dJ02 * -cam.fx / z2;
        const float dty = dJ12 * -cam.fy / z2;
        if (p.clampX)
            dpc[2] += dtx * p.limTx;
        else
            dpc[0] += dtx;
        if (p.clampY)
            dpc[2] += dty * p.limTy;
        else
            dpc[1] += dty;
        dpc[0] += dmx * cam.fx / z;
        dpc[1] += dmy * cam.fy / z;
        dpc[2] += -dmx * cam.fx * p.pc[0] / z2 - dmy * cam.fy * p.pc[1] / z2;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            gMeans[k] = R[k] * dpc[0] + R[3 + k] * dpc[1] + R[6 + k] * dpc[2];
    }

    if constexpr (kAdam) {
        const Params &M = a.m, &V = a.v;
        const float inv = a.desc ? a.desc->invSqrtBc2 : a.invSqrtBc2;
        const float *lr = a.desc ? a.desc->stepSize : a.stepSize;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            adamOne(P.means[3 * i + k], M.means[3 * i + k], V.means[3 * i + k], gMeans[k], lr[0], inv);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            adamOne(P.scales[3 * i + k], M.scales[3 * i + k], V.scales[3 * i + k], gScales[k], lr[1], inv);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            adamOne(P.quats[4 * i + k], M.quats[4 * i + k], V.quats[4 * i + k], gQuats[k], lr[2], inv);
        adamOne(P.opac[i], M.opac[i], V.opac[i], gOpac, lr[3], inv);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            adamOne(P.colors[3 * i + k], M.colors[3 * i + k], V.colors[3 * i + k], gColors[k], lr[4], inv);
    } else {
        const Params &G = a.grads;
        if (a.radius[i] > 0) {
            for (int k = 0; k < 3; ++k)
                G.means[3 * i + k] += gMeans[k];
            for (int k = 0; k < 3; ++k)
                G.scales[3 * i + k] += gScales[k];
            for (int k = 0; k < 4; ++k)
                G.quats[4 * i + k] += gQuats[k];
            G.opac[i] += gOpac;
            for (int k = 0; k < 3; ++k)
                G.colors[3 * i + k] += gColors[k];
        }
    }
}

// Adam::step over one group segment: `len` elements starting at p/g/m/v.
__global__ void adamKernel(float *p, const float *g, float *m, float *v, int len, float stepSize, float invSqrtBc2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < len) {
        float pk = p[k], mk = m[k], vk = v[k];
        adamOne(pk, mk, vk, g[k], stepSize, invSqrtBc2);
        p[k] = pk;
        m[k] = mk;
        v[k] = vk;
    }
}

// Trainer::densifyAndPrune (Trainer.cpp:105-169), step 1: per Gaussian, prune flag and candidate
// kind (0 none, 1 clone, 2 split); `cost` doubles as the number of slots a candidate needs.
__global__ void densifyClassifyKernel(Params P, int n, const float *gradAccum, const int *gradCount, float extent,
                                      float splitScale, float pruneOpacity, float gradThreshold, int opacityWasReset,
                                      int *keep, int *cost)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float s0 = P.scales[3 * i], s1 = P.scales[3 * i + 1], s2 = P.scales[3 * i + 2];
    // std::max({a, b, c}) keeps the first of equal maxima: max(max(a, b), c) with (x < y) ? y : x.
    const float maxLog = stdMax(stdMax(s0, s1), s2);
    const float maxScale = expCR(maxLog);
    const float alpha = sigmoidCR(P.opac[i]);
    int k = 1, c = 0;
    if (alpha < pruneOpacity || (opacityWasReset && maxScale > 0.1f * extent)) {
        k = 0;
    } else if (gradCount[i] != 0) {
        const float avg = gradAccum[i] / float(gradCount[i]);
        if (!(avg < gradThreshold))
            c = (maxScale <= splitScale) ? 1 : 2;
    }
    keep[i] = k;
    cost[i] = c;
}

// Step 2: the first candidate the greedy budget rejects (Trainer.cpp:130-137): the lowest i with
// prefix(cost) + cost > budget. *first starts at a value >= n (none).
__global__ void densifyFirstRejectKernel(int n, const int *cost, const int *costScan, long long budget, int *first)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && cost[i] > 0 && (long long)costScan[i] + cost[i] > budget)
        atomicMin(first, i);
}

// Step 3: if that first rejected candidate was a split with exactly one slot left, the next clone
// after it still fits (and then the budget is full). *second starts at a value >= n (none).
__global__ void densifyLastCloneKernel(int n, const int *cost, const int *costScan, long long budget, const int *first,
                                       int *second)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = *first;
    if (f >= n || i >= n || i <= f)
        return;
    if (cost[f] == 2 && (long long)costScan[f] == budget - 1 && cost[i] == 1)
        atomicMin(second, i);
}

// Step 4: accepted candidates: slots they take (accCost), whether they are splits (isSplit), and
// keep = 0 for accepted splits (the parent is replaced by its two children).
__global__ void densifyAcceptKernel(int n, const int *cost, const int *first, const int *second, int *keep, int *accCost,
                                    int *isSplit)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int c = cost[i];
    const bool acc = c > 0 && (i < *first || i == *second);
    accCost[i] = acc ? c : 0;
    isSplit[i] = (acc && c == 2) ? 1 : 0;
    if (acc && c == 2)
        keep[i] = 0;
}

// Step 5: write the densified model into the other arena: survivors in order, then the clones and
// split children in candidate order (GaussianModel::compact + appendFrom, Adam::compact + grow).
// normals holds 6 N(0,1) samples per accepted split, drawn on the host in the reference's order.
__global__ void densifyWriteKernel(Params P, Params M, Params V, Params P2, Params M2, Params V2, int n,
                                   const int *keep, const int *keepScan, const int *accCost, const int *accScan,
                                   const int *isSplit, const int *splitScan, int keptTotal, const float *normals,
                                   float log16)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    if (keep[i]) {
        const int o = keepScan[i];
        for (int k = 0; k < 3; ++k) {
            P2.means[3 * o + k] = P.means[3 * i + k];
            M2.means[3 * o + k] = M.means[3 * i + k];
            V2.means[3 * o + k] = V.means[3 * i + k];
            P2.scales[3 * o + k] = P.scales[3 * i + k];
            M2.scales[3 * o + k] = M.scales[3 * i + k];
            V2.scales[3 * o + k] = V.scales[3 * i + k];
            P2.colors[3 * o + k] = P.colors[3 * i + k];
            M2.colors[3 * o + k] = M.colors[3 * i + k];
            V2.colors[3 * o + k] = V.colors[3 * i + k];
        }
        for (int k = 0; k < 4; ++k) {
            P2.quats[4 * o + k] = P.quats[4 * i + k];
            M2.quats[4 * o + k] = M.quats[4 * i + k];
            V2.quats[4 * o + k] = V.quats[4 * i + k];
        }
        P2.opac[o] = P.opac[i];
        M2.opac[o] = M.opac[i];
        V2.opac[o] = V.opac[i];
    }
    const int c = accCost[i];
    if (c == 0)
        return;
    const int base = keptTotal + accScan[i];
    float R[9];
    if (isSplit[i]) {
        const float *q = &P.quats[4 * i];
        const float qn = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + 1e-12f;
        quatToRot(q[0] / qn, q[1] / qn, q[2] / qn, q[3] / qn, R);
    }
    const float *nrm = normals + size_t(splitScan[i]) * 6;
    for (int child = 0; child < c; ++child) {
        const int o = base + child;
        float mean[3] = {P.means[3 * i], P.means[3 * i + 1], P.means[3 * i + 2]};
        float sc[3] = {P.scales[3 * i], P.scales[3 * i + 1], P.scales[3 * i + 2]};
        if (isSplit[i]) {
            float local[3];
            for (int k = 0; k < 3; ++k)
                local[k] = nrm[child * 3 + k] * expCR(P.scales[3 * i + k]);
            for (int r = 0; r < 3; ++r)
                mean[r] += R[r * 3] * local[0] + R[r * 3 + 1] * local[1] + R[r * 3 + 2] * local[2];
            for (int k = 0; k < 3; ++k)
                sc[k] -= log16;
        }
        for (int k = 0; k < 3; ++k) {
            P2.means[3 * o + k] = mean[k];
            P2.scales[3 * o + k] = sc[k];
            P2.colors[3 * o + k] = P.colors[3 * i + k];
            M2.means[3 * o + k] = M2.scales[3 * o + k] = M2.colors[3 * o + k] = 0.0f;
            V2.means[3 * o + k] = V2.scales[3 * o + k] = V2.colors[3 * o + k] = 0.0f;
        }
        for (int k = 0; k < 4; ++k) {
            P2.quats[4 * o + k] = P.quats[4 * i + k];
            M2.quats[4 * o + k] = 0.0f;
            V2.quats[4 * o + k] = 0.0f;
        }
        P2.opac[o] = P.opac[i];
        M2.opac[o] = 0.0f;
        V2.opac[o] = 0.0f;
    }
}

// Trainer::resetOpacity (Trainer.cpp:171-178): opacity = std::min(opacity, cap); opacity moments = 0.
__global__ void opacityResetKernel(float *opac, float *mOpac, float *vOpac, int n, float cap, const BinCounts *counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (counts != nullptr && counts->abortIter >= 0)
        return;
    if (i < n) {
        const float o = opac[i];
        opac[i] = (cap < o) ? cap : o;
        mOpac[i] = 0.0f;
        vOpac[i] = 0.0f;
    }
}

inline int blocks(long long n, int threads) { return int((n + threads - 1) / threads); }

} // namespace

void launchProject(const Params &P, int n, const u3dg_camera &cam, const u3dg_raster_settings &st, int tilesX,
                   int tilesY, const float *shRest, int shDegree, const ProjOut &out, cudaStream_t s,
                   const StepDesc *desc)
{
    if (n <= 0)
        return;
    float3 camPos = make_float3(0, 0, 0);
    if (shRest != nullptr && shDegree > 0) {
        // Camera centre -R^T t in float, the same expression order as the CPU oracle.
        camPos.x = -(cam.R[0] * cam.t[0] + cam.R[3] * cam.t[1] + cam.R[6] * cam.t[2]);
        camPos.y = -(cam.R[1] * cam.t[0] + cam.R[4] * cam.t[1] + cam.R[7] * cam.t[2]);
        camPos.z = -(cam.R[2] * cam.t[0] + cam.R[5] * cam.t[1] + cam.R[8] * cam.t[2]);
    }
    if (desc)
        shDegree = 0;
    { launchPdl(projectKernel, blocks(n, 256), 256, 0, s, P, n, cam, st, tilesX, tilesY, shRest, shDegree, camPos, out, desc); countLaunch(); }
}

void launchChain(const ChainArgs &a, bool adam, cudaStream_t s)
{
    if (a.n <= 0)
        return;
    { launchPdl(partialSumKernel, std::min(blocks((long long)(a.n + 31) / 32 * 32, 256), 148 * 16), 256, 0, s, 
          a.partial, std::max(a.subSlots, 1), a.subStride, a.offs, a.sortedIds, a.n, a.counts, a.g2d); countLaunch(); }
    if (adam)
        { launchPdl(chainKernel<true>, blocks(a.n, 256), 256, 0, s, a); countLaunch(); }
    else
        { launchPdl(chainKernel<false>, blocks(a.n, 256), 256, 0, s, a); countLaunch(); }
}

void launchAdamSegment(float *p, const float *g, float *m, float *v, int len, float stepSize, float invSqrtBc2,
                       cudaStream_t s)
{
    if (len > 0)
        { adamKernel<<<blocks(len, 256), 256, 0, s>>>(p, g, m, v, len, stepSize, invSqrtBc2); countLaunch(); }
}

void launchDensifyClassify(const Params &P, int n, const float *gradAccum, const int *gradCount, float extent,
                           float splitScale, float pruneOpacity, float gradThreshold, int opacityWasReset, int *keep,
                           int *cost, cudaStream_t s)
{
    { densifyClassifyKernel<<<blocks(n, 256), 256, 0, s>>>(P, n, gradAccum, gradCount, extent, splitScale, pruneOpacity,
                                                         gradThreshold, opacityWasReset, keep, cost); countLaunch(); }
}

void launchDensifySelect(int n, const int *cost, const int *costScan, long long budget, int *firstSecond, int *keep,
                         int *accCost, int *isSplit, cudaStream_t s)
{
    { densifyFirstRejectKernel<<<blocks(n, 256), 256, 0, s>>>(n, cost, costScan, budget, firstSecond); countLaunch(); }
    { densifyLastCloneKernel<<<blocks(n, 256), 256, 0, s>>>(n, cost, costScan, budget, firstSecond, firstSecond + 1); countLaunch(); }
    { densifyAcceptKernel<<<blocks(n, 256), 256, 0, s>>>(n, cost, firstSecond, firstSecond + 1, keep, accCost, isSplit); countLaunch(); }
}

void launchDensifyWrite(const Params &P, const Params &M, const Params &V, const Params &P2, const Params &M2,
                        const Params &V2, int n, const int *keep, const int *keepScan, const int *accCost,
                        const int *accScan, const int *isSplit, const int *splitScan, int keptTotal,
                        const float *normals, float log16, cudaStream_t s)
{
    { densifyWriteKernel<<<blocks(n, 256), 256, 0, s>>>(P, M, V, P2, M2, V2, n, keep, keepScan, accCost, accScan, isSplit,
                                                      splitScan, keptTotal, normals, log16); countLaunch(); }
}

void launchOpacityReset(float *opac, float *mOpac, float *vOpac, int n, float cap, const BinCounts *counts,
                        cudaStream_t s)
{
    if (n > 0)
        { opacityResetKernel<<<blocks(n, 256), 256, 0, s>>>(opac, mOpac, vOpac, n, cap, counts); countLaunch(); }
}

} // namespace u3dg
