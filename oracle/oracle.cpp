// oracle.cpp - CPU restatement of the reference splat trainer. TEST INFRASTRUCTURE ONLY.
//
// This file is the checker for the GPU trainer: only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it (as liboracle.so through ctypes). The product library
// never links or calls it.
//
// It restates, function by function, the algorithm of Abner0907/univeral_3d_reconstruction_system
// engine/src/splat (citations are file:line inside that project). Where the reference's float
// results depend on the order of operations (projection, compositing, SSIM blurs, Adam), the
// same order is kept, and the build uses the reference's flags (-O3, no -march, so no FMA
// contraction), so that with one worker thread the results are bit-identical to the reference
// run with ThreadPool(1). Cross-tile gradient accumulation is done in tile order, which is what
// the reference's CAS atomics produce with a single thread (Rasterizer.cpp:16-21,419-425).
// Multithreading here only splits independent work (tiles, pixels, Gaussians) and keeps every
// reduction in a fixed order, so results do not depend on the thread count.
//
// Parity pin: tests/test_oracle_pin.py compares this file with the reference built from its
// own sources (oracle/_ref) and with the committed fixtures in tests/golden/.

#include "../include/u3dg.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace orc {

// ------------------------------------------------------------------ helpers

constexpr float kShC0 = 0.28209479177387814f; // GaussianModel.h:10
constexpr float kMaxAlpha = 0.99f;            // Rasterizer.cpp:13
constexpr int kG2d = 9;                       // Rasterizer.cpp:14 (dmx dmy dA dB dC dr dg db dalpha)

inline float sigmoidf(float x) { return 1.0f / (1.0f + std::exp(-x)); } // GaussianModel.h:12
inline float logitf(float p) { return std::log(p / (1.0f - p)); }     // GaussianModel.h:13

// Static-chunk parallel for over [0, n) with `threads` workers; fn(begin, end).
void parallel(int threads, int n, const std::function<void(int, int)> &fn)
{
    if (n <= 0)
        return;
    threads = std::max(1, std::min(threads, n));
    if (threads == 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    const int chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e)
            break;
        pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto &th : pool)
        th.join();
}

struct Model {
    std::vector<float> means, scales, quats, opac, colors;
    size_t size() const { return opac.size(); }
    void resize(size_t n)
    {
        means.resize(n * 3);
        scales.resize(n * 3);
        quats.resize(n * 4);
        opac.resize(n);
        colors.resize(n * 3);
    }
    void zero()
    {
        for (auto *v : {&means, &scales, &quats, &opac, &colors})
            std::fill(v->begin(), v->end(), 0.0f);
    }
};

Model fromView(const u3dg_model &m)
{
    Model o;
    o.resize(m.count);
    std::copy(m.means, m.means + 3 * m.count, o.means.begin());
    std::copy(m.scales, m.scales + 3 * m.count, o.scales.begin());
    std::copy(m.quats, m.quats + 4 * m.count, o.quats.begin());
    std::copy(m.opacities, m.opacities + m.count, o.opac.begin());
    std::copy(m.colors, m.colors + 3 * m.count, o.colors.begin());
    return o;
}

void toView(const Model &o, u3dg_model &m)
{
    std::copy(o.means.begin(), o.means.end(), m.means);
    std::copy(o.scales.begin(), o.scales.end(), m.scales);
    std::copy(o.quats.begin(), o.quats.end(), m.quats);
    std::copy(o.opac.begin(), o.opac.end(), m.opacities);
    std::copy(o.colors.begin(), o.colors.end(), m.colors);
}

// ------------------------------------------------------------------ projection

// Quaternion (normalised, w x y z) to row-major rotation; Rasterizer.cpp:24-29.
inline void rotationOf(float w, float x, float y, float z, float R[9])
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

// computeProjection (Rasterizer.cpp:48-110). False when behind the near plane.
bool ewa(const Model &m, size_t i, const u3dg_camera &cam, const u3dg_raster_settings &st, Ewa &p)
{
    const float *mu = &m.means[i * 3];
    const float *R = cam.R;
    p.pc[0] = R[0] * mu[0] + R[1] * mu[1] + R[2] * mu[2] + cam.t[0];
    p.pc[1] = R[3] * mu[0] + R[4] * mu[1] + R[5] * mu[2] + cam.t[1];
    p.pc[2] = R[6] * mu[0] + R[7] * mu[1] + R[8] * mu[2] + cam.t[2];
    const float z = p.pc[2];
    if (z < st.near_plane)
        return false;
    const float *qr = &m.quats[i * 4];
    p.qNorm = std::sqrt(qr[0] * qr[0] + qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
    if (p.qNorm < 1e-12f) {
        p.qNorm = 1.0f;
        p.q[0] = 1;
        p.q[1] = p.q[2] = p.q[3] = 0;
    } else {
        for (int k = 0; k < 4; ++k)
            p.q[k] = qr[k] / p.qNorm;
    }
    rotationOf(p.q[0], p.q[1], p.q[2], p.q[3], p.Rq);
    for (int k = 0; k < 3; ++k)
        p.s[k] = std::exp(m.scales[i * 3 + k]);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            p.M[r * 3 + c] = p.Rq[r * 3 + c] * p.s[c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            p.Sigma[r * 3 + c] = p.M[r * 3] * p.M[c * 3] + p.M[r * 3 + 1] * p.M[c * 3 + 1] + p.M[r * 3 + 2] * p.M[c * 3 + 2];
    const float W = float(cam.width), H = float(cam.height);
    const float limXPos = (W - cam.cx) / cam.fx + 0.3f * 0.5f * W / cam.fx;
    const float limXNeg = cam.cx / cam.fx + 0.3f * 0.5f * W / cam.fx;
    const float limYPos = (H - cam.cy) / cam.fy + 0.3f * 0.5f * H / cam.fy;
    const float limYNeg = cam.cy / cam.fy + 0.3f * 0.5f * H / cam.fy;
    const float xz = p.pc[0] / z, yz = p.pc[1] / z;
    const float cxz = std::min(limXPos, std::max(-limXNeg, xz));
    const float cyz = std::min(limYPos, std::max(-limYNeg, yz));
    p.clampX = cxz != xz;
    p.clampY = cyz != yz;
    p.limTx = cxz;
    p.limTy = cyz;
    p.tx = z * cxz;
    p.ty = z * cyz;
    const float J00 = cam.fx / z, J02 = -cam.fx * p.tx / (z * z);
    const float J11 = cam.fy / z, J12 = -cam.fy * p.ty / (z * z);
    for (int k = 0; k < 3; ++k) {
        p.T0[k] = J00 * R[k] + J02 * R[6 + k];
        p.T1[k] = J11 * R[3 + k] + J12 * R[6 + k];
    }
    float S0[3], S1[3];
    for (int r = 0; r < 3; ++r) {
        S0[r] = p.Sigma[r * 3] * p.T0[0] + p.Sigma[r * 3 + 1] * p.T0[1] + p.Sigma[r * 3 + 2] * p.T0[2];
        S1[r] = p.Sigma[r * 3] * p.T1[0] + p.Sigma[r * 3 + 1] * p.T1[1] + p.Sigma[r * 3 + 2] * p.T1[2];
    }
    p.a = p.T0[0] * S0[0] + p.T0[1] * S0[1] + p.T0[2] * S0[2] + st.eps2d;
    p.b = p.T0[0] * S1[0] + p.T0[1] * S1[1] + p.T0[2] * S1[2];
    p.c = p.T1[0] * S1[0] + p.T1[1] * S1[1] + p.T1[2] * S1[2] + st.eps2d;
    return true;
}

// Real spherical-harmonic colour terms of degree 1..3 in the 3DGS sign convention, evaluated for
// unit direction d; coefficients k = 1..15, channel ch. Returns their sum (no reference counterpart:
// the reference is DC only, Rasterizer.cpp:189-194). The constants are the real-SH normalisations
// sqrt((2l+1)/(4 pi) * (l-|m|)!/(l+|m|)!) (times sqrt(2) for m != 0) folded with the polynomial
// factors.
float shRest(const float *coef, int degree, int ch, const float d[3])
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

// Everything Rasterizer::forward keeps between forward and backward (Rasterizer.h:57-89).
struct Raster {
    u3dg_camera cam{};
    u3dg_raster_settings st{};
    size_t n = 0;
    int tilesX = 0, tilesY = 0;
    std::vector<float> mean2d, conic, cov2d, depth, rgb, alpha;
    std::vector<int> radius, rect;
    std::vector<uint8_t> flags;
    std::vector<int> tileOffsets, tileList;
    std::vector<float> finalT;
    std::vector<int> nContrib;
    std::vector<float> g2d; // last backward's accumulated 2D gradients (n * 9)
    int threads = 1;

    // Rasterizer::project (Rasterizer.cpp:137-204). shRestCoef != null renders SH colours.
    void project(const Model &m, const float *shRestCoef, int shDegree)
    {
        n = m.size();
        mean2d.assign(n * 2, 0.0f);
        conic.assign(n * 3, 0.0f);
        cov2d.assign(n * 3, 0.0f);
        depth.assign(n, 0.0f);
        rgb.assign(n * 3, 0.0f);
        alpha.assign(n, 0.0f);
        radius.assign(n, 0);
        rect.assign(n * 4, 0);
        flags.assign(n, 0);
        const int ts = st.tile_size;
        float camPos[3] = {0, 0, 0};
        if (shRestCoef && shDegree > 0)
            for (int k = 0; k < 3; ++k)
                camPos[k] = -(cam.R[k] * cam.t[0] + cam.R[3 + k] * cam.t[1] + cam.R[6 + k] * cam.t[2]);
        const int K = (shDegree + 1) * (shDegree + 1) - 1;
        parallel(threads, int(n), [&](int b, int e) {
            for (int ii = b; ii < e; ++ii) {
                const size_t i = size_t(ii);
                Ewa p;
                if (!ewa(m, i, cam, st, p))
                    continue;
                const float det = p.a * p.c - p.b * p.b;
                if (!(det > 0.0f))
                    continue;
                const float invDet = 1.0f / det;
                const float z = p.pc[2];
                const float u = cam.fx * p.pc[0] / z + cam.cx;
                const float v = cam.fy * p.pc[1] / z + cam.cy;
                const float mid = 0.5f * (p.a + p.c);
                const float lambda = mid + std::sqrt(std::max(0.1f, mid * mid - det));
                const int r = int(std::ceil(3.0f * std::sqrt(lambda)));
                if (u + r < 0 || v + r < 0 || u - r >= cam.width || v - r >= cam.height)
                    continue;
                const int tx0 = std::max(0, int(std::floor((u - r) / ts)));
                const int ty0 = std::max(0, int(std::floor((v - r) / ts)));
                const int tx1 = std::min(tilesX, int(std::floor((u + r) / ts)) + 1);
                const int ty1 = std::min(tilesY, int(std::floor((v + r) / ts)) + 1);
                if (tx0 >= tx1 || ty0 >= ty1)
                    continue;
                mean2d[i * 2] = u;
                mean2d[i * 2 + 1] = v;
                cov2d[i * 3] = p.a;
                cov2d[i * 3 + 1] = p.b;
                cov2d[i * 3 + 2] = p.c;
                conic[i * 3] = p.c * invDet;
                conic[i * 3 + 1] = -p.b * invDet;
                conic[i * 3 + 2] = p.a * invDet;
                depth[i] = z;
                uint8_t f = uint8_t((p.clampX ? 1 : 0) | (p.clampY ? 2 : 0));
                float dir[3] = {0, 0, 0};
                if (shRestCoef && shDegree > 0) {
                    float dd[3], nrm = 0;
                    for (int k = 0; k < 3; ++k) {
                        dd[k] = m.means[i * 3 + k] - camPos[k];
                        nrm += dd[k] * dd[k];
                    }
                    nrm = std::sqrt(nrm);
                    for (int k = 0; k < 3; ++k)
                        dir[k] = dd[k] / nrm;
                }
                for (int ch = 0; ch < 3; ++ch) {
                    float term = kShC0 * m.colors[i * 3 + ch];
                    if (shRestCoef && shDegree > 0)
                        term = term + shRest(shRestCoef + i * size_t(K) * 3, shDegree, ch, dir);
                    const float col = 0.5f + term;
                    if (col < 0.0f)
                        f |= uint8_t(4 << ch);
                    rgb[i * 3 + ch] = std::max(col, 0.0f);
                }
                flags[i] = f;
                alpha[i] = sigmoidf(m.opac[i]);
                rect[i * 4] = tx0;
                rect[i * 4 + 1] = ty0;
                rect[i * 4 + 2] = tx1;
                rect[i * 4 + 3] = ty1;
                radius[i] = r;
            }
        });
    }

    // Rasterizer::binTiles (Rasterizer.cpp:206-261): visible ids sorted by the float bits of their
    // depth, stable (ties keep index order), then bucketed per tile in that order.
    void binTiles()
    {
        std::vector<int> order;
        order.reserve(n);
        for (size_t i = 0; i < n; ++i)
            if (radius[i] > 0)
                order.push_back(int(i));
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            uint32_t ka, kb;
            std::memcpy(&ka, &depth[size_t(a)], 4);
            std::memcpy(&kb, &depth[size_t(b)], 4);
            return ka < kb;
        });
        const int tiles = tilesX * tilesY;
        tileOffsets.assign(size_t(tiles) + 1, 0);
        for (int g : order) {
            const int *r = &rect[size_t(g) * 4];
            for (int ty = r[1]; ty < r[3]; ++ty)
                for (int tx = r[0]; tx < r[2]; ++tx)
                    ++tileOffsets[size_t(ty * tilesX + tx) + 1];
        }
        for (int t = 0; t < tiles; ++t)
            tileOffsets[size_t(t) + 1] += tileOffsets[size_t(t)];
        tileList.assign(size_t(tileOffsets.back()), 0);
        std::vector<int> cursor(tileOffsets.begin(), tileOffsets.end() - 1);
        for (int g : order) {
            const int *r = &rect[size_t(g) * 4];
            for (int ty = r[1]; ty < r[3]; ++ty)
                for (int tx = r[0]; tx < r[2]; ++tx)
                    tileList[size_t(cursor[size_t(ty * tilesX + tx)]++)] = g;
        }
    }

    void setup(const u3dg_camera &c, const u3dg_raster_settings &s)
    {
        cam = c;
        st = s;
        tilesX = (cam.width + st.tile_size - 1) / st.tile_size;
        tilesY = (cam.height + st.tile_size - 1) / st.tile_size;
    }

    // Per-tile compositing of Rasterizer::forward (Rasterizer.cpp:281-329).
    void composite(std::vector<float> &out)
    {
        const int W = cam.width, H = cam.height, ts = st.tile_size;
        out.assign(size_t(W) * H * 3, 0.0f);
        finalT.assign(size_t(W) * H, 0.0f);
        nContrib.assign(size_t(W) * H, 0);
        const float minA = st.min_alpha, minT = st.min_transmittance;
        const float *bg = st.background;
        parallel(threads, tilesX * tilesY, [&](int b, int e) {
            std::vector<float> rec;
            for (int tile = b; tile < e; ++tile) {
                const int tx = tile % tilesX, ty = tile / tilesX;
                const int first = tileOffsets[size_t(tile)], cnt = tileOffsets[size_t(tile) + 1] - first;
                rec.resize(size_t(cnt) * 9);
                for (int j = 0; j < cnt; ++j) {
                    const size_t g = size_t(tileList[size_t(first + j)]);
                    float *d = &rec[size_t(j) * 9];
                    d[0] = mean2d[g * 2];
                    d[1] = mean2d[g * 2 + 1];
                    d[2] = conic[g * 3];
                    d[3] = conic[g * 3 + 1];
                    d[4] = conic[g * 3 + 2];
                    d[5] = alpha[g];
                    d[6] = rgb[g * 3];
                    d[7] = rgb[g * 3 + 1];
                    d[8] = rgb[g * 3 + 2];
                }
                const int x0 = tx * ts, y0 = ty * ts, x1 = std::min(W, x0 + ts), y1 = std::min(H, y0 + ts);
                for (int py = y0; py < y1; ++py)
                    for (int px = x0; px < x1; ++px) {
                        float T = 1.0f, cr = 0, cg = 0, cb = 0;
                        int last = 0;
                        for (int j = 0; j < cnt; ++j) {
                            const float *d = &rec[size_t(j) * 9];
                            const float dx = d[0] - float(px), dy = d[1] - float(py);
                            const float power = -0.5f * (d[2] * dx * dx + d[4] * dy * dy) - d[3] * dx * dy;
                            if (power > 0.0f)
                                continue;
                            const float a = std::min(kMaxAlpha, d[5] * std::exp(power));
                            if (a < minA)
                                continue;
                            const float nextT = T * (1.0f - a);
                            if (nextT < minT)
                                break;
                            const float w = a * T;
                            cr += d[6] * w;
                            cg += d[7] * w;
                            cb += d[8] * w;
                            T = nextT;
                            last = j + 1;
                        }
                        const size_t pix = size_t(py) * W + px;
                        out[pix * 3] = cr + T * bg[0];
                        out[pix * 3 + 1] = cg + T * bg[1];
                        out[pix * 3 + 2] = cb + T * bg[2];
                        finalT[pix] = T;
                        nContrib[pix] = last;
                    }
            }
        });
    }

    // Rasterizer::forward (Rasterizer.cpp:263-330).
    void forward(const Model &m, const u3dg_camera &c, const u3dg_raster_settings &s, std::vector<float> &out,
                 const float *shRestCoef = nullptr, int shDegree = 0)
    {
        setup(c, s);
        project(m, shRestCoef, shDegree);
        binTiles();
        composite(out);
    }

    // Rasterizer::backward (Rasterizer.cpp:334-545). Adds into grads (and mean2dGradNdc).
    void backward(const Model &m, const float *dLdRgb, Model &grads, float *mean2dGradNdc)
    {
        const int W = cam.width, H = cam.height, ts = st.tile_size;
        const float *bg = st.background;
        const float minA = st.min_alpha;
        const int tiles = tilesX * tilesY;
        // Pass 1 per tile (Rasterizer.cpp:353-418): per-tile accumulators, kept per tile so the
        // cross-tile sum below can run in tile order.
        std::vector<std::vector<float>> accs(static_cast<size_t>(tiles));
        parallel(threads, tiles, [&](int b, int e) {
            std::vector<float> rec;
            for (int tile = b; tile < e; ++tile) {
                const int tx = tile % tilesX, ty = tile / tilesX;
                const int first = tileOffsets[size_t(tile)], cnt = tileOffsets[size_t(tile) + 1] - first;
                if (cnt == 0)
                    continue;
                rec.resize(size_t(cnt) * 9);
                std::vector<float> &acc = accs[size_t(tile)];
                acc.assign(size_t(cnt) * kG2d, 0.0f);
                for (int j = 0; j < cnt; ++j) {
                    const size_t g = size_t(tileList[size_t(first + j)]);
                    float *d = &rec[size_t(j) * 9];
                    d[0] = mean2d[g * 2];
                    d[1] = mean2d[g * 2 + 1];
                    d[2] = conic[g * 3];
                    d[3] = conic[g * 3 + 1];
                    d[4] = conic[g * 3 + 2];
                    d[5] = alpha[g];
                    d[6] = rgb[g * 3];
                    d[7] = rgb[g * 3 + 1];
                    d[8] = rgb[g * 3 + 2];
                }
                const int x0 = tx * ts, y0 = ty * ts, x1 = std::min(W, x0 + ts), y1 = std::min(H, y0 + ts);
                for (int py = y0; py < y1; ++py)
                    for (int px = x0; px < x1; ++px) {
                        const size_t pix = size_t(py) * W + px;
                        const float *dp = &dLdRgb[pix * 3];
                        const float fT = finalT[pix];
                        const float bgDot = bg[0] * dp[0] + bg[1] * dp[1] + bg[2] * dp[2];
                        float T = fT;
                        float accum[3] = {0, 0, 0}, lastColor[3] = {0, 0, 0};
                        float lastAlpha = 0;
                        for (int j = nContrib[pix] - 1; j >= 0; --j) {
                            const float *d = &rec[size_t(j) * 9];
                            const float dx = d[0] - float(px), dy = d[1] - float(py);
                            const float power = -0.5f * (d[2] * dx * dx + d[4] * dy * dy) - d[3] * dx * dy;
                            if (power > 0.0f)
                                continue;
                            const float G = std::exp(power);
                            const float raw = d[5] * G;
                            const float a = std::min(kMaxAlpha, raw);
                            if (a < minA)
                                continue;
                            T = T / (1.0f - a);
                            const float w = a * T;
                            float *o = &acc[size_t(j) * kG2d];
                            float dA = 0.0f;
                            for (int ch = 0; ch < 3; ++ch) {
                                accum[ch] = lastAlpha * lastColor[ch] + (1.0f - lastAlpha) * accum[ch];
                                lastColor[ch] = d[6 + ch];
                                dA += (d[6 + ch] - accum[ch]) * dp[ch];
                                o[5 + ch] += w * dp[ch];
                            }
                            dA *= T;
                            lastAlpha = a;
                            dA += -fT / (1.0f - a) * bgDot;
                            if (raw > kMaxAlpha)
                                continue;
                            o[8] += G * dA;
                            const float dPow = d[5] * dA * G;
                            o[0] += dPow * -(d[2] * dx + d[3] * dy);
                            o[1] += dPow * -(d[4] * dy + d[3] * dx);
                            o[2] += dPow * -0.5f * dx * dx;
                            o[3] += dPow * -dx * dy;
                            o[4] += dPow * -0.5f * dy * dy;
                        }
                    }
            }
        });
        // Cross-tile sum in tile order (Rasterizer.cpp:419-425 with one thread).
        g2d.assign(n * kG2d, 0.0f);
        for (int tile = 0; tile < tiles; ++tile) {
            const std::vector<float> &acc = accs[size_t(tile)];
            if (acc.empty())
                continue;
            const int first = tileOffsets[size_t(tile)], cnt = tileOffsets[size_t(tile) + 1] - first;
            for (int j = 0; j < cnt; ++j) {
                float *dst = &g2d[size_t(tileList[size_t(first + j)]) * kG2d];
                for (int k = 0; k < kG2d; ++k)
                    if (acc[size_t(j) * kG2d + k] != 0.0f)
                        dst[k] += acc[size_t(j) * kG2d + k];
            }
        }
        // Pass 2 per Gaussian (Rasterizer.cpp:432-544).
        parallel(threads, int(n), [&](int b, int e) {
            for (int ii = b; ii < e; ++ii) {
                const size_t i = size_t(ii);
                if (radius[i] == 0)
                    continue;
                const float *g = &g2d[i * kG2d];
                const float dmx = g[0], dmy = g[1], dA = g[2], dB = g[3], dC = g[4];
                if (mean2dGradNdc) {
                    const float nx = dmx * 0.5f * float(cam.width), ny = dmy * 0.5f * float(cam.height);
                    mean2dGradNdc[i] += std::sqrt(nx * nx + ny * ny);
                }
                for (int ch = 0; ch < 3; ++ch)
                    if (!(flags[i] & (4 << ch)))
                        grads.colors[i * 3 + ch] += kShC0 * g[5 + ch];
                const float op = alpha[i];
                grads.opac[i] += g[8] * op * (1.0f - op);
                Ewa p;
                ewa(m, i, cam, st, p);
                const float z = p.pc[2];
                const float a = p.a, bb = p.b, c = p.c;
                const float det = a * c - bb * bb;
                const float det2 = det * det;
                const float da = (dA * -c * c + dB * bb * c + dC * -bb * bb) / det2;
                const float db = (dA * 2 * bb * c + dC * 2 * a * bb) / det2 + dB * (-1.0f / det - 2 * bb * bb / det2);
                const float dc = (dA * -bb * bb + dB * a * bb + dC * -a * a) / det2;
                const float G00 = da, G01 = 0.5f * db, G11 = dc;
                float dSigma[9];
                for (int k = 0; k < 3; ++k)
                    for (int l = 0; l < 3; ++l)
                        dSigma[k * 3 + l] = p.T0[k] * (G00 * p.T0[l] + G01 * p.T1[l]) + p.T1[k] * (G01 * p.T0[l] + G11 * p.T1[l]);
                float TS0[3], TS1[3];
                for (int col = 0; col < 3; ++col) {
                    TS0[col] = p.T0[0] * p.Sigma[col] + p.T0[1] * p.Sigma[3 + col] + p.T0[2] * p.Sigma[6 + col];
                    TS1[col] = p.T1[0] * p.Sigma[col] + p.T1[1] * p.Sigma[3 + col] + p.T1[2] * p.Sigma[6 + col];
                }
                float dT0[3], dT1[3];
                for (int col = 0; col < 3; ++col) {
                    dT0[col] = 2.0f * (G00 * TS0[col] + G01 * TS1[col]);
                    dT1[col] = 2.0f * (G01 * TS0[col] + G11 * TS1[col]);
                }
                float dM[9];
                for (int r = 0; r < 3; ++r)
                    for (int col = 0; col < 3; ++col)
                        dM[r * 3 + col] = 2.0f * (dSigma[r * 3] * p.M[col] + dSigma[r * 3 + 1] * p.M[3 + col] + dSigma[r * 3 + 2] * p.M[6 + col]);
                float dRq[9];
                for (int col = 0; col < 3; ++col) {
                    float ds = 0;
                    for (int r = 0; r < 3; ++r) {
                        ds += dM[r * 3 + col] * p.Rq[r * 3 + col];
                        dRq[r * 3 + col] = dM[r * 3 + col] * p.s[col];
                    }
                    grads.scales[i * 3 + col] += ds * p.s[col];
                }
                const float w = p.q[0], x = p.q[1], y = p.q[2], zq = p.q[3];
                const float dw = 2 * (-zq * dRq[1] + y * dRq[2] + zq * dRq[3] - x * dRq[5] - y * dRq[6] + x * dRq[7]);
                const float dx = 2 * (y * dRq[1] + zq * dRq[2] + y * dRq[3] - 2 * x * dRq[4] - w * dRq[5] + zq * dRq[6] + w * dRq[7] - 2 * x * dRq[8]);
                const float dy = 2 * (-2 * y * dRq[0] + x * dRq[1] + w * dRq[2] + x * dRq[3] + zq * dRq[5] - w * dRq[6] + zq * dRq[7] - 2 * y * dRq[8]);
                const float dz = 2 * (-2 * zq * dRq[0] - w * dRq[1] + x * dRq[2] + w * dRq[3] - 2 * zq * dRq[4] + y * dRq[5] + x * dRq[6] + y * dRq[7]);
                const float dq[4] = {dw, dx, dy, dz};
                const float qdot = dq[0] * p.q[0] + dq[1] * p.q[1] + dq[2] * p.q[2] + dq[3] * p.q[3];
                for (int k = 0; k < 4; ++k)
                    grads.quats[i * 4 + k] += (dq[k] - qdot * p.q[k]) / p.qNorm;
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
                for (int k = 0; k < 3; ++k)
                    grads.means[i * 3 + k] += R[k] * dpc[0] + R[3 + k] * dpc[1] + R[6 + k] * dpc[2];
            }
        });
    }
};

// ------------------------------------------------------------------ loss (Loss.cpp)

constexpr int kWin = 5; // Loss.cpp:11, 11x11 window

struct Window {
    float w[2 * kWin + 1];
    Window()
    {
        float sum = 0;
        for (int k = -kWin; k <= kWin; ++k) {
            w[k + kWin] = std::exp(-float(k * k) / (2.0f * 1.5f * 1.5f));
            sum += w[k + kWin];
        }
        for (float &v : w)
            v /= sum;
    }
};

// photometricLoss (Loss.cpp:47-184), four separable passes; double partial sums taken per chunk of
// 4 (channel, row) pairs in order, as the reference's parallelFor(rows, ..., 4) does with one thread.
u3dg_loss_value photometricLoss(const float *render, const float *target, int W, int H, float lambda, float *grad)
{
    static const Window win;
    const float *wk = win.w;
    const size_t P = size_t(W) * H;
    const float invCount = 1.0f / float(P * 3);
    const int rows = 3 * H;
    std::vector<float> h[5], abc[3], h2[3];
    for (auto &v : h)
        v.assign(3 * P, 0.0f);
    for (auto &v : abc)
        v.assign(3 * P, 0.0f);
    for (auto &v : h2)
        v.assign(3 * P, 0.0f);
    double l1Total = 0;
    for (int r0 = 0; r0 < rows; r0 += 4) {
        double l1 = 0;
        for (int r = r0; r < std::min(rows, r0 + 4); ++r) {
            const int c = r / H, y = r % H;
            const size_t base = size_t(c) * P + size_t(y) * W;
            for (int x = 0; x < W; ++x) {
                const size_t idx = (size_t(y) * W + x) * 3 + size_t(c);
                const float d = render[idx] - target[idx];
                l1 += std::fabs(d);
                grad[idx] = (1.0f - lambda) * invCount * (d > 0 ? 1.0f : (d < 0 ? -1.0f : 0.0f));
            }
            if (lambda <= 0.0f)
                continue;
            for (int x = 0; x < W; ++x) {
                float sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
                const int k0 = std::max(-kWin, -x), k1 = std::min(kWin, W - 1 - x);
                for (int k = k0; k <= k1; ++k) {
                    const size_t idx = (size_t(y) * W + size_t(x + k)) * 3 + size_t(c);
                    const float a = render[idx], b = target[idx], w = wk[k + kWin];
                    sx += w * a;
                    sy += w * b;
                    sxx += w * a * a;
                    syy += w * b * b;
                    sxy += w * a * b;
                }
                h[0][base + x] = sx;
                h[1][base + x] = sy;
                h[2][base + x] = sxx;
                h[3][base + x] = syy;
                h[4][base + x] = sxy;
            }
        }
        l1Total += l1;
    }
    u3dg_loss_value res{};
    res.l1 = float(l1Total * invCount);
    if (lambda <= 0.0f) {
        res.total = res.l1;
        return res;
    }
    const float kC1 = 0.01f * 0.01f, kC2 = 0.03f * 0.03f;
    const float dLds = -lambda * invCount;
    double ssimTotal = 0;
    for (int r0 = 0; r0 < rows; r0 += 4) {
        double ssim = 0;
        for (int r = r0; r < std::min(rows, r0 + 4); ++r) {
            const int c = r / H, y = r % H;
            const size_t cbase = size_t(c) * P;
            const int k0 = std::max(-kWin, -y), k1 = std::min(kWin, H - 1 - y);
            for (int x = 0; x < W; ++x) {
                float mm[5] = {0, 0, 0, 0, 0};
                for (int k = k0; k <= k1; ++k) {
                    const size_t i = cbase + size_t(y + k) * W + x;
                    const float w = wk[k + kWin];
                    for (int j = 0; j < 5; ++j)
                        mm[j] += w * h[j][i];
                }
                const float mx = mm[0], my = mm[1];
                const float sx = mm[2] - mx * mx, sy = mm[3] - my * my, sxy = mm[4] - mx * my;
                const float a1 = 2 * mx * my + kC1, a2 = 2 * sxy + kC2;
                const float b1 = mx * mx + my * my + kC1, b2 = sx + sy + kC2;
                const float v = (a1 * a2) / (b1 * b2);
                ssim += v;
                const float dmu = (2 * my * a2 - 2 * my * a1) / (b1 * b2) - v * (2 * mx / b1 - 2 * mx / b2);
                const size_t o = cbase + size_t(y) * W + x;
                abc[0][o] = dLds * dmu;
                abc[1][o] = dLds * (-v / b2);
                abc[2][o] = dLds * (2 * a1 / (b1 * b2));
            }
        }
        ssimTotal += ssim;
    }
    for (int r = 0; r < rows; ++r) {
        const size_t base = size_t(r / H) * P + size_t(r % H) * W;
        for (int x = 0; x < W; ++x) {
            float acc[3] = {0, 0, 0};
            const int k0 = std::max(-kWin, -x), k1 = std::min(kWin, W - 1 - x);
            for (int k = k0; k <= k1; ++k) {
                const float w = wk[k + kWin];
                for (int j = 0; j < 3; ++j)
                    acc[j] += w * abc[j][base + size_t(x + k)];
            }
            for (int j = 0; j < 3; ++j)
                h2[j][base + x] = acc[j];
        }
    }
    for (int r = 0; r < rows; ++r) {
        const int c = r / H, y = r % H;
        const size_t cbase = size_t(c) * P;
        const int k0 = std::max(-kWin, -y), k1 = std::min(kWin, H - 1 - y);
        for (int x = 0; x < W; ++x) {
            float g[3] = {0, 0, 0};
            for (int k = k0; k <= k1; ++k) {
                const size_t i = cbase + size_t(y + k) * W + x;
                const float w = wk[k + kWin];
                for (int j = 0; j < 3; ++j)
                    g[j] += w * h2[j][i];
            }
            const size_t idx = (size_t(y) * W + x) * 3 + size_t(c);
            grad[idx] += g[0] + 2.0f * render[idx] * g[1] + target[idx] * g[2];
        }
    }
    res.ssim = float(ssimTotal * invCount);
    res.total = (1.0f - lambda) * res.l1 + lambda * (1.0f - res.ssim);
    return res;
}

// psnr (Loss.cpp:187-196).
float psnr(const float *a, const float *b, size_t count)
{
    double mse = 0;
    for (size_t k = 0; k < count; ++k) {
        const double d = double(a[k]) - double(b[k]);
        mse += d * d;
    }
    mse /= double(std::max<size_t>(count, 1));
    return mse <= 1e-12 ? 99.0f : float(-10.0 * std::log10(mse));
}

// ------------------------------------------------------------------ Adam (Adam.cpp)

struct Adam {
    Model m, v;
    int step = 0;
    void reset(size_t n)
    {
        m.resize(n);
        v.resize(n);
        m.zero();
        v.zero();
        step = 0;
    }
    // adamArray (Adam.cpp:13-28).
    static void update(std::vector<float> &p, const std::vector<float> &g, std::vector<float> &mm, std::vector<float> &vv,
                       float lr, float bc1, float bc2)
    {
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-15f;
        const float stepSize = lr / bc1;
        const float invSqrtBc2 = 1.0f / std::sqrt(bc2);
        for (size_t k = 0; k < p.size(); ++k) {
            const float gk = g[k];
            mm[k] = b1 * mm[k] + (1.0f - b1) * gk;
            vv[k] = b2 * vv[k] + (1.0f - b2) * gk * gk;
            p[k] -= stepSize * mm[k] / (std::sqrt(vv[k]) * invSqrtBc2 + eps);
        }
    }
    // Adam::step (Adam.cpp:68-78).
    void apply(Model &p, const Model &g, const u3dg_learning_rates &lr)
    {
        ++step;
        const float bc1 = 1.0f - std::pow(0.9f, float(step));
        const float bc2 = 1.0f - std::pow(0.999f, float(step));
        update(p.means, g.means, m.means, v.means, lr.means, bc1, bc2);
        update(p.scales, g.scales, m.scales, v.scales, lr.scales, bc1, bc2);
        update(p.quats, g.quats, m.quats, v.quats, lr.quats, bc1, bc2);
        update(p.opac, g.opac, m.opac, v.opac, lr.opacities, bc1, bc2);
        update(p.colors, g.colors, m.colors, v.colors, lr.colors, bc1, bc2);
    }
};

// GaussianModel::compact (GaussianModel.cpp:50-57): keep order, drop keep[i] == 0.
void compact(Model &m, const std::vector<uint8_t> &keep)
{
    auto one = [&](std::vector<float> &v, int dim) {
        size_t out = 0;
        for (size_t i = 0; i < keep.size(); ++i) {
            if (!keep[i])
                continue;
            if (out != i)
                std::copy_n(&v[i * dim], dim, &v[out * dim]);
            ++out;
        }
        v.resize(out * dim);
    };
    one(m.means, 3);
    one(m.scales, 3);
    one(m.quats, 4);
    one(m.opac, 1);
    one(m.colors, 3);
}

// GaussianModel::appendFrom (GaussianModel.cpp:59-66).
void append(Model &dst, const Model &src, size_t i)
{
    dst.means.insert(dst.means.end(), src.means.begin() + i * 3, src.means.begin() + i * 3 + 3);
    dst.scales.insert(dst.scales.end(), src.scales.begin() + i * 3, src.scales.begin() + i * 3 + 3);
    dst.quats.insert(dst.quats.end(), src.quats.begin() + i * 4, src.quats.begin() + i * 4 + 4);
    dst.opac.push_back(src.opac[i]);
    dst.colors.insert(dst.colors.end(), src.colors.begin() + i * 3, src.colors.begin() + i * 3 + 3);
}

// Adam::grow (Adam.cpp:46-60): zero moments for new entries.
void growZero(Model &m, size_t count)
{
    const size_t n = m.size();
    m.resize(n + count);
    std::fill(m.means.begin() + n * 3, m.means.end(), 0.0f);
    std::fill(m.scales.begin() + n * 3, m.scales.end(), 0.0f);
    std::fill(m.quats.begin() + n * 4, m.quats.end(), 0.0f);
    std::fill(m.opac.begin() + n, m.opac.end(), 0.0f);
    std::fill(m.colors.begin() + n * 3, m.colors.end(), 0.0f);
}

// Trainer::densifyAndPrune (Trainer.cpp:105-169). Returns {pruned, clones, splits}.
struct DensifyCounts {
    int pruned = 0, clones = 0, splits = 0;
};

DensifyCounts densifyAndPrune(Model &model, Adam &adam, std::vector<float> &gradAccum, std::vector<int> &gradCount,
                              float extent, const u3dg_train_options &o, bool opacityWasReset, std::mt19937 &rng)
{
    DensifyCounts counts;
    const size_t n = model.size();
    const float splitScale = o.percent_dense * extent;
    const size_t budget = o.max_gaussians > int(n) ? size_t(o.max_gaussians) - n : 0;
    std::vector<uint8_t> keep(n, 1);
    Model extra;
    size_t added = 0;
    std::normal_distribution<float> normal(0.0f, 1.0f);
    for (size_t i = 0; i < n; ++i) {
        const float maxLog = std::max({model.scales[i * 3], model.scales[i * 3 + 1], model.scales[i * 3 + 2]});
        const float maxScale = std::exp(maxLog);
        const float a = sigmoidf(model.opac[i]);
        if (a < o.prune_opacity || (opacityWasReset && maxScale > 0.1f * extent)) {
            keep[i] = 0;
            ++counts.pruned;
            continue;
        }
        if (gradCount[i] == 0)
            continue;
        const float avg = gradAccum[i] / float(gradCount[i]);
        if (avg < o.densify_grad_threshold)
            continue;
        if (maxScale <= splitScale) {
            if (added + 1 > budget)
                continue;
            append(extra, model, i);
            added += 1;
            ++counts.clones;
        } else {
            if (added + 2 > budget)
                continue;
            const float *q = &model.quats[i * 4];
            const float qn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + 1e-12f;
            float R[9];
            rotationOf(q[0] / qn, q[1] / qn, q[2] / qn, q[3] / qn, R);
            for (int c = 0; c < 2; ++c) {
                const size_t j = extra.size();
                append(extra, model, i);
                float local[3];
                for (int k = 0; k < 3; ++k)
                    local[k] = normal(rng) * std::exp(model.scales[i * 3 + k]);
                for (int r = 0; r < 3; ++r)
                    extra.means[j * 3 + r] += R[r * 3] * local[0] + R[r * 3 + 1] * local[1] + R[r * 3 + 2] * local[2];
                for (int k = 0; k < 3; ++k)
                    extra.scales[j * 3 + k] -= std::log(1.6f);
            }
            keep[i] = 0;
            added += 2;
            ++counts.splits;
        }
    }
    compact(model, keep);
    compact(adam.m, keep);
    compact(adam.v, keep);
    for (size_t j = 0; j < extra.size(); ++j)
        append(model, extra, j);
    growZero(adam.m, extra.size());
    growZero(adam.v, extra.size());
    gradAccum.assign(model.size(), 0.0f);
    gradCount.assign(model.size(), 0);
    return counts;
}

// ------------------------------------------------------------------ Trainer (Trainer.cpp)

struct Trainer {
    Model model, grads;
    std::vector<u3dg_camera> cams;
    std::vector<std::vector<uint8_t>> images;
    float extent;
    u3dg_train_options o;
    Raster raster;
    Adam adam;
    std::mt19937 rng;
    std::vector<int> order;
    size_t orderPos = 0;
    int iteration = 0;
    bool opacityWasReset = false;
    std::vector<float> target, render, dLoss, gradAccum;
    std::vector<int> gradCount;
    u3dg_train_stats stats{};
    std::vector<int> viewLog; // view index used by every step, for tests

    Trainer(Model init, const u3dg_image *imgs, int count, float sceneExtent, const u3dg_train_options &opt, int threads)
        : model(std::move(init)), extent(std::max(sceneExtent, 1e-6f)), o(opt), rng(opt.seed)
    {
        raster.threads = threads;
        for (int k = 0; k < count; ++k) {
            cams.push_back(imgs[k].camera);
            const size_t sz = size_t(imgs[k].camera.width) * imgs[k].camera.height * 3;
            images.emplace_back(imgs[k].rgb, imgs[k].rgb + sz);
        }
        adam.reset(model.size());
        gradAccum.assign(model.size(), 0.0f);
        gradCount.assign(model.size(), 0);
        stats.gaussians = model.size();
    }

    bool done() const { return iteration >= o.iterations; }

    // Trainer::loadTarget (Trainer.cpp:18-24).
    void loadTarget(size_t v)
    {
        const std::vector<uint8_t> &img = images[v];
        target.resize(img.size());
        const float inv = 1.0f / 255.0f;
        for (size_t k = 0; k < img.size(); ++k)
            target[k] = float(img[k]) * inv;
    }

    // Trainer::step (Trainer.cpp:53-103).
    void step()
    {
        if (images.empty() || done())
            return;
        if (orderPos >= order.size()) {
            order.resize(images.size());
            for (size_t k = 0; k < order.size(); ++k)
                order[k] = int(k);
            std::shuffle(order.begin(), order.end(), rng);
            orderPos = 0;
        }
        const size_t v = size_t(order[orderPos++]);
        viewLog.push_back(int(v));
        const u3dg_camera &cam = cams[v];
        loadTarget(v);
        raster.forward(model, cam, o.raster, render);
        dLoss.resize(render.size());
        const u3dg_loss_value loss = photometricLoss(render.data(), target.data(), cam.width, cam.height, o.ssim_lambda, dLoss.data());
        grads.resize(model.size());
        grads.zero();
        raster.backward(model, dLoss.data(), grads, gradAccum.data());
        for (size_t i = 0; i < raster.radius.size(); ++i)
            if (raster.radius[i] > 0)
                ++gradCount[i];
        u3dg_learning_rates lr = o.lr;
        const float t = float(iteration) / float(std::max(1, o.iterations - 1));
        lr.means = std::exp(std::log(o.lr.means) * (1 - t) + std::log(o.means_lr_final) * t) * extent;
        adam.apply(model, grads, lr);
        ++iteration;
        const float p = psnr(render.data(), target.data(), render.size());
        const float k = stats.iteration == 0 ? 1.0f : 0.05f;
        stats.loss += k * (loss.total - stats.loss);
        stats.psnr += k * (p - stats.psnr);
        stats.iteration = iteration;
        if (iteration >= o.refine_start && iteration < o.refine_stop && iteration % o.refine_interval == 0)
            densifyAndPrune(model, adam, gradAccum, gradCount, extent, o, opacityWasReset, rng);
        if (o.opacity_reset_interval > 0 && iteration < o.refine_stop && iteration % o.opacity_reset_interval == 0)
            resetOpacity();
        stats.gaussians = model.size();
    }

    // Trainer::resetOpacity (Trainer.cpp:171-178).
    void resetOpacity()
    {
        const float cap = logitf(0.01f);
        for (float &x : model.opac)
            x = std::min(x, cap);
        std::fill(adam.m.opac.begin(), adam.m.opac.end(), 0.0f);
        std::fill(adam.v.opac.begin(), adam.v.opac.end(), 0.0f);
        opacityWasReset = true;
    }

    // Trainer::evaluatePsnr (Trainer.cpp:180-192).
    float evaluatePsnr()
    {
        if (images.empty())
            return 0;
        double sum = 0;
        std::vector<float> rgb;
        for (size_t v = 0; v < images.size(); ++v) {
            loadTarget(v);
            raster.forward(model, cams[v], o.raster, rgb);
            sum += psnr(rgb.data(), target.data(), rgb.size());
        }
        return float(sum / double(images.size()));
    }
};

// ------------------------------------------------------------------ initGaussiansFromPoints

// initGaussiansFromPoints (GaussianModel.cpp:68-144): uniform hash grid (cell = 2 extent / cbrt n),
// 3 nearest neighbours among the 27 surrounding cells, isotropic log-scale log sqrt(mean d^2).
Model initFromPoints(const float *xyz, const float *rgb, size_t n)
{
    Model m;
    m.resize(n);
    if (n == 0)
        return m;
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = std::numeric_limits<float>::max();
        hi[k] = -lo[k];
    }
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], xyz[i * 3 + k]);
            hi[k] = std::max(hi[k], xyz[i * 3 + k]);
        }
    const float ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-6f});
    const float cell = std::max(ext / std::cbrt(float(n)) * 2.0f, 1e-6f);
    auto key = [](int x, int y, int z) {
        return (int64_t(x) * 73856093) ^ (int64_t(y) * 19349663) ^ (int64_t(z) * 83492791);
    };
    auto cellOf = [&](size_t i, int c[3]) {
        for (int k = 0; k < 3; ++k)
            c[k] = int(std::floor((xyz[i * 3 + k] - lo[k]) / cell));
    };
    std::unordered_map<int64_t, std::vector<uint32_t>> grid;
    grid.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        int c[3];
        cellOf(i, c);
        grid[key(c[0], c[1], c[2])].push_back(uint32_t(i));
    }
    const float fmax = std::numeric_limits<float>::max();
    for (size_t i = 0; i < n; ++i) {
        float best[3] = {fmax, fmax, fmax};
        int c[3];
        cellOf(i, c);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = grid.find(key(c[0] + dx, c[1] + dy, c[2] + dz));
                    if (it == grid.end())
                        continue;
                    for (uint32_t j : it->second) {
                        if (j == i)
                            continue;
                        const float ex = xyz[j * 3] - xyz[i * 3], ey = xyz[j * 3 + 1] - xyz[i * 3 + 1], ez = xyz[j * 3 + 2] - xyz[i * 3 + 2];
                        float d2 = ex * ex + ey * ey + ez * ez;
                        for (int k = 0; k < 3; ++k)
                            if (d2 < best[k])
                                std::swap(d2, best[k]);
                    }
                }
        float sum = 0;
        int cnt = 0;
        for (float b : best)
            if (b < fmax) {
                sum += b;
                ++cnt;
            }
        const float meanD2 = cnt ? sum / float(cnt) : cell * cell;
        const float logScale = std::log(std::sqrt(std::max(meanD2, 1e-14f)));
        for (int k = 0; k < 3; ++k) {
            m.means[i * 3 + k] = xyz[i * 3 + k];
            m.scales[i * 3 + k] = logScale;
            const float col = rgb ? rgb[i * 3 + k] : 0.5f;
            m.colors[i * 3 + k] = (col - 0.5f) / kShC0;
        }
        m.quats[i * 4] = 1.0f;
        m.quats[i * 4 + 1] = m.quats[i * 4 + 2] = m.quats[i * 4 + 3] = 0.0f;
        m.opac[i] = logitf(0.1f);
    }
    return m;
}

} // namespace orc

// ------------------------------------------------------------------ C ABI for ctypes

using namespace orc;

extern "C" {

struct orc_raster {
    Raster r;
    Model model;
};

orc_raster *orc_raster_create(int threads)
{
    auto *o = new orc_raster();
    o->r.threads = std::max(1, threads);
    return o;
}

void orc_raster_destroy(orc_raster *o) { delete o; }

// Rasterizer::forward with optional SH colours (sh_rest may be NULL).
void orc_raster_forward(orc_raster *o, const u3dg_model *m, const float *sh_rest, int degree, const u3dg_camera *cam,
                        const u3dg_raster_settings *st, float *rgb)
{
    o->model = fromView(*m);
    std::vector<float> out;
    o->r.forward(o->model, *cam, *st, out, sh_rest, degree);
    std::copy(out.begin(), out.end(), rgb);
}

// Projection only (no binning), for projection-level comparisons.
void orc_raster_project(orc_raster *o, const u3dg_model *m, const u3dg_camera *cam, const u3dg_raster_settings *st)
{
    o->model = fromView(*m);
    o->r.setup(*cam, *st);
    o->r.project(o->model, nullptr, 0);
}

// Rasterizer::binTiles on explicitly given projected records.
void orc_bin_tiles(const float *depth, const int *radius, const int *rect, size_t n, int tiles_x, int tiles_y,
                   int *offsets, int *list, size_t list_capacity, size_t *list_length)
{
    Raster r;
    r.n = n;
    r.tilesX = tiles_x;
    r.tilesY = tiles_y;
    r.depth.assign(depth, depth + n);
    r.radius.assign(radius, radius + n);
    r.rect.assign(rect, rect + 4 * n);
    r.binTiles();
    std::copy(r.tileOffsets.begin(), r.tileOffsets.end(), offsets);
    *list_length = r.tileList.size();
    std::copy_n(r.tileList.begin(), std::min(list_capacity, r.tileList.size()), list);
}

void orc_raster_backward(orc_raster *o, const float *dl_drgb, u3dg_model *grads, float *mean2d_grad_ndc)
{
    Model g = fromView(*grads);
    o->r.backward(o->model, dl_drgb, g, mean2d_grad_ndc);
    toView(g, *grads);
}

void orc_raster_projection(orc_raster *o, float *mean2d, float *conic, float *cov2d, float *depth, float *rgb, float *alpha,
                           int *radius, int *rect, uint8_t *flags)
{
    const Raster &r = o->r;
    if (mean2d) std::copy(r.mean2d.begin(), r.mean2d.end(), mean2d);
    if (conic) std::copy(r.conic.begin(), r.conic.end(), conic);
    if (cov2d) std::copy(r.cov2d.begin(), r.cov2d.end(), cov2d);
    if (depth) std::copy(r.depth.begin(), r.depth.end(), depth);
    if (rgb) std::copy(r.rgb.begin(), r.rgb.end(), rgb);
    if (alpha) std::copy(r.alpha.begin(), r.alpha.end(), alpha);
    if (radius) std::copy(r.radius.begin(), r.radius.end(), radius);
    if (rect) std::copy(r.rect.begin(), r.rect.end(), rect);
    if (flags) std::copy(r.flags.begin(), r.flags.end(), flags);
}

size_t orc_raster_list_length(orc_raster *o) { return o->r.tileList.size(); }

void orc_raster_tiles(orc_raster *o, int *offsets, int *list)
{
    std::copy(o->r.tileOffsets.begin(), o->r.tileOffsets.end(), offsets);
    std::copy(o->r.tileList.begin(), o->r.tileList.end(), list);
}

void orc_raster_pixel_state(orc_raster *o, float *final_t, int *n_contrib)
{
    std::copy(o->r.finalT.begin(), o->r.finalT.end(), final_t);
    std::copy(o->r.nContrib.begin(), o->r.nContrib.end(), n_contrib);
}

void orc_raster_g2d(orc_raster *o, float *g2d) { std::copy(o->r.g2d.begin(), o->r.g2d.end(), g2d); }

void orc_photometric_loss(const float *render, const float *target, int w, int h, float lambda, float *grad, u3dg_loss_value *out)
{
    *out = photometricLoss(render, target, w, h, lambda, grad);
}

float orc_psnr(const float *a, const float *b, size_t count) { return psnr(a, b, count); }

// One Adam::step over given moments (all host arrays, updated in place); step = the new step count.
void orc_adam_step(u3dg_model *params, const u3dg_model *grads, u3dg_model *m, u3dg_model *v, int step,
                   const u3dg_learning_rates *lr)
{
    Adam a;
    a.m = fromView(*m);
    a.v = fromView(*v);
    a.step = step - 1;
    Model p = fromView(*params), g = fromView(*grads);
    a.apply(p, g, *lr);
    toView(p, *params);
    toView(a.m, *m);
    toView(a.v, *v);
}

// Trainer::densifyAndPrune on a given state with an mt19937 seeded by `seed`. model/m/v are
// resized: capacity must hold max_gaussians; *count gets the new size. counts (3 ints) gets
// pruned, clones, splits.
void orc_densify(u3dg_model *model, u3dg_model *m, u3dg_model *v, float *grad_accum, int *grad_count, size_t capacity,
                 float extent, const u3dg_train_options *o, int opacity_was_reset, unsigned seed, size_t *count, int *counts)
{
    Model md = fromView(*model);
    Adam a;
    a.m = fromView(*m);
    a.v = fromView(*v);
    std::vector<float> acc(grad_accum, grad_accum + model->count);
    std::vector<int> cnt(grad_count, grad_count + model->count);
    std::mt19937 rng(seed);
    DensifyCounts c = densifyAndPrune(md, a, acc, cnt, extent, *o, opacity_was_reset != 0, rng);
    *count = md.size();
    counts[0] = c.pruned;
    counts[1] = c.clones;
    counts[2] = c.splits;
    if (md.size() > capacity)
        return;
    toView(md, *model);
    toView(a.m, *m);
    toView(a.v, *v);
}

Trainer *orc_trainer_create(const u3dg_model *initial, const u3dg_image *images, int count, float extent,
                            const u3dg_train_options *o, int threads)
{
    return new Trainer(fromView(*initial), images, count, extent, *o, std::max(1, threads));
}

void orc_trainer_step(Trainer *t, int count)
{
    for (int k = 0; k < count; ++k)
        t->step();
}

void orc_trainer_stats(Trainer *t, u3dg_train_stats *out) { *out = t->stats; }
size_t orc_trainer_size(Trainer *t) { return t->model.size(); }
int orc_trainer_iteration(Trainer *t) { return t->iteration; }
void orc_trainer_download(Trainer *t, u3dg_model *out) { toView(t->model, *out); }
float orc_trainer_eval_psnr(Trainer *t) { return t->evaluatePsnr(); }
void orc_trainer_destroy(Trainer *t) { delete t; }
int orc_trainer_view_log(Trainer *t, int *out, int capacity)
{
    const int n = int(t->viewLog.size());
    for (int k = 0; k < std::min(n, capacity); ++k)
        out[k] = t->viewLog[size_t(k)];
    return n;
}

// cropModel (engine/src/splat/Crop.cpp:44-52): centre inside the box and sigmoid(opacity) >= floor.
size_t orc_crop_model(const u3dg_model *model, const u3dg_crop_box *box, float min_opacity, u3dg_model *out)
{
    const orc::Model m = orc::fromView(*model);
    size_t kept = 0;
    for (size_t i = 0; i < m.size(); ++i) {
        const float *p = &m.means[i * 3];
        const bool in = p[0] >= box->min[0] && p[0] <= box->max[0] && p[1] >= box->min[1] && p[1] <= box->max[1] &&
                        p[2] >= box->min[2] && p[2] <= box->max[2];
        if (!in || !(orc::sigmoidf(m.opac[i]) >= min_opacity))
            continue;
        if (out) {
            std::copy(&m.means[i * 3], &m.means[i * 3] + 3, out->means + kept * 3);
            std::copy(&m.scales[i * 3], &m.scales[i * 3] + 3, out->scales + kept * 3);
            std::copy(&m.quats[i * 4], &m.quats[i * 4] + 4, out->quats + kept * 4);
            out->opacities[kept] = m.opac[i];
            std::copy(&m.colors[i * 3], &m.colors[i * 3] + 3, out->colors + kept * 3);
        }
        ++kept;
    }
    return kept;
}

// quantileBox (Crop.cpp:12-40): per axis, the lo / hi quantiles (std::nth_element) of the centres of
// Gaussians at least min_opacity opaque (all centres when none is), widened by margin (at least 1e-4).
void orc_crop_box(const u3dg_model *model, float lo, float hi, float margin, float min_opacity, u3dg_crop_box *box)
{
    const orc::Model m = orc::fromView(*model);
    std::vector<float> axis;
    for (int k = 0; k < 3; ++k) {
        axis.clear();
        for (size_t i = 0; i < m.size(); ++i)
            if (orc::sigmoidf(m.opac[i]) >= min_opacity)
                axis.push_back(m.means[i * 3 + size_t(k)]);
        if (axis.empty())
            for (size_t i = 0; i < m.size(); ++i)
                axis.push_back(m.means[i * 3 + size_t(k)]);
        if (axis.empty()) {
            box->min[k] = -1.0f;
            box->max[k] = 1.0f;
            continue;
        }
        auto at = [&](float q) {
            const size_t idx = std::min(axis.size() - 1, size_t(q * float(axis.size() - 1) + 0.5f));
            std::nth_element(axis.begin(), axis.begin() + std::ptrdiff_t(idx), axis.end());
            return axis[idx];
        };
        const float a = at(lo), b = at(hi);
        const float pad = std::max((b - a) * margin, 1e-4f);
        box->min[k] = a - pad;
        box->max[k] = b + pad;
    }
}

void orc_init_from_points(const float *xyz, const float *rgb, size_t n, u3dg_model *out)
{
    Model m = initFromPoints(xyz, rgb, n);
    toView(m, *out);
}

// TrainOptions::forIterations (Trainer.cpp:26-35) and the struct defaults (Trainer.h:20-38,
// Rasterizer.h:23-32, Adam.h:8-14), restated for the host-logic tests.
void orc_options_for_iterations(int iterations, u3dg_train_options *o)
{
    u3dg_train_options d{};
    d.iterations = 3000;
    d.max_gaussians = 200000;
    d.ssim_lambda = 0.2f;
    d.lr = {1.6e-4f, 5e-3f, 1e-3f, 5e-2f, 2.5e-3f};
    d.means_lr_final = 1.6e-6f;
    d.densify_grad_threshold = 2e-4f;
    d.percent_dense = 0.01f;
    d.refine_start = 500;
    d.refine_stop = 15000;
    d.refine_interval = 100;
    d.opacity_reset_interval = 3000;
    d.prune_opacity = 0.005f;
    d.seed = 42;
    d.raster.tile_size = 16;
    d.raster.near_plane = 0.01f;
    d.raster.eps2d = 0.3f;
    d.raster.background[0] = d.raster.background[1] = d.raster.background[2] = 0.0f;
    d.raster.min_alpha = 1.0f / 255.0f;
    d.raster.min_transmittance = 1e-4f;
    if (iterations > 0) {
        d.iterations = std::max(1, iterations);
        d.refine_start = std::min(500, d.iterations / 10);
        d.refine_stop = d.iterations * 6 / 10;
        d.refine_interval = 100;
        d.opacity_reset_interval = d.iterations >= 6000 ? 3000 : 0;
    }
    *o = d;
}

} // extern "C"
