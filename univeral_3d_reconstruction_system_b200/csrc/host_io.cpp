// host_io.cpp - the plain point-cloud initialisation on the host (its hash grid is shared with the
// GPU neighbour search in init.cu). Runs once per training run, outside the hot loop. The PLY
// reader and writer are in ply.cpp.

#include "host_io.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

namespace u3dg {

namespace {

constexpr float kC0 = 0.28209479177387814f;

float logitHost(float p) { return std::log(p / (1.0f - p)); }

} // namespace

// The reference buckets points by a hash of their grid cell and scans the 27 neighbouring keys
// (GaussianModel.cpp:84-121). Points whose cells hash to the same key share a bucket there, and
// a bucket whose key appears twice among the 27 is scanned twice; both effects change which
// distances compete for the 3 nearest, so they are kept: here the buckets are runs of a
// key-sorted index, looked up by binary search.
int64_t initHashKey(int x, int y, int z)
{
    return (int64_t(x) * 73856093) ^ (int64_t(y) * 19349663) ^ (int64_t(z) * 83492791);
}

void buildInitGrid(const float *xyz, size_t n, InitGrid &g)
{
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
    g.cell = std::max(ext / std::cbrt(float(n)) * 2.0f, 1e-6f);
    g.cx.resize(n);
    g.cy.resize(n);
    g.cz.resize(n);
    std::vector<std::pair<int64_t, uint32_t>> bucket(n);
    for (size_t i = 0; i < n; ++i) {
        g.cx[i] = int(std::floor((xyz[i * 3] - lo[0]) / g.cell));
        g.cy[i] = int(std::floor((xyz[i * 3 + 1] - lo[1]) / g.cell));
        g.cz[i] = int(std::floor((xyz[i * 3 + 2] - lo[2]) / g.cell));
        bucket[i] = {initHashKey(g.cx[i], g.cy[i], g.cz[i]), uint32_t(i)};
    }
    std::sort(bucket.begin(), bucket.end());
    g.keys.resize(n);
    g.ids.resize(n);
    for (size_t i = 0; i < n; ++i) {
        g.keys[i] = bucket[i].first;
        g.ids[i] = bucket[i].second;
    }
}

void finishInitFromNeighbours(const float *xyz, const float *rgb, size_t n, float cell, const float *best,
                              u3dg_model &out)
{
    const float fmax = std::numeric_limits<float>::max();
    const float op = logitHost(0.1f);
    for (size_t i = 0; i < n; ++i) {
        float sum = 0;
        int cnt = 0;
        for (int k = 0; k < 3; ++k)
            if (best[i * 3 + k] < fmax) {
                sum += best[i * 3 + k];
                ++cnt;
            }
        const float meanD2 = cnt ? sum / float(cnt) : cell * cell;
        const float logScale = std::log(std::sqrt(std::max(meanD2, 1e-14f)));
        for (int k = 0; k < 3; ++k) {
            out.means[i * 3 + k] = xyz[i * 3 + k];
            out.scales[i * 3 + k] = logScale;
            const float col = rgb ? rgb[i * 3 + k] : 0.5f;
            out.colors[i * 3 + k] = (col - 0.5f) / kC0;
        }
        out.quats[i * 4] = 1.0f;
        out.quats[i * 4 + 1] = out.quats[i * 4 + 2] = out.quats[i * 4 + 3] = 0.0f;
        out.opacities[i] = op;
    }
}

void initGaussiansFromPointsHost(const float *xyz, const float *rgb, size_t n, u3dg_model &out)
{
    if (n == 0)
        return;
    InitGrid g;
    buildInitGrid(xyz, n, g);
    const float fmax = std::numeric_limits<float>::max();
    std::vector<float> best(n * 3, fmax);
    for (size_t i = 0; i < n; ++i) {
        float *b = &best[i * 3];
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    const int64_t key = initHashKey(g.cx[i] + dx, g.cy[i] + dy, g.cz[i] + dz);
                    size_t it = size_t(std::lower_bound(g.keys.begin(), g.keys.end(), key) - g.keys.begin());
                    for (; it < n && g.keys[it] == key; ++it) {
                        const size_t j = g.ids[it];
                        if (j == i)
                            continue;
                        const float ex = xyz[j * 3] - xyz[i * 3], ey = xyz[j * 3 + 1] - xyz[i * 3 + 1],
                                    ez = xyz[j * 3 + 2] - xyz[i * 3 + 2];
                        float d2 = ex * ex + ey * ey + ez * ez;
                        for (int k = 0; k < 3; ++k)
                            if (d2 < b[k])
                                std::swap(d2, b[k]);
                    }
                }
    }
    finishInitFromNeighbours(xyz, rgb, n, g.cell, best.data(), out);
}

} // namespace u3dg
