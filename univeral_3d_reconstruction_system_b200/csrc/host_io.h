// host_io.h - host-side model I/O and initialisation (no GPU needed).
#pragma once

#include "../../include/u3dg.h"

#include <cstdint>
#include <string>
#include <vector>

namespace u3dg {

struct HostModel {
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
};

// initGaussiansFromPoints (GaussianModel.cpp:68-144) on the host; out must hold n Gaussians. Used by
// the PLY reader for point clouds (readSplatPly does the same in the reference).
void initGaussiansFromPointsHost(const float *xyz, const float *rgb, size_t n, u3dg_model &out);

// Its pieces, shared with the GPU version (initGaussiansFromPointsDevice): the hash grid
// (GaussianModel.cpp:72-98), the cell key, and the model written from every point's 3 smallest
// squared neighbour distances (best[3n], FLT_MAX where fewer were found; GaussianModel.cpp:122-142).
struct InitGrid {
    float cell = 0.0f;
    std::vector<int> cx, cy, cz;  // cell coordinates per point
    std::vector<int64_t> keys;    // cell keys, sorted
    std::vector<uint32_t> ids;    // point index per sorted key (ties in index order)
};
int64_t initHashKey(int x, int y, int z);
void buildInitGrid(const float *xyz, size_t n, InitGrid &g);
void finishInitFromNeighbours(const float *xyz, const float *rgb, size_t n, float cell, const float *best,
                              u3dg_model &out);
// The same initialisation with the 27-cell neighbour search on the current GPU (bit-identical).
void initGaussiansFromPointsDevice(const float *xyz, const float *rgb, size_t n, u3dg_model &out);
// writeSplatPly (SplatPly.cpp:261-282). With shRest (shDegree 1..3; K = (shDegree + 1)^2 - 1
// coefficients per channel, laid out as u3dg_render_sh takes them: [i][k][channel]), the common 3DGS
// extension: properties f_rest_0 .. f_rest_{3K-1} after f_dc_2, channel-major (f_rest_{c K + k}).
bool writeSplatPlyHost(const std::string &path, const u3dg_model &m, std::string *error, const float *shRest = nullptr,
                       int shDegree = 0);
// readSplatPly (SplatPly.cpp:284-342).
bool readSplatPlyHost(const std::string &path, HostModel &m, std::string *error, bool *isSplat);

} // namespace u3dg
