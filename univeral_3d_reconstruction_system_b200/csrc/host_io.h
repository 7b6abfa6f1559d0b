// host_io.h - host-side model I/O and initialisation (no GPU needed).
#pragma once

#include "../../include/u3dg.h"

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

// initGaussiansFromPoints (GaussianModel.cpp:68-144); out must hold n Gaussians.
void initGaussiansFromPointsHost(const float *xyz, const float *rgb, size_t n, u3dg_model &out);
// writeSplatPly (SplatPly.cpp:261-282).
bool writeSplatPlyHost(const std::string &path, const u3dg_model &m, std::string *error);
// readSplatPly (SplatPly.cpp:284-342).
bool readSplatPlyHost(const std::string &path, HostModel &m, std::string *error, bool *isSplat);

} // namespace u3dg
