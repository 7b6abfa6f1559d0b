// stage_test.cpp - the pipeline's training stage (engine/src/pipeline/Reconstructor.cpp:296-361) on
// the GPU trainer, through u3d::gpu::trainSplatStage with the reference's own types.
//
// A synthetic project as the pipeline sees it after pose estimation and alignment: full-resolution
// cameras (u3d::Camera, 192x144) on an orbit, training images at half that size, and a sparse cloud of
// 150 points (fewer than 1000, so the stage adds the random ones). Checks that the stage computes
// the reference pipeline's extent, random points and training cameras (restated here from
// Reconstructor.cpp with the reference's Camera::scaled and RenderCamera::fromCamera), reports
// progress, trains, writes a PLY the reference's reader accepts, and stops on cancellation. Prints
// "stage ok" and exits 0 on success.

#include "u3d/Camera.h"
#include "u3d/splat/Rasterizer.h"
#include "u3d/splat/SplatPly.h"
#include "u3d/splat/Trainer.h"

#include "u3d_gpu.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>

namespace {

int failures = 0;

#define EXPECT(cond)                                                              \
    do {                                                                          \
        if (!(cond)) {                                                            \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);         \
            ++failures;                                                           \
        }                                                                         \
    } while (0)

// A full-resolution camera on a circle of `radius` around the origin, looking at it (OpenCV axes).
u3d::Camera orbit(int w, int h, double f, double angle, double radius, double height)
{
    u3d::Camera c;
    c.width = w;
    c.height = h;
    c.fx = c.fy = f;
    c.cx = 0.5 * (w - 1);
    c.cy = 0.5 * (h - 1);
    const double C[3] = {radius * std::sin(angle), height, -radius * std::cos(angle)};
    double z[3] = {-C[0], -C[1], -C[2]};
    const double zn = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
    for (double &v : z)
        v /= zn;
    double x[3] = {z[2], 0.0, -z[0]};
    const double xn = std::sqrt(x[0] * x[0] + x[2] * x[2]);
    for (double &v : x)
        v /= -xn;
    const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
    for (int k = 0; k < 3; ++k) {
        c.R[std::size_t(k)] = x[k];
        c.R[std::size_t(3 + k)] = y[k];
        c.R[std::size_t(6 + k)] = z[k];
    }
    for (int r = 0; r < 3; ++r)
        c.t[std::size_t(r)] = -(c.R[std::size_t(r * 3)] * C[0] + c.R[std::size_t(r * 3 + 1)] * C[1] +
                                c.R[std::size_t(r * 3 + 2)] * C[2]);
    return c;
}

bool sameCamera(const u3d::RenderCamera &a, const u3d::RenderCamera &b)
{
    return a.width == b.width && a.height == b.height && a.fx == b.fx && a.fy == b.fy && a.cx == b.cx &&
           a.cy == b.cy && std::memcmp(a.R, b.R, sizeof a.R) == 0 && std::memcmp(a.t, b.t, sizeof a.t) == 0;
}

} // namespace

int main()
{
    u3d::ThreadPool pool(4);
    std::mt19937 rng(5);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f), u01(0.0f, 1.0f);
    u3d::GaussianModel truth;
    truth.resize(300);
    for (std::size_t i = 0; i < 300; ++i) {
        for (int k = 0; k < 3; ++k) {
            truth.means[i * 3 + k] = u(rng) * (k == 1 ? 0.8f : 1.0f);
            truth.scales[i * 3 + k] = std::log(0.03f + 0.09f * u01(rng));
            truth.colors[i * 3 + k] = (0.15f + 0.7f * u01(rng) - 0.5f) / u3d::kShC0;
        }
        for (int k = 0; k < 4; ++k)
            truth.quats[i * 4 + k] = u(rng) + (k == 0 ? 1.5f : 0.0f);
        truth.opacities[i] = u3d::logit(0.8f);
    }
    // The project: full-resolution cameras, training images at half the width (their cameras are set
    // by the stage), the full widths, and 150 noisy sparse points.
    std::vector<u3d::Camera> cameras;
    std::vector<u3d::TrainImage> train;
    std::vector<int> fullW;
    u3d::Rasterizer raster(pool);
    for (int k = 0; k < 16; ++k) {
        const u3d::Camera full = orbit(192, 144, 160.0, 6.2831853 * k / 16.0, 4.0, -1.0 + 0.15 * (k % 4));
        cameras.push_back(full);
        fullW.push_back(full.width);
        u3d::TrainImage img;
        img.camera = u3d::RenderCamera::fromCamera(full.scaled(0.5));
        std::vector<float> rendered;
        raster.forward(truth, img.camera, u3d::RasterSettings(), rendered);
        img.rgb = u3d::TrainImage::quantize(rendered);
        img.camera.fx = img.camera.fy = 1.0f; // the stage must set the training cameras itself
        train.push_back(std::move(img));
    }
    std::normal_distribution<float> noise(0.0f, 0.05f);
    std::vector<float> xyz, rgb;
    for (std::size_t i = 0; i < truth.size(); i += 2)
        for (int k = 0; k < 3; ++k) {
            xyz.push_back(truth.means[i * 3 + k] + noise(rng));
            rgb.push_back(0.5f);
        }
    const std::vector<float> sparse = xyz, sparseRgb = rgb;

    int reports = 0, logs = 0;
    double lastFraction = 0;
    bool monotone = true;
    auto report = [&](const std::string &stage, double fraction, const std::string &) {
        ++reports;
        monotone = monotone && (fraction >= lastFraction) && (stage == "training" || stage == "export");
        lastFraction = fraction;
    };
    auto say = [&](const std::string &) { ++logs; };
    u3d::gpu::StageResult res;
    std::string err;
    const bool ok = u3d::gpu::trainSplatStage(cameras, train, fullW, xyz, rgb, 800, 4000, 0.5, "stage_test.ply",
                                              report, say, [] { return false; }, res, &err);
    EXPECT(ok);
    if (!ok)
        std::printf("stage failed: %s\n", err.c_str());

    // Extent as Reconstructor.cpp:288-296 computes it.
    double mean[3] = {0, 0, 0};
    for (const u3d::Camera &c : cameras) {
        const auto cc = c.center();
        for (int k = 0; k < 3; ++k)
            mean[k] += cc[std::size_t(k)] / double(cameras.size());
    }
    double extent = 0;
    for (const u3d::Camera &c : cameras) {
        const auto cc = c.center();
        extent = std::max(extent, std::sqrt((cc[0] - mean[0]) * (cc[0] - mean[0]) + (cc[1] - mean[1]) * (cc[1] - mean[1]) +
                                            (cc[2] - mean[2]) * (cc[2] - mean[2])));
    }
    extent = std::max(extent * 1.1, 1e-3);
    EXPECT(res.extent == extent);
    // The random points of Reconstructor.cpp:298-309, appended to the sparse cloud.
    std::vector<float> wantXyz = sparse, wantRgb = sparseRgb;
    {
        std::mt19937 r(1);
        std::uniform_real_distribution<float> uu(-1.0f, 1.0f), uu01(0.0f, 1.0f);
        const float rr = float(extent) * 0.6f;
        for (int k = 0; k < 10000; ++k) {
            wantXyz.insert(wantXyz.end(), {uu(r) * rr, uu(r) * rr, uu(r) * rr});
            wantRgb.insert(wantRgb.end(), {uu01(r), uu01(r), uu01(r)});
        }
    }
    EXPECT(xyz == wantXyz && rgb == wantRgb);
    // Training cameras: Camera::scaled to the image, converted by RenderCamera::fromCamera.
    for (std::size_t k = 0; k < train.size(); ++k) {
        u3d::Camera c = cameras[k].scaled(96.0 / 192.0);
        c.width = 96;
        c.height = 72;
        EXPECT(sameCamera(train[k].camera, u3d::RenderCamera::fromCamera(c)));
    }
    std::printf("stage: extent %.4f, %zu initial points, %zu Gaussians, PSNR %.2f dB, %d reports, %d log lines\n",
                res.extent, xyz.size() / 3, res.gaussians, res.psnr, reports, logs);
    EXPECT(res.psnr > 24.0f);
    EXPECT(reports >= 80 && monotone && logs >= 4);
    // The PLY through the reference's own reader.
    u3d::GaussianModel back;
    bool isSplat = false;
    EXPECT(u3d::readSplatPly("stage_test.ply", back, &err, &isSplat));
    EXPECT(isSplat && back.size() == res.gaussians);
    std::remove("stage_test.ply");

    // Cancellation between steps, as the pipeline polls it.
    int polls = 0;
    std::vector<float> xyz2 = sparse, rgb2 = sparseRgb;
    std::vector<u3d::TrainImage> train2 = train;
    u3d::gpu::StageResult res2;
    const bool ok2 = u3d::gpu::trainSplatStage(cameras, train2, fullW, xyz2, rgb2, 800, 4000, 0.5, "stage_cancel.ply",
                                               report, say, [&] { return ++polls > 50; }, res2, &err);
    EXPECT(!ok2 && err == "Cancelled" && polls == 51);
    if (failures == 0)
        std::printf("stage ok\n");
    return failures == 0 ? 0 : 1;
}
