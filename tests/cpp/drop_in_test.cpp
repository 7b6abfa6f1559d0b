// drop_in_test.cpp - the reference's own trainer test, with only the trainer switched to the GPU one.
//
// training_recovers_a_synthetic_scene of the reference (tests/test_splat.cpp:227-268) written against
// the reference's types (u3d::GaussianModel, TrainImage, TrainOptions, ThreadPool, Rasterizer for the
// ground truth, initGaussiansFromPoints), training with u3d::gpu::Trainer: the change a maintainer
// makes in engine/src/pipeline/Reconstructor.cpp:331. Also checks the PLY written from the GPU model
// through the reference's own readSplatPly. Prints "drop-in ok" and exits 0 on success.

#include "u3d/splat/Rasterizer.h"
#include "u3d/splat/SplatPly.h"
#include "u3d/splat/Trainer.h"

#include "u3d_gpu.hpp"

#include <cmath>
#include <cstdio>
#include <random>

namespace {

int failures = 0;

#define EXPECT(cond)                                                              \
    do {                                                                          \
        if (!(cond)) {                                                            \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);         \
            ++failures;                                                           \
        }                                                                         \
    } while (0)

u3d::RenderCamera orbit(int w, int h, float f, float angle, float radius, float height)
{
    u3d::RenderCamera c;
    c.width = w;
    c.height = h;
    c.fx = c.fy = f;
    c.cx = 0.5f * float(w - 1);
    c.cy = 0.5f * float(h - 1);
    const float C[3] = {radius * std::sin(angle), height, -radius * std::cos(angle)};
    float z[3] = {-C[0], -C[1], -C[2]};
    const float zn = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
    for (float &v : z)
        v /= zn;
    // x = -(down x z) / |down x z| with down = (0, 1, 0); y = z x x.
    float x[3] = {z[2], 0.0f, -z[0]};
    const float xn = std::sqrt(x[0] * x[0] + x[2] * x[2]);
    for (float &v : x)
        v /= -xn;
    const float y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
    for (int k = 0; k < 3; ++k) {
        c.R[k] = x[k];
        c.R[3 + k] = y[k];
        c.R[6 + k] = z[k];
    }
    for (int r = 0; r < 3; ++r)
        c.t[r] = -(c.R[r * 3] * C[0] + c.R[r * 3 + 1] * C[1] + c.R[r * 3 + 2] * C[2]);
    return c;
}

} // namespace

int main()
{
    u3d::ThreadPool pool(4);
    std::mt19937 rng(11);
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
    std::vector<u3d::TrainImage> images;
    u3d::Rasterizer raster(pool);
    for (int k = 0; k < 16; ++k) {
        u3d::TrainImage img;
        img.camera = orbit(96, 72, 80.0f, 6.2831853f * float(k) / 16.0f, 4.0f, -1.0f + 0.15f * float(k % 4));
        std::vector<float> rendered;
        raster.forward(truth, img.camera, u3d::RasterSettings(), rendered);
        img.rgb = u3d::TrainImage::quantize(rendered);
        images.push_back(std::move(img));
    }
    std::normal_distribution<float> noise(0.0f, 0.08f);
    std::vector<float> xyz, rgb;
    for (std::size_t i = 0; i < truth.size(); i += 2)
        for (int k = 0; k < 3; ++k) {
            xyz.push_back(truth.means[i * 3 + k] + noise(rng));
            rgb.push_back(0.5f);
        }
    const u3d::GaussianModel init = u3d::initGaussiansFromPoints(xyz, rgb);
    u3d::TrainOptions opt = u3d::TrainOptions::forIterations(1500);
    opt.maxGaussians = 4000;

    u3d::gpu::Trainer trainer(init, images, 4.4f, opt, pool); // <- the only change from the reference test
    const float before = trainer.evaluatePsnr();
    while (!trainer.done())
        trainer.step();
    const float after = trainer.evaluatePsnr();
    std::printf("PSNR %.2f dB -> %.2f dB, %zu -> %zu Gaussians\n", before, after, init.size(), trainer.model().size());
    EXPECT(after > before + 8.0f);
    EXPECT(after > 26.0f);
    EXPECT(trainer.model().size() != init.size());
    EXPECT(trainer.stats().iteration == 1500);

    // The trained model goes out through the reference's own PLY writer and reader.
    const u3d::GaussianModel out = u3d::gpu::modelTo<u3d::GaussianModel>(trainer.model());
    std::string err;
    EXPECT(u3d::writeSplatPly("drop_in_test.ply", out, &err));
    u3d::GaussianModel back;
    bool isSplat = false;
    EXPECT(u3d::readSplatPly("drop_in_test.ply", back, &err, &isSplat));
    EXPECT(isSplat && back.size() == out.size());
    std::remove("drop_in_test.ply");

    // Rendering a training view through the drop-in API matches the evaluation.
    std::vector<float> img;
    trainer.render(images[0].camera, img);
    EXPECT(img.size() == std::size_t(96 * 72 * 3));

    // The learned warm-start without a network is initGaussiansFromPoints exactly.
    std::vector<u3d::gpu::TrainImage> gpuImages;
    for (const u3d::TrainImage &i : images)
        gpuImages.push_back(u3d::gpu::imageFrom(i));
    const u3d::gpu::GaussianModel plain = u3d::gpu::warmStartFromPoints(nullptr, xyz, rgb, gpuImages);
    const u3d::gpu::GaussianModel ref = u3d::gpu::modelFrom(init);
    EXPECT(plain.means == ref.means && plain.scales == ref.scales && plain.quats == ref.quats &&
           plain.opacities == ref.opacities && plain.colors == ref.colors);

    // Two copies of the scene trained as one batch end where the single trainer ended.
    std::vector<u3d::gpu::BatchTrainer::Scene> scenes(2);
    for (auto &sc : scenes) {
        sc.initial = ref;
        sc.images = gpuImages;
        sc.sceneExtent = 4.4f;
        sc.options = u3d::gpu::optionsFrom(opt);
    }
    u3d::gpu::BatchTrainer batch(std::move(scenes), false);
    batch.step(1500);
    const u3d::gpu::GaussianModel single = u3d::gpu::modelFrom(out);
    for (int s = 0; s < 2; ++s) {
        const u3d::gpu::GaussianModel m = batch.model(s);
        EXPECT(m.means == single.means && m.opacities == single.opacities && m.colors == single.colors);
        EXPECT(std::fabs(batch.evaluatePsnr(s) - after) < 1e-6f);
    }
    if (failures == 0)
        std::printf("drop-in ok\n");
    return failures == 0 ? 0 : 1;
}
