// u3d_gpu.hpp - C++ drop-in for the reference's splat trainer API, over the C ABI of u3dg.h.
//
// Same types, names and semantics as engine/include/u3d/splat (Trainer.h, Rasterizer.h, Loss.h,
// GaussianModel.h, SplatPly.h) of Abner0907/univeral_3d_reconstruction_system, in namespace u3d::gpu.
// Header-only; link against libu3dg.so. Errors of the GPU library throw u3d::gpu::Error (the reference
// has no error channel except the bool results of the PLY functions, which are kept).
//
// The constructors and fromReference/toReference helpers are templates over any type with the
// reference's field names, so code holding the reference's own u3d::GaussianModel / TrainImage /
// TrainOptions / RenderCamera can pass them straight in.
#pragma once

#include "u3dg.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace u3d {
namespace gpu {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(int status)
{
    if (status != U3DG_OK)
        throw Error(status, u3dg_last_error());
}

constexpr float kShC0 = 0.28209479177387814f; // GaussianModel.h:10

// GaussianModel (GaussianModel.h:23-37).
struct GaussianModel {
    std::vector<float> means, scales, quats, opacities, colors;
    std::size_t size() const { return opacities.size(); }
    void resize(std::size_t n)
    {
        means.resize(n * 3);
        scales.resize(n * 3);
        quats.resize(n * 4);
        opacities.resize(n);
        colors.resize(n * 3);
    }
    u3dg_model view() const
    {
        return {const_cast<float *>(means.data()), const_cast<float *>(scales.data()),
                const_cast<float *>(quats.data()), const_cast<float *>(opacities.data()),
                const_cast<float *>(colors.data()), size()};
    }
};

// RenderCamera / RasterSettings (Rasterizer.h:13-32).
struct RenderCamera : u3dg_camera {
    RenderCamera() : u3dg_camera{0, 0, 0, 0, 0, 0, {1, 0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 0}} {}
};

struct RasterSettings : u3dg_raster_settings {
    RasterSettings() : u3dg_raster_settings{} { u3dg_raster_settings_default(this); }
};

struct LearningRates : u3dg_learning_rates {
    LearningRates() : u3dg_learning_rates{1.6e-4f, 5e-3f, 1e-3f, 5e-2f, 2.5e-3f} {}
};

// TrainOptions (Trainer.h:20-38).
struct TrainOptions : u3dg_train_options {
    TrainOptions() : u3dg_train_options{} { u3dg_train_options_default(this); }
    static TrainOptions forIterations(int iterations)
    {
        TrainOptions o;
        u3dg_train_options_for_iterations(iterations, &o);
        return o;
    }
};

// TrainImage (Trainer.h:13-18).
struct TrainImage {
    RenderCamera camera;
    std::vector<std::uint8_t> rgb; // height * width * 3
};

// TrainStats (Trainer.h:40-45).
struct TrainStats {
    int iteration = 0;
    float loss = 0;
    float psnr = 0;
    std::size_t gaussians = 0;
};

// ------------------------------------------------------------------ adapters from / to reference types

template <class Cam>
RenderCamera cameraFrom(const Cam &c)
{
    RenderCamera r;
    r.width = c.width;
    r.height = c.height;
    r.fx = c.fx;
    r.fy = c.fy;
    r.cx = c.cx;
    r.cy = c.cy;
    for (int k = 0; k < 9; ++k)
        r.R[k] = c.R[k];
    for (int k = 0; k < 3; ++k)
        r.t[k] = c.t[k];
    return r;
}

template <class M>
GaussianModel modelFrom(const M &m)
{
    GaussianModel g;
    g.means.assign(m.means.begin(), m.means.end());
    g.scales.assign(m.scales.begin(), m.scales.end());
    g.quats.assign(m.quats.begin(), m.quats.end());
    g.opacities.assign(m.opacities.begin(), m.opacities.end());
    g.colors.assign(m.colors.begin(), m.colors.end());
    return g;
}

template <class M>
M modelTo(const GaussianModel &g)
{
    M m;
    m.means.assign(g.means.begin(), g.means.end());
    m.scales.assign(g.scales.begin(), g.scales.end());
    m.quats.assign(g.quats.begin(), g.quats.end());
    m.opacities.assign(g.opacities.begin(), g.opacities.end());
    m.colors.assign(g.colors.begin(), g.colors.end());
    return m;
}

template <class O>
TrainOptions optionsFrom(const O &o)
{
    TrainOptions t;
    t.iterations = o.iterations;
    t.max_gaussians = o.maxGaussians;
    t.ssim_lambda = o.ssimLambda;
    t.lr.means = o.lr.means;
    t.lr.scales = o.lr.scales;
    t.lr.quats = o.lr.quats;
    t.lr.opacities = o.lr.opacities;
    t.lr.colors = o.lr.colors;
    t.means_lr_final = o.meansLrFinal;
    t.densify_grad_threshold = o.densifyGradThreshold;
    t.percent_dense = o.percentDense;
    t.refine_start = o.refineStart;
    t.refine_stop = o.refineStop;
    t.refine_interval = o.refineInterval;
    t.opacity_reset_interval = o.opacityResetInterval;
    t.prune_opacity = o.pruneOpacity;
    t.seed = o.seed;
    t.raster.tile_size = o.raster.tileSize;
    t.raster.near_plane = o.raster.nearPlane;
    t.raster.eps2d = o.raster.eps2d;
    for (int k = 0; k < 3; ++k)
        t.raster.background[k] = o.raster.background[k];
    t.raster.min_alpha = o.raster.minAlpha;
    t.raster.min_transmittance = o.raster.minTransmittance;
    return t;
}

inline TrainOptions optionsFrom(const TrainOptions &o) { return o; }

template <class I>
TrainImage imageFrom(const I &img)
{
    TrainImage t;
    t.camera = cameraFrom(img.camera);
    t.rgb.assign(img.rgb.begin(), img.rgb.end());
    return t;
}

inline TrainImage imageFrom(const TrainImage &img) { return img; }
inline GaussianModel modelFrom(const GaussianModel &m) { return m; }

// ------------------------------------------------------------------ Trainer (Trainer.h:47-93)

class Trainer
{
public:
    // Trainer(GaussianModel initial, std::vector<TrainImage> images, float sceneExtent,
    //         const TrainOptions &options, ThreadPool &pool). The pool is accepted for API
    // compatibility and not used: the work runs on the current CUDA device.
    template <class Model, class Image, class Options, class Pool>
    Trainer(const Model &initial, const std::vector<Image> &images, float sceneExtent, const Options &options, Pool &)
        : Trainer(modelFrom(initial), convert(images), sceneExtent, optionsFrom(options))
    {
    }

    Trainer(GaussianModel initial, std::vector<TrainImage> images, float sceneExtent, const TrainOptions &options)
        : m_images(std::move(images)), m_options(options)
    {
        std::vector<u3dg_image> views(m_images.size());
        for (std::size_t k = 0; k < m_images.size(); ++k)
            views[k] = {m_images[k].camera, m_images[k].rgb.data()};
        const u3dg_model v = initial.view();
        // The trainer owns its images (as the reference's does), so they can go to the GPU while
        // the first steps run.
        check(u3dg_trainer_create_background_upload(&v, views.data(), int(views.size()), sceneExtent, &m_options,
                                                    &m_t));
    }

    ~Trainer() { u3dg_trainer_destroy(m_t); }
    Trainer(const Trainer &) = delete;
    Trainer &operator=(const Trainer &) = delete;

    void step() { check(u3dg_trainer_step(m_t, 1)); }
    bool done() const
    {
        int d = 0;
        check(u3dg_trainer_done(m_t, &d));
        return d != 0;
    }
    int iteration() const
    {
        int it = 0;
        check(u3dg_trainer_iteration(m_t, &it));
        return it;
    }
    // The current model, copied back from the GPU; valid until the next step().
    const GaussianModel &model() const
    {
        std::size_t n = 0;
        check(u3dg_trainer_size(m_t, &n));
        m_model.resize(n);
        u3dg_model v = m_model.view();
        check(u3dg_trainer_download(m_t, &v, n, &n));
        return m_model;
    }
    const TrainStats &stats() const
    {
        u3dg_train_stats s{};
        check(u3dg_trainer_stats(m_t, &s));
        m_stats.iteration = s.iteration;
        m_stats.loss = s.loss;
        m_stats.psnr = s.psnr;
        m_stats.gaussians = std::size_t(s.gaussians);
        return m_stats;
    }
    const std::vector<TrainImage> &images() const { return m_images; }
    float evaluatePsnr()
    {
        float p = 0;
        check(u3dg_trainer_eval_psnr(m_t, &p));
        return p;
    }
    template <class Cam>
    void render(const Cam &camera, std::vector<float> &rgb)
    {
        const RenderCamera c = cameraFrom(camera);
        rgb.resize(std::size_t(c.width) * c.height * 3);
        check(u3dg_trainer_render(m_t, &c, rgb.data()));
    }
    // The C ABI handle (for entry points with no reference counterpart, e.g. the PLY export).
    u3dg_trainer *handle() const { return m_t; }

private:
    template <class Image>
    static std::vector<TrainImage> convert(const std::vector<Image> &images)
    {
        std::vector<TrainImage> out;
        out.reserve(images.size());
        for (const Image &i : images)
            out.push_back(imageFrom(i));
        return out;
    }

    u3dg_trainer *m_t = nullptr;
    std::vector<TrainImage> m_images;
    TrainOptions m_options;
    mutable GaussianModel m_model;
    mutable TrainStats m_stats;
};

// ------------------------------------------------------------------ free functions

// initGaussiansFromPoints (GaussianModel.h:41).
inline GaussianModel initGaussiansFromPoints(const std::vector<float> &xyz, const std::vector<float> &rgb)
{
    GaussianModel m;
    const std::size_t n = xyz.size() / 3;
    m.resize(n);
    u3dg_model v = m.view();
    check(u3dg_init_gaussians_from_points(xyz.data(), rgb.size() >= n * 3 ? rgb.data() : nullptr, n, &v));
    return m;
}

// writeSplatPly / readSplatPly (SplatPly.h:12-18): bool results and an optional error string.
inline bool writeSplatPly(const std::string &path, const GaussianModel &model, std::string *error = nullptr)
{
    const u3dg_model v = model.view();
    if (u3dg_write_splat_ply(path.c_str(), &v) == U3DG_OK)
        return true;
    if (error)
        *error = u3dg_last_error();
    return false;
}

inline bool readSplatPly(const std::string &path, GaussianModel &model, std::string *error = nullptr,
                         bool *isSplat = nullptr)
{
    std::size_t n = 0;
    int splat = 0;
    if (u3dg_read_splat_ply(path.c_str(), nullptr, 0, &n, &splat) != U3DG_OK) {
        if (error)
            *error = u3dg_last_error();
        return false;
    }
    model.resize(n);
    u3dg_model v = model.view();
    if (u3dg_read_splat_ply(path.c_str(), &v, n, &n, &splat) != U3DG_OK) {
        if (error)
            *error = u3dg_last_error();
        return false;
    }
    if (isSplat)
        *isSplat = splat != 0;
    return true;
}

// photometricLoss / psnr (Loss.h:18-21).
struct LossValue {
    float total = 0, l1 = 0, ssim = 0;
};

inline LossValue photometricLoss(const float *render, const float *target, int width, int height, float ssimLambda,
                                 float *grad)
{
    u3dg_loss_value v{};
    check(u3dg_photometric_loss(render, target, width, height, ssimLambda, grad, &v));
    return {v.total, v.l1, v.ssim};
}

inline float psnr(const float *a, const float *b, std::size_t count)
{
    float p = 0;
    check(u3dg_psnr(a, b, count, &p));
    return p;
}

// ------------------------------------------------------------------ pipeline training stage

// The training stage of reconstructProject (engine/src/pipeline/Reconstructor.cpp:296-361) on the GPU
// trainer: scene extent, random initial points for sparse clouds, training cameras scaled to the
// training images, initGaussiansFromPoints, the training loop with cancellation and progress, the
// splat PLY and the mean training PSNR. Templated over the reference's types: Cam is u3d::Camera
// (center(), scaled()), Img its TrainImage (camera, rgb); report / say / cancelled are the pipeline's
// progress, log and cancel hooks (Progress-like objects with stage, fraction, message; strings;
// bool()). The caller keeps the steps around it (loading, poses, alignment, cameras.txt and
// sparse.ply, which need the cameras and points this updates in place).
struct StageResult {
    std::string splatPath;
    std::size_t gaussians = 0;
    float psnr = 0;
    double extent = 0;
};

template <class Cam, class Img, class Report, class Say, class Cancelled>
bool trainSplatStage(const std::vector<Cam> &cameras, std::vector<Img> &train, const std::vector<int> &fullWidth,
                     std::vector<float> &xyz, std::vector<float> &rgb, int iterations, int maxGaussians,
                     double trainStart, const std::string &splatPath, Report report, Say say, Cancelled cancelled,
                     StageResult &result, std::string *error = nullptr)
{
    auto fail = [&](const std::string &m) {
        if (error)
            *error = m;
        return false;
    };
    auto format = [](const char *fmt, double a = 0, double b = 0, double c = 0, double d = 0) {
        char buf[256];
        std::snprintf(buf, sizeof buf, fmt, a, b, c, d);
        return std::string(buf);
    };
    if (cameras.empty() || cameras.size() != train.size() || fullWidth.size() != train.size())
        return fail("Training needs one camera and one full-resolution width per image.");
    // Extent: 1.1 x the largest camera distance from the mean camera centre (Reconstructor.cpp:288-296).
    double mean[3] = {0, 0, 0};
    for (const Cam &c : cameras) {
        const auto cc = c.center();
        for (int k = 0; k < 3; ++k)
            mean[k] += cc[k] / double(cameras.size());
    }
    double extent = 0;
    for (const Cam &c : cameras) {
        const auto cc = c.center();
        const double dx = cc[0] - mean[0], dy = cc[1] - mean[1], dz = cc[2] - mean[2];
        extent = std::max(extent, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    extent = std::max(extent * 1.1, 1e-3);
    // Too few points: 10,000 random ones in a cube of 0.6 x extent (Reconstructor.cpp:298-309).
    if (xyz.size() / 3 < 1000) {
        std::mt19937 rng(1);
        std::uniform_real_distribution<float> u(-1.0f, 1.0f), u01(0.0f, 1.0f);
        const float r = float(extent) * 0.6f;
        for (int k = 0; k < 10000; ++k) {
            xyz.insert(xyz.end(), {u(rng) * r, u(rng) * r, u(rng) * r});
            rgb.insert(rgb.end(), {u01(rng), u01(rng), u01(rng)});
        }
        say("Few sparse points: added random initial points");
    }
    // Training cameras: each full-resolution camera scaled to its training image (Reconstructor.cpp:311-316).
    std::vector<TrainImage> views(train.size());
    for (std::size_t k = 0; k < train.size(); ++k) {
        Cam c = cameras[k].scaled(double(train[k].camera.width) / double(fullWidth[k]));
        c.width = train[k].camera.width;
        c.height = train[k].camera.height;
        train[k].camera = std::decay_t<decltype(train[k].camera)>::fromCamera(c);
        views[k] = imageFrom(train[k]);
    }
    // Train (Reconstructor.cpp:318-345).
    const GaussianModel init = initGaussiansFromPoints(xyz, rgb);
    TrainOptions topt = TrainOptions::forIterations(iterations);
    topt.max_gaussians = maxGaussians;
    say(format("Training %.0f iterations at %.0f px from %.0f Gaussians (scene extent %.3f)", iterations,
               double(views[0].camera.width > views[0].camera.height ? views[0].camera.width : views[0].camera.height),
               double(init.size()), extent));
    Trainer trainer(init, std::move(views), float(extent), topt);
    const auto begin = std::chrono::steady_clock::now();
    while (!trainer.done()) {
        if (cancelled())
            return fail("Cancelled");
        trainer.step();
        const TrainStats &st = trainer.stats();
        if (st.iteration % 10 == 0 || trainer.done()) {
            const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
            const double eta = elapsed / st.iteration * (iterations - st.iteration);
            report("training", trainStart + (0.98 - trainStart) * st.iteration / double(iterations),
                   format("Training %.0f / %.0f - %.1f dB - ", st.iteration, iterations, st.psnr) +
                       format("%.0f Gaussians - %.0f s left", double(st.gaussians), eta));
        }
        if (st.iteration % 250 == 0)
            say(format("iter %5.0f  loss %.4f  psnr %.2f dB  gaussians %.0f", st.iteration, st.loss, st.psnr,
                       double(st.gaussians)));
    }
    // Export (Reconstructor.cpp:347-356): the splat PLY straight from the GPU model.
    report("export", 0.98, "Saving result");
    if (u3dg_trainer_write_splat_ply(trainer.handle(), splatPath.c_str()) != U3DG_OK)
        return fail(u3dg_last_error());
    result.splatPath = splatPath;
    result.gaussians = trainer.model().size();
    result.psnr = trainer.evaluatePsnr();
    result.extent = extent;
    return true;
}

// ------------------------------------------------------------------ learned warm-start (no reference counterpart)

// The warm-start network (134 -> 128 -> 128 -> 128 -> 11). fromFile reads the 51,723 little-endian
// float32 parameters the package ships (data/warmstart_high.f32).
class WarmStartNet
{
public:
    explicit WarmStartNet(const std::vector<float> &params)
    {
        if (params.size() != std::size_t(U3DG_MLP_PARAMS))
            throw Error(U3DG_ERR_INVALID_ARG, "warm-start network needs 51723 parameters");
        check(u3dg_mlp_create(params.data(), 0, &m_h));
    }
    static WarmStartNet fromFile(const std::string &path)
    {
        std::vector<float> p(U3DG_MLP_PARAMS);
        std::FILE *f = std::fopen(path.c_str(), "rb");
        if (!f)
            throw Error(U3DG_ERR_IO, "cannot open " + path);
        const std::size_t got = std::fread(p.data(), sizeof(float), p.size(), f);
        std::fclose(f);
        if (got != p.size())
            throw Error(U3DG_ERR_IO, path + " is not a warm-start parameter file");
        return WarmStartNet(p);
    }
    WarmStartNet(WarmStartNet &&o) noexcept : m_h(o.m_h) { o.m_h = nullptr; }
    WarmStartNet(const WarmStartNet &) = delete;
    WarmStartNet &operator=(const WarmStartNet &) = delete;
    ~WarmStartNet() { u3dg_mlp_destroy(m_h); }
    u3dg_mlp *handle() const { return m_h; }

private:
    u3dg_mlp *m_h = nullptr;
};

// initGaussiansFromPoints refined by the network from the points' neighbourhoods and the training
// views; net == nullptr gives initGaussiansFromPoints exactly.
inline GaussianModel warmStartFromPoints(const WarmStartNet *net, const std::vector<float> &xyz,
                                         const std::vector<float> &rgb, const std::vector<TrainImage> &images)
{
    GaussianModel m;
    const std::size_t n = xyz.size() / 3;
    m.resize(n);
    std::vector<u3dg_image> views(images.size());
    for (std::size_t k = 0; k < images.size(); ++k)
        views[k] = {images[k].camera, images[k].rgb.data()};
    u3dg_model v = m.view();
    check(u3dg_warmstart_init(net ? net->handle() : nullptr, xyz.data(), rgb.size() >= n * 3 ? rgb.data() : nullptr,
                              n, views.data(), int(views.size()), &v));
    return m;
}

// ------------------------------------------------------------------ batched training (no reference counterpart)

// Several scenes trained at once on the current device; scene(k) gives the per-scene queries.
class BatchTrainer
{
public:
    struct Scene {
        GaussianModel initial;
        std::vector<TrainImage> images;
        float sceneExtent = 1.0f;
        TrainOptions options;
    };
    explicit BatchTrainer(std::vector<Scene> scenes, bool autotune = true) : m_scenes(std::move(scenes))
    {
        const std::size_t S = m_scenes.size();
        std::vector<u3dg_model> models(S);
        std::vector<std::vector<u3dg_image>> views(S);
        std::vector<const u3dg_image *> viewPtrs(S);
        std::vector<int> counts(S);
        std::vector<float> extents(S);
        std::vector<u3dg_train_options> opts(S);
        for (std::size_t s = 0; s < S; ++s) {
            models[s] = m_scenes[s].initial.view();
            for (const TrainImage &i : m_scenes[s].images)
                views[s].push_back({i.camera, i.rgb.data()});
            viewPtrs[s] = views[s].data();
            counts[s] = int(views[s].size());
            extents[s] = m_scenes[s].sceneExtent;
            opts[s] = m_scenes[s].options;
        }
        check(u3dg_batch_create(models.data(), viewPtrs.data(), counts.data(), extents.data(), opts.data(), int(S),
                                autotune ? 1 : 0, &m_b));
    }
    ~BatchTrainer() { u3dg_batch_destroy(m_b); }
    BatchTrainer(const BatchTrainer &) = delete;
    BatchTrainer &operator=(const BatchTrainer &) = delete;

    // Every scene advances by `count` iterations (or to the end of its schedule).
    void step(int count = 1) { check(u3dg_batch_step(m_b, count)); }
    std::size_t size() const { return m_scenes.size(); }
    int tileSize(int scene) const
    {
        int t = 0;
        check(u3dg_batch_tile_size(m_b, scene, &t, nullptr));
        return t;
    }
    // Compositing schedule chosen with the tile size: the forward kernel's pixel block edge and the
    // list entries each forward / backward thread stages per batch (u3dg_trainer_set_raster_schedule).
    struct RasterSchedule {
        int forwardBlock, forwardDepth, backwardDepth;
    };
    RasterSchedule rasterSchedule(int scene) const
    {
        RasterSchedule r{};
        check(u3dg_batch_schedule(m_b, scene, nullptr, &r.forwardBlock, &r.forwardDepth, &r.backwardDepth, nullptr));
        return r;
    }
    // The scene's model, copied back from the GPU.
    GaussianModel model(int scene) const
    {
        u3dg_trainer *t = trainer(scene);
        std::size_t n = 0;
        check(u3dg_trainer_size(t, &n));
        GaussianModel m;
        m.resize(n);
        u3dg_model v = m.view();
        check(u3dg_trainer_download(t, &v, n, &n));
        return m;
    }
    float evaluatePsnr(int scene)
    {
        float p = 0;
        check(u3dg_trainer_eval_psnr(trainer(scene), &p));
        return p;
    }

private:
    u3dg_trainer *trainer(int scene) const
    {
        u3dg_trainer *t = nullptr;
        check(u3dg_batch_trainer(m_b, scene, &t));
        return t;
    }
    std::vector<Scene> m_scenes;
    u3dg_batch *m_b = nullptr;
};

} // namespace gpu
} // namespace u3d
