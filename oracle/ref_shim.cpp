// ref_shim.cpp - C ABI over the public C++ API of the reference splat core. TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file together with the reference's own sources
// (engine/src/splat/*.cpp, engine/src/ThreadPool.cpp, engine/src/Camera.cpp of
// Abner0907/univeral_3d_reconstruction_system, read where they lie, never copied) into
// oracle/_ref/libu3dref.so. tests/ use it to pin the oracle restatement, and bench.py's reference
// arm times the reference trainer through it. Nothing in the product library links it.
//
// Only the reference's public API is called: Trainer (Trainer.h:50-65), Rasterizer
// (Rasterizer.h:38-54), photometricLoss / psnr (Loss.h:18-21), Adam (Adam.h:18-31),
// initGaussiansFromPoints (GaussianModel.h:41), writeSplatPly / readSplatPly (SplatPly.h:12-24).

#include "u3d/ThreadPool.h"
#include "u3d/splat/Adam.h"
#include "u3d/splat/Crop.h"
#include "u3d/splat/GaussianModel.h"
#include "u3d/splat/Loss.h"
#include "u3d/splat/Rasterizer.h"
#include "u3d/splat/SplatPly.h"
#include "u3d/splat/Trainer.h"

#include "../include/u3dg.h"

#include <algorithm>
#include <memory>
#include <thread>

using namespace u3d;

namespace {

GaussianModel toModel(const u3dg_model &m)
{
    GaussianModel g;
    g.resize(m.count);
    std::copy(m.means, m.means + 3 * m.count, g.means.begin());
    std::copy(m.scales, m.scales + 3 * m.count, g.scales.begin());
    std::copy(m.quats, m.quats + 4 * m.count, g.quats.begin());
    std::copy(m.opacities, m.opacities + m.count, g.opacities.begin());
    std::copy(m.colors, m.colors + 3 * m.count, g.colors.begin());
    return g;
}

void fromModel(const GaussianModel &g, u3dg_model &m)
{
    std::copy(g.means.begin(), g.means.end(), m.means);
    std::copy(g.scales.begin(), g.scales.end(), m.scales);
    std::copy(g.quats.begin(), g.quats.end(), m.quats);
    std::copy(g.opacities.begin(), g.opacities.end(), m.opacities);
    std::copy(g.colors.begin(), g.colors.end(), m.colors);
}

RenderCamera toCamera(const u3dg_camera &c)
{
    RenderCamera r;
    r.width = c.width;
    r.height = c.height;
    r.fx = c.fx;
    r.fy = c.fy;
    r.cx = c.cx;
    r.cy = c.cy;
    std::copy(c.R, c.R + 9, r.R);
    std::copy(c.t, c.t + 3, r.t);
    return r;
}

RasterSettings toSettings(const u3dg_raster_settings &s)
{
    RasterSettings r;
    r.tileSize = s.tile_size;
    r.nearPlane = s.near_plane;
    r.eps2d = s.eps2d;
    std::copy(s.background, s.background + 3, r.background);
    r.minAlpha = s.min_alpha;
    r.minTransmittance = s.min_transmittance;
    return r;
}

TrainOptions toOptions(const u3dg_train_options &o)
{
    TrainOptions t;
    t.iterations = o.iterations;
    t.maxGaussians = o.max_gaussians;
    t.ssimLambda = o.ssim_lambda;
    t.lr.means = o.lr.means;
    t.lr.scales = o.lr.scales;
    t.lr.quats = o.lr.quats;
    t.lr.opacities = o.lr.opacities;
    t.lr.colors = o.lr.colors;
    t.meansLrFinal = o.means_lr_final;
    t.densifyGradThreshold = o.densify_grad_threshold;
    t.percentDense = o.percent_dense;
    t.refineStart = o.refine_start;
    t.refineStop = o.refine_stop;
    t.refineInterval = o.refine_interval;
    t.opacityResetInterval = o.opacity_reset_interval;
    t.pruneOpacity = o.prune_opacity;
    t.seed = o.seed;
    t.raster = toSettings(o.raster);
    return t;
}

void fromOptions(const TrainOptions &t, u3dg_train_options &o)
{
    o.iterations = t.iterations;
    o.max_gaussians = t.maxGaussians;
    o.ssim_lambda = t.ssimLambda;
    o.lr = {t.lr.means, t.lr.scales, t.lr.quats, t.lr.opacities, t.lr.colors};
    o.means_lr_final = t.meansLrFinal;
    o.densify_grad_threshold = t.densifyGradThreshold;
    o.percent_dense = t.percentDense;
    o.refine_start = t.refineStart;
    o.refine_stop = t.refineStop;
    o.refine_interval = t.refineInterval;
    o.opacity_reset_interval = t.opacityResetInterval;
    o.prune_opacity = t.pruneOpacity;
    o.seed = t.seed;
    o.raster.tile_size = t.raster.tileSize;
    o.raster.near_plane = t.raster.nearPlane;
    o.raster.eps2d = t.raster.eps2d;
    std::copy(t.raster.background, t.raster.background + 3, o.raster.background);
    o.raster.min_alpha = t.raster.minAlpha;
    o.raster.min_transmittance = t.raster.minTransmittance;
}

} // namespace

extern "C" {

struct ref_raster {
    std::unique_ptr<ThreadPool> pool;
    std::unique_ptr<Rasterizer> r;
    GaussianModel model;
};

ref_raster *ref_raster_create(int threads)
{
    auto *o = new ref_raster();
    o->pool = std::make_unique<ThreadPool>(threads);
    o->r = std::make_unique<Rasterizer>(*o->pool);
    return o;
}

void ref_raster_destroy(ref_raster *o) { delete o; }

void ref_raster_forward(ref_raster *o, const u3dg_model *m, const u3dg_camera *cam, const u3dg_raster_settings *st,
                        float *rgb)
{
    o->model = toModel(*m);
    std::vector<float> out;
    o->r->forward(o->model, toCamera(*cam), toSettings(*st), out);
    std::copy(out.begin(), out.end(), rgb);
}

void ref_raster_backward(ref_raster *o, const float *dl_drgb, u3dg_model *grads, float *mean2d_grad_ndc)
{
    GaussianModel g = toModel(*grads);
    o->r->backward(o->model, dl_drgb, g, mean2d_grad_ndc);
    fromModel(g, *grads);
}

void ref_raster_radii(ref_raster *o, int *radii)
{
    const std::vector<int> &r = o->r->radii();
    std::copy(r.begin(), r.end(), radii);
}

void ref_photometric_loss(const float *render, const float *target, int w, int h, float lambda, float *grad, int threads,
                          u3dg_loss_value *out)
{
    ThreadPool pool(threads);
    const LossValue v = photometricLoss(render, target, w, h, lambda, grad, pool);
    out->total = v.total;
    out->l1 = v.l1;
    out->ssim = v.ssim;
}

float ref_psnr(const float *a, const float *b, size_t count) { return psnr(a, b, count); }

struct ref_adam {
    Adam adam;
    std::unique_ptr<ThreadPool> pool;
};

ref_adam *ref_adam_create(size_t n, int threads)
{
    auto *a = new ref_adam();
    a->pool = std::make_unique<ThreadPool>(threads);
    a->adam.reset(n);
    return a;
}

void ref_adam_step(ref_adam *a, u3dg_model *params, const u3dg_model *grads, const u3dg_learning_rates *lr)
{
    GaussianModel p = toModel(*params), g = toModel(*grads);
    LearningRates l;
    l.means = lr->means;
    l.scales = lr->scales;
    l.quats = lr->quats;
    l.opacities = lr->opacities;
    l.colors = lr->colors;
    a->adam.step(p, g, l, *a->pool);
    fromModel(p, *params);
}

void ref_adam_compact(ref_adam *a, const uint8_t *keep, size_t n) { a->adam.compact(std::vector<uint8_t>(keep, keep + n)); }
void ref_adam_grow(ref_adam *a, size_t count) { a->adam.grow(count); }
void ref_adam_reset_opacity_moments(ref_adam *a) { a->adam.resetOpacityMoments(); }
void ref_adam_destroy(ref_adam *a) { delete a; }

struct ref_trainer {
    std::unique_ptr<ThreadPool> pool;
    std::unique_ptr<Trainer> t;
};

ref_trainer *ref_trainer_create(const u3dg_model *initial, const u3dg_image *images, int count, float extent,
                                const u3dg_train_options *o, int threads)
{
    auto *r = new ref_trainer();
    r->pool = std::make_unique<ThreadPool>(threads);
    std::vector<TrainImage> imgs(size_t(count > 0 ? count : 0));
    for (int k = 0; k < count; ++k) {
        imgs[size_t(k)].camera = toCamera(images[k].camera);
        const size_t sz = size_t(images[k].camera.width) * size_t(images[k].camera.height) * 3;
        imgs[size_t(k)].rgb.assign(images[k].rgb, images[k].rgb + sz);
    }
    r->t = std::make_unique<Trainer>(toModel(*initial), std::move(imgs), extent, toOptions(*o), *r->pool);
    return r;
}

void ref_trainer_step(ref_trainer *r, int count)
{
    for (int k = 0; k < count; ++k)
        r->t->step();
}

void ref_trainer_stats(ref_trainer *r, u3dg_train_stats *out)
{
    const TrainStats &s = r->t->stats();
    out->iteration = s.iteration;
    out->loss = s.loss;
    out->psnr = s.psnr;
    out->gaussians = s.gaussians;
}

int ref_trainer_done(ref_trainer *r) { return r->t->done() ? 1 : 0; }
size_t ref_trainer_size(ref_trainer *r) { return r->t->model().size(); }
void ref_trainer_download(ref_trainer *r, u3dg_model *out) { fromModel(r->t->model(), *out); }
float ref_trainer_eval_psnr(ref_trainer *r) { return r->t->evaluatePsnr(); }

void ref_trainer_render(ref_trainer *r, const u3dg_camera *cam, float *rgb)
{
    std::vector<float> out;
    r->t->render(toCamera(*cam), out);
    std::copy(out.begin(), out.end(), rgb);
}

void ref_trainer_destroy(ref_trainer *r) { delete r; }

int ref_pool_threads(int threads)
{
    ThreadPool p(threads);
    return p.size();
}

void ref_init_from_points(const float *xyz, const float *rgb, size_t n, u3dg_model *out)
{
    std::vector<float> x(xyz, xyz + 3 * n), c;
    if (rgb)
        c.assign(rgb, rgb + 3 * n);
    const GaussianModel g = initGaussiansFromPoints(x, c);
    fromModel(g, *out);
}

void ref_options_for_iterations(int iterations, u3dg_train_options *out)
{
    fromOptions(iterations > 0 ? TrainOptions::forIterations(iterations) : TrainOptions(), *out);
}

int ref_write_splat_ply(const char *path, const u3dg_model *m)
{
    return writeSplatPly(path, toModel(*m)) ? 1 : 0;
}

// Two calls: out == NULL returns the count only.
int ref_read_splat_ply(const char *path, u3dg_model *out, size_t *count, int *is_splat)
{
    GaussianModel g;
    bool splat = false;
    if (!readSplatPly(path, g, nullptr, &splat))
        return 0;
    *count = g.size();
    if (is_splat)
        *is_splat = splat ? 1 : 0;
    if (out)
        fromModel(g, *out);
    return 1;
}

size_t ref_crop_model(const u3dg_model *model, const u3dg_crop_box *box, float min_opacity, u3dg_model *out)
{
    CropBox b;
    for (int k = 0; k < 3; ++k) {
        b.min[k] = box->min[k];
        b.max[k] = box->max[k];
    }
    const GaussianModel g = cropModel(toModel(*model), b, min_opacity);
    if (out)
        fromModel(g, *out);
    return g.size();
}

void ref_crop_box(const u3dg_model *model, float lo, float hi, float margin, int bounds, u3dg_crop_box *box)
{
    const CropBox b = bounds ? modelBounds(toModel(*model)) : suggestCropBox(toModel(*model), lo, hi, margin);
    for (int k = 0; k < 3; ++k) {
        box->min[k] = b.min[k];
        box->max[k] = b.max[k];
    }
}

} // extern "C"
