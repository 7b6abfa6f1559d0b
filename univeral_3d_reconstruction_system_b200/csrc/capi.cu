// capi.cu - the extern "C" entry points of include/u3dg.h. Every call catches every C++ exception
// and turns it into a status code plus a thread-local message (u3dg_last_error).

#include "engine.h"
#include "host_io.h"

#include <cstring>
#include <memory>
#include <mutex>

using namespace u3dg;

namespace {

template <class F>
int guarded(F &&f)
{
    return guardedCall(std::forward<F>(f));
}

void requireDevice()
{
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw StatusError(U3DG_ERR_NO_DEVICE, "no CUDA device is available");
    }
}

void requireModel(const u3dg_model *m, const char *what)
{
    if (!m)
        throw StatusError(U3DG_ERR_INVALID_ARG, std::string(what) + " is NULL");
    if (m->count > 0 && (!m->means || !m->scales || !m->quats || !m->opacities || !m->colors))
        throw StatusError(U3DG_ERR_INVALID_ARG, std::string(what) + " has NULL arrays");
    if (m->count > size_t(INT_MAX / 64))
        throw StatusError(U3DG_ERR_CAPACITY, std::string(what) + " has too many Gaussians");
}

// A model uploaded into a 14-float-per-Gaussian arena (capacity == count).
struct DevModel {
    DevBuf<float> buf;
    size_t cap = 0;
    void upload(const u3dg_model &m, cudaStream_t s)
    {
        cap = std::max<size_t>(m.count, 1);
        buf.reserve(14 * cap, true);
        const Params P = paramsAt(buf.p, cap);
        const size_t n = m.count;
        if (n == 0)
            return;
        U3DG_CUDA(cudaMemcpyAsync(P.means, m.means, n * 12, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(P.scales, m.scales, n * 12, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(P.quats, m.quats, n * 16, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(P.opac, m.opacities, n * 4, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(P.colors, m.colors, n * 12, cudaMemcpyHostToDevice, s));
    }
    void download(u3dg_model &m, size_t n, cudaStream_t s) const
    {
        const Params P = paramsAt(buf.p, cap);
        if (n == 0)
            return;
        U3DG_CUDA(cudaMemcpyAsync(m.means, P.means, n * 12, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(m.scales, P.scales, n * 12, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(m.quats, P.quats, n * 16, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(m.opacities, P.opac, n * 4, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(m.colors, P.colors, n * 12, cudaMemcpyDeviceToHost, s));
    }
    Params params() const { return paramsAt(buf.p, cap); }
};

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { U3DG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream()
    {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
    void sync() { U3DG_CUDA(cudaStreamSynchronize(s)); }
};

} // namespace

struct u3dg_rasterizer {
    int device = 0;
    Stream stream;
    RasterWorkspace ws;
    DevModel model;
    DevBuf<float> dl;
    bool haveForward = false;
};

struct u3dg_adam {
    int device = 0;
    Stream stream;
    size_t count = 0;
    DevBuf<float> m, v, p, g; // group-major arenas of 14 * count floats
    int step = 0;
};

extern "C" {

const char *u3dg_last_error(void) { return lastError(); }

int u3dg_abi_version(void) { return U3DG_ABI_VERSION; }

uint64_t u3dg_launch_count(void) { return uint64_t(launchCount()); }

int u3dg_device_count(void)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count;
}

int u3dg_set_device(int device)
{
    return guarded([&] {
        requireDevice();
        U3DG_CUDA(cudaSetDevice(device));
    });
}

void u3dg_raster_settings_default(u3dg_raster_settings *out)
{
    if (!out)
        return;
    u3dg_raster_settings s{};
    s.tile_size = 16;
    s.near_plane = 0.01f;
    s.eps2d = 0.3f;
    s.background[0] = s.background[1] = s.background[2] = 0.0f;
    s.min_alpha = 1.0f / 255.0f;
    s.min_transmittance = 1e-4f;
    *out = s;
}

void u3dg_train_options_default(u3dg_train_options *out)
{
    if (!out)
        return;
    u3dg_train_options o{};
    o.iterations = 3000;
    o.max_gaussians = 200000;
    o.ssim_lambda = 0.2f;
    o.lr.means = 1.6e-4f;
    o.lr.scales = 5e-3f;
    o.lr.quats = 1e-3f;
    o.lr.opacities = 5e-2f;
    o.lr.colors = 2.5e-3f;
    o.means_lr_final = 1.6e-6f;
    o.densify_grad_threshold = 2e-4f;
    o.percent_dense = 0.01f;
    o.refine_start = 500;
    o.refine_stop = 15000;
    o.refine_interval = 100;
    o.opacity_reset_interval = 3000;
    o.prune_opacity = 0.005f;
    o.seed = 42;
    u3dg_raster_settings_default(&o.raster);
    *out = o;
}

void u3dg_train_options_for_iterations(int iterations, u3dg_train_options *out)
{
    if (!out)
        return;
    u3dg_train_options_default(out);
    out->iterations = std::max(1, iterations);
    out->refine_start = std::min(500, out->iterations / 10);
    out->refine_stop = out->iterations * 6 / 10;
    out->refine_interval = 100;
    out->opacity_reset_interval = out->iterations >= 6000 ? 3000 : 0;
}

// ------------------------------------------------------------------ trainer

int u3dg_trainer_create(const u3dg_model *initial, const u3dg_image *images, int image_count, float scene_extent,
                        const u3dg_train_options *options, u3dg_trainer **out)
{
    return guarded([&] {
        if (!out || !options)
            throw StatusError(U3DG_ERR_INVALID_ARG, "options and out must not be NULL");
        *out = nullptr;
        requireModel(initial, "initial model");
        requireDevice();
        auto t = std::make_unique<u3dg_trainer>();
        t->impl = std::make_unique<TrainerImpl>(*initial, images, image_count, scene_extent, *options);
        *out = t.release();
    });
}

int u3dg_trainer_create_background_upload(const u3dg_model *initial, const u3dg_image *images, int image_count,
                                          float scene_extent, const u3dg_train_options *options,
                                          u3dg_trainer **out)
{
    return guarded([&] {
        if (!out || !options)
            throw StatusError(U3DG_ERR_INVALID_ARG, "options and out must not be NULL");
        *out = nullptr;
        requireModel(initial, "initial model");
        requireDevice();
        auto t = std::make_unique<u3dg_trainer>();
        t->impl = std::make_unique<TrainerImpl>(*initial, images, image_count, scene_extent, *options, true);
        *out = t.release();
    });
}

static TrainerImpl &impl(u3dg_trainer *t)
{
    if (!t || !t->impl)
        throw StatusError(U3DG_ERR_INVALID_ARG, "trainer is NULL");
    U3DG_CUDA(cudaSetDevice(t->impl->device));
    return *t->impl;
}

int u3dg_trainer_wait_uploads(u3dg_trainer *trainer)
{
    return guarded([&] { impl(trainer).waitUploads(); });
}

int u3dg_trainer_step(u3dg_trainer *trainer, int count)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (count > 0)
            t.stepTo(t.iteration + count);
    });
}

int u3dg_trainer_done(const u3dg_trainer *trainer, int *done)
{
    return guarded([&] {
        if (!trainer || !trainer->impl || !done)
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        *done = trainer->impl->done() ? 1 : 0;
    });
}

int u3dg_trainer_iteration(const u3dg_trainer *trainer, int *iteration)
{
    return guarded([&] {
        if (!trainer || !trainer->impl || !iteration)
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        *iteration = trainer->impl->iteration;
    });
}

int u3dg_trainer_stats(u3dg_trainer *trainer, u3dg_train_stats *out)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        t.finish();
        out->iteration = t.iteration;
        out->loss = t.hStats.p->loss;
        out->psnr = t.hStats.p->psnr;
        out->gaussians = uint64_t(t.n);
    });
}

int u3dg_trainer_size(u3dg_trainer *trainer, size_t *count)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!count)
            throw StatusError(U3DG_ERR_INVALID_ARG, "count is NULL");
        t.finish();
        *count = size_t(t.n);
    });
}

int u3dg_trainer_download(u3dg_trainer *trainer, u3dg_model *out, size_t capacity, size_t *count)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        t.finish();
        if (count)
            *count = size_t(t.n);
        if (size_t(t.n) > capacity)
            throw StatusError(U3DG_ERR_CAPACITY, "output capacity " + std::to_string(capacity) + " < model size " +
                                                     std::to_string(t.n));
        requireModel(out, "output model");
        t.download(*out);
    });
}

int u3dg_trainer_write_splat_ply(u3dg_trainer *trainer, const char *path)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!path)
            throw StatusError(U3DG_ERR_INVALID_ARG, "path is NULL");
        t.finish();
        HostModel m;
        m.resize(size_t(t.n));
        u3dg_model v{m.means.data(), m.scales.data(), m.quats.data(), m.opac.data(), m.colors.data(), m.size()};
        t.download(v);
        std::string err;
        if (!writeSplatPlyHost(path, v, &err))
            throw StatusError(U3DG_ERR_IO, err);
    });
}

int u3dg_trainer_eval_psnr(u3dg_trainer *trainer, float *psnr)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!psnr)
            throw StatusError(U3DG_ERR_INVALID_ARG, "psnr is NULL");
        *psnr = t.evaluatePsnr();
    });
}

int u3dg_trainer_render(u3dg_trainer *trainer, const u3dg_camera *camera, float *rgb)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!camera || !rgb)
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        t.render(*camera, rgb);
    });
}

int u3dg_trainer_stream(u3dg_trainer *trainer, void **stream)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!stream)
            throw StatusError(U3DG_ERR_INVALID_ARG, "stream is NULL");
        *stream = reinterpret_cast<void *>(t.stream);
    });
}

int u3dg_trainer_synchronize(u3dg_trainer *trainer)
{
    return guarded([&] { impl(trainer).sync(); });
}

int u3dg_trainer_set_profiling(u3dg_trainer *trainer, int enable)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (enable && !t.timer)
            t.timer = new PhaseTimer();
        t.profiling = enable != 0;
    });
}

int u3dg_trainer_phase_times(u3dg_trainer *trainer, u3dg_phase_times *out)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        t.sync();
        if (t.timer) {
            *out = t.timer->acc;
            t.timer->acc = u3dg_phase_times{};
        } else {
            *out = u3dg_phase_times{};
        }
    });
}

int u3dg_trainer_set_intersection_capacity(u3dg_trainer *trainer, size_t capacity)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        t.finish();
        capacity = std::max<size_t>(capacity, 1024);
        if (capacity > size_t(INT_MAX / 16))
            throw StatusError(U3DG_ERR_CAPACITY, "capacity too large");
        t.ws.iKeys0.release();
        t.ws.icap = 0;
        t.ws.reserveIntersections(capacity);
    });
}

int u3dg_trainer_replays(u3dg_trainer *trainer, int *replays)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!replays)
            throw StatusError(U3DG_ERR_INVALID_ARG, "replays is NULL");
        *replays = t.replays;
    });
}

int u3dg_trainer_set_graphs(u3dg_trainer *trainer, int enable)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        t.useGraphs = enable != 0;
        if (!t.useGraphs)
            t.resetGraphs();
    });
}

int u3dg_trainer_set_raster_schedule(u3dg_trainer *trainer, int forward_block, int forward_depth,
                                     int backward_depth)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (forward_block != 8 && forward_block != 16)
            throw StatusError(U3DG_ERR_INVALID_ARG, "forward block must be 8 or 16");
        for (int d : {forward_depth, backward_depth})
            if (d != 1 && d != 2)
                throw StatusError(U3DG_ERR_INVALID_ARG, "batch depth must be 1 or 2");
        t.finish();
        t.ws.forwardBlock = forward_block;
        t.ws.forwardDepth = forward_depth;
        t.ws.backwardDepth = backward_depth;
        t.resetGraphs(); // its kernels were recorded for the other depth
    });
}

int u3dg_trainer_set_tile_culling(u3dg_trainer *trainer, int enable)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        t.finish();
        t.ws.cullTiles = enable != 0;
        t.resetGraphs(); // its emission kernels were recorded with the other setting
    });
}

int u3dg_trainer_graph_launches(u3dg_trainer *trainer, long long *launches)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!launches)
            throw StatusError(U3DG_ERR_INVALID_ARG, "launches is NULL");
        *launches = t.graphChunks;
    });
}

int u3dg_trainer_time_steps(u3dg_trainer *trainer, int count, float *ms)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        if (!ms)
            throw StatusError(U3DG_ERR_INVALID_ARG, "ms is NULL");
        cudaEvent_t a, b;
        U3DG_CUDA(cudaEventCreate(&a));
        U3DG_CUDA(cudaEventCreate(&b));
        t.finish();
        // The first run's graph is recorded before the timed region (recording executes nothing).
        if (count > 0)
            t.primeGraph(t.iteration + count);
        U3DG_CUDA(cudaEventRecord(a, t.stream));
        if (count > 0)
            t.stepTo(t.iteration + count);
        U3DG_CUDA(cudaEventRecord(b, t.stream));
        U3DG_CUDA(cudaEventSynchronize(b));
        U3DG_CUDA(cudaEventElapsedTime(ms, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    });
}

void u3dg_trainer_destroy(u3dg_trainer *trainer)
{
    if (!trainer || trainer->ownedByBatch)
        return;
    try {
        if (trainer->impl)
            cudaSetDevice(trainer->impl->device);
        delete trainer;
    } catch (...) {
    }
}

// ------------------------------------------------------------------ rasterizer

int u3dg_rasterizer_create(u3dg_rasterizer **out)
{
    return guarded([&] {
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        *out = nullptr;
        requireDevice();
        auto r = std::make_unique<u3dg_rasterizer>();
        U3DG_CUDA(cudaGetDevice(&r->device));
        *out = r.release();
    });
}

static u3dg_rasterizer &rz(u3dg_rasterizer *r)
{
    if (!r)
        throw StatusError(U3DG_ERR_INVALID_ARG, "rasterizer is NULL");
    U3DG_CUDA(cudaSetDevice(r->device));
    return *r;
}

static void rasterForward(u3dg_rasterizer &r, const u3dg_model *model, const float *shRest, int degree,
                          const u3dg_camera *camera, const u3dg_raster_settings *settings, float *rgb)
{
    requireModel(model, "model");
    if (!camera || !settings || !rgb)
        throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
    if (degree < 0 || degree > 3)
        throw StatusError(U3DG_ERR_INVALID_ARG, "SH degree must be 0..3");
    checkSettings(*settings);
    checkCamera(*camera);
    cudaStream_t s = r.stream.s;
    r.model.upload(*model, s);
    DevBuf<float> sh;
    const float *shDev = nullptr;
    if (shRest && degree > 0 && model->count > 0) {
        const size_t K = size_t((degree + 1) * (degree + 1) - 1);
        sh.reserve(model->count * K * 3, true);
        U3DG_CUDA(cudaMemcpyAsync(sh.p, shRest, model->count * K * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
        shDev = sh.p;
    }
    r.ws.forwardChecked(r.model.params(), int(model->count), *camera, *settings, shDev, degree, s);
    U3DG_CUDA(cudaGetLastError());
    U3DG_CUDA(cudaMemcpyAsync(rgb, r.ws.rgb.p, size_t(camera->width) * camera->height * 3 * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
    r.stream.sync();
    r.haveForward = true;
}

int u3dg_rasterizer_forward(u3dg_rasterizer *r, const u3dg_model *model, const u3dg_camera *camera,
                            const u3dg_raster_settings *settings, float *rgb)
{
    return guarded([&] { rasterForward(rz(r), model, nullptr, 0, camera, settings, rgb); });
}

int u3dg_rasterizer_backward(u3dg_rasterizer *r, const u3dg_model *model, const float *dl_drgb, u3dg_model *grads,
                             float *mean2d_grad_ndc)
{
    return guarded([&] {
        u3dg_rasterizer &R = rz(r);
        if (!R.haveForward)
            throw StatusError(U3DG_ERR_STATE, "backward before forward");
        requireModel(model, "model");
        requireModel(grads, "grads");
        if (!dl_drgb)
            throw StatusError(U3DG_ERR_INVALID_ARG, "dl_drgb is NULL");
        if (model->count != size_t(R.ws.n) || grads->count != model->count)
            throw StatusError(U3DG_ERR_INVALID_ARG, "model / grads size differs from the last forward");
        cudaStream_t s = R.stream.s;
        const size_t n = model->count;
        const size_t P = size_t(R.ws.cam.width) * R.ws.cam.height;
        R.model.upload(*model, s);
        R.dl.reserve(P * 3);
        U3DG_CUDA(cudaMemcpyAsync(R.dl.p, dl_drgb, P * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
        DevModel g;
        g.upload(*grads, s);
        DevBuf<float> ndc;
        ndc.reserve(std::max<size_t>(n, 1), true);
        if (mean2d_grad_ndc && n > 0)
            U3DG_CUDA(cudaMemcpyAsync(ndc.p, mean2d_grad_ndc, n * sizeof(float), cudaMemcpyHostToDevice, s));
        R.ws.backwardComposite(R.dl.p, s);
        ChainArgs a = R.ws.chainArgs(R.model.params());
        a.grads = g.params();
        a.gradAccum = mean2d_grad_ndc ? ndc.p : nullptr;
        a.gradCount = nullptr;
        launchChain(a, false, s);
        U3DG_CUDA(cudaGetLastError());
        g.download(*grads, n, s);
        if (mean2d_grad_ndc && n > 0)
            U3DG_CUDA(cudaMemcpyAsync(mean2d_grad_ndc, ndc.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
        R.stream.sync();
    });
}

int u3dg_rasterizer_radii(u3dg_rasterizer *r, int *radii, size_t n)
{
    return guarded([&] {
        u3dg_rasterizer &R = rz(r);
        if (!R.haveForward || n != size_t(R.ws.n) || (!radii && n))
            throw StatusError(U3DG_ERR_INVALID_ARG, "radii needs the size of the last forward");
        if (n)
            U3DG_CUDA(cudaMemcpyAsync(radii, R.ws.radius.p, n * sizeof(int), cudaMemcpyDeviceToHost, R.stream.s));
        R.stream.sync();
    });
}

int u3dg_rasterizer_projection(u3dg_rasterizer *r, size_t n, float *mean2d, float *conic, float *cov2d, float *depth,
                               float *rgb, float *alpha, int *rect, uint8_t *flags)
{
    return guarded([&] {
        u3dg_rasterizer &R = rz(r);
        if (!R.haveForward || n != size_t(R.ws.n))
            throw StatusError(U3DG_ERR_INVALID_ARG, "projection needs the size of the last forward");
        cudaStream_t s = R.stream.s;
        std::vector<SplatRec> rec(n);
        std::vector<int4> rc(n);
        std::vector<float4> cv(n);
        if (n) {
            U3DG_CUDA(cudaMemcpyAsync(rec.data(), R.ws.rec.p, n * sizeof(SplatRec), cudaMemcpyDeviceToHost, s));
            U3DG_CUDA(cudaMemcpyAsync(cv.data(), R.ws.cov2d.p, n * sizeof(float4), cudaMemcpyDeviceToHost, s));
            U3DG_CUDA(cudaMemcpyAsync(rc.data(), R.ws.rect.p, n * sizeof(int4), cudaMemcpyDeviceToHost, s));
            if (depth)
                U3DG_CUDA(cudaMemcpyAsync(depth, R.ws.depth.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
            if (flags)
                U3DG_CUDA(cudaMemcpyAsync(flags, R.ws.flags.p, n * sizeof(uint8_t), cudaMemcpyDeviceToHost, s));
        }
        std::vector<int> rad(n);
        if (n)
            U3DG_CUDA(cudaMemcpyAsync(rad.data(), R.ws.radius.p, n * sizeof(int), cudaMemcpyDeviceToHost, s));
        R.stream.sync();
        for (size_t i = 0; i < n; ++i) {
            const bool vis = rad[i] > 0;
            const SplatRec &q = rec[i];
            if (mean2d) { mean2d[2 * i] = vis ? q.mx : 0; mean2d[2 * i + 1] = vis ? q.my : 0; }
            if (conic) { conic[3 * i] = vis ? q.A : 0; conic[3 * i + 1] = vis ? q.B : 0; conic[3 * i + 2] = vis ? q.C : 0; }
            if (cov2d) { cov2d[3 * i] = vis ? cv[i].x : 0; cov2d[3 * i + 1] = vis ? cv[i].y : 0; cov2d[3 * i + 2] = vis ? cv[i].z : 0; }
            if (rgb) { rgb[3 * i] = vis ? q.r : 0; rgb[3 * i + 1] = vis ? q.g : 0; rgb[3 * i + 2] = vis ? q.b : 0; }
            if (alpha) alpha[i] = vis ? q.alpha : 0;
            if (depth && !vis) depth[i] = 0;
            if (rect) { rect[4 * i] = rc[i].x; rect[4 * i + 1] = rc[i].y; rect[4 * i + 2] = rc[i].z; rect[4 * i + 3] = rc[i].w; }
        }
    });
}

int u3dg_rasterizer_tiles(u3dg_rasterizer *r, int *tiles_x, int *tiles_y, int *offsets, size_t offsets_capacity, int *list,
                          size_t list_capacity, size_t *list_length)
{
    return guarded([&] {
        u3dg_rasterizer &R = rz(r);
        if (!R.haveForward)
            throw StatusError(U3DG_ERR_STATE, "tiles before forward");
        const size_t tiles = size_t(R.ws.tilesX) * R.ws.tilesY;
        if (tiles_x) *tiles_x = R.ws.tilesX;
        if (tiles_y) *tiles_y = R.ws.tilesY;
        if (list_length) *list_length = size_t(R.ws.total());
        cudaStream_t s = R.stream.s;
        if (offsets && offsets_capacity >= tiles + 1)
            U3DG_CUDA(cudaMemcpyAsync(offsets, R.ws.tileOffsets.p, (tiles + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
        const size_t L = std::min(list_capacity, size_t(R.ws.total()));
        if (list && L)
            // The Gaussian ids: the first int of each (id, emission index) entry.
            U3DG_CUDA(cudaMemcpy2DAsync(list, sizeof(int), R.ws.entries.p, sizeof(int2), sizeof(int), L,
                                        cudaMemcpyDeviceToHost, s));
        R.stream.sync();
    });
}

int u3dg_rasterizer_pixel_state(u3dg_rasterizer *r, float *final_t, int *n_contrib, size_t pixels)
{
    return guarded([&] {
        u3dg_rasterizer &R = rz(r);
        const size_t P = size_t(R.ws.cam.width) * R.ws.cam.height;
        if (!R.haveForward || pixels != P)
            throw StatusError(U3DG_ERR_INVALID_ARG, "pixel_state needs width*height of the last forward");
        if (final_t)
            U3DG_CUDA(cudaMemcpyAsync(final_t, R.ws.finalT.p, P * sizeof(float), cudaMemcpyDeviceToHost, R.stream.s));
        if (n_contrib)
            U3DG_CUDA(cudaMemcpyAsync(n_contrib, R.ws.nContrib.p, P * sizeof(int), cudaMemcpyDeviceToHost, R.stream.s));
        R.stream.sync();
    });
}

int u3dg_rasterizer_set_tile_culling(u3dg_rasterizer *r, int enable)
{
    return guarded([&] {
        u3dg_rasterizer &R = rz(r);
        R.ws.cullTiles = enable != 0;
        R.haveForward = false; // the next backward needs a forward with the new lists
    });
}

void u3dg_rasterizer_destroy(u3dg_rasterizer *r)
{
    if (!r)
        return;
    cudaSetDevice(r->device);
    delete r;
}

int u3dg_bin_tiles(const float *depth, const int *radius, const int *rect, size_t n, int tiles_x, int tiles_y,
                   int *offsets, int *list, size_t list_capacity, size_t *list_length)
{
    return guarded([&] {
        if (n > 0 && (!depth || !radius || !rect))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL input");
        if (tiles_x <= 0 || tiles_y <= 0 || !offsets)
            throw StatusError(U3DG_ERR_INVALID_ARG, "tile grid must be non-empty and offsets non-NULL");
        if (n > size_t(INT_MAX / 64))
            throw StatusError(U3DG_ERR_CAPACITY, "too many Gaussians");
        requireDevice();
        Stream st;
        RasterWorkspace ws;
        ws.n = int(n);
        ws.tilesX = tiles_x;
        ws.tilesY = tiles_y;
        const size_t nn = std::max<size_t>(n, 1);
        ws.depthKey.reserve(nn);
        ws.depthPairs[0].reserve(nn);
        ws.depthPairs[1].reserve(nn);
        ws.depthOrder.reserve(nn);
        ws.rect.reserve(nn);
        ws.radius.reserve(nn);
        ws.cnt.reserve(nn);
        ws.offs.reserve(nn + 1);
        ws.scanPartial.reserve(scanPartialEntries(int(nn)) + 1);
        std::vector<uint32_t> keys(n);
        std::vector<int4> rc(n);
        std::vector<int> cnt(n); // tiles per Gaussian: its whole rectangle (no culling at this boundary)
        for (size_t i = 0; i < n; ++i) {
            uint32_t b;
            std::memcpy(&b, &depth[i], 4);
            keys[i] = radius[i] > 0 ? b : 0xFFFFFFFFu;
            rc[i] = make_int4(rect[4 * i], rect[4 * i + 1], rect[4 * i + 2], rect[4 * i + 3]);
            if (radius[i] > 0 && (rc[i].x < 0 || rc[i].y < 0 || rc[i].z > tiles_x || rc[i].w > tiles_y ||
                                  rc[i].x >= rc[i].z || rc[i].y >= rc[i].w))
                throw StatusError(U3DG_ERR_INVALID_ARG, "rect of a visible Gaussian is outside the tile grid");
            cnt[i] = radius[i] > 0 ? (rc[i].z - rc[i].x) * (rc[i].w - rc[i].y) : 0;
        }
        ws.reserveIntersections(std::max<size_t>(size_t(1) << 16, 4 * nn));
        for (int attempt = 0;; ++attempt) {
            // The depth sort overwrites its keys, so every attempt uploads them again.
            if (n) {
                U3DG_CUDA(cudaMemcpyAsync(ws.depthKey.p, keys.data(), n * 4, cudaMemcpyHostToDevice, st.s));
                U3DG_CUDA(cudaMemcpyAsync(ws.rect.p, rc.data(), n * sizeof(int4), cudaMemcpyHostToDevice, st.s));
                U3DG_CUDA(cudaMemcpyAsync(ws.radius.p, radius, n * sizeof(int), cudaMemcpyHostToDevice, st.s));
                U3DG_CUDA(cudaMemcpyAsync(ws.cnt.p, cnt.data(), n * sizeof(int), cudaMemcpyHostToDevice, st.s));
            }
            ws.clearCounts(st.s);
            ws.bin(st.s, 0);
            U3DG_CUDA(cudaGetLastError());
            U3DG_CUDA(cudaMemcpyAsync(ws.hostCounts.p, ws.counts.p, sizeof(BinCounts), cudaMemcpyDeviceToHost, st.s));
            st.sync();
            if (ws.hostCounts.p->abortIter < 0)
                break;
            if (attempt >= 8)
                throw StatusError(U3DG_ERR_CAPACITY, "intersection buffers could not be sized");
            ws.reserveIntersections(size_t(ws.hostCounts.p->need) + size_t(ws.hostCounts.p->need) / 4);
        }
        const size_t tiles = size_t(tiles_x) * tiles_y;
        U3DG_CUDA(cudaMemcpyAsync(offsets, ws.tileOffsets.p, (tiles + 1) * sizeof(int), cudaMemcpyDeviceToHost, st.s));
        const size_t L = std::min(list_capacity, size_t(ws.total()));
        if (list && L)
            U3DG_CUDA(cudaMemcpy2DAsync(list, sizeof(int), ws.entries.p, sizeof(int2), sizeof(int), L,
                                        cudaMemcpyDeviceToHost, st.s));
        if (list_length)
            *list_length = size_t(ws.total());
        st.sync();
    });
}

// ------------------------------------------------------------------ loss

int u3dg_photometric_loss(const float *render, const float *target, int width, int height, float lambda, float *grad,
                          u3dg_loss_value *out)
{
    return guarded([&] {
        if (!render || !target || !grad || width <= 0 || height <= 0)
            throw StatusError(U3DG_ERR_INVALID_ARG, "invalid loss arguments");
        requireDevice();
        Stream st;
        const size_t P = size_t(width) * height;
        DevBuf<float> dr, dt, dg, dabc;
        DevBuf<double> sums;
        DevBuf<float> vals;
        dr.reserve(P * 3, true);
        dt.reserve(P * 3, true);
        dg.reserve(P * 3, true);
        dabc.reserve(P * 9, true);
        const int blocks = lossBlocks(width, height);
        sums.reserve(size_t(blocks) * 3, true);
        vals.reserve(4, true);
        U3DG_CUDA(cudaMemcpyAsync(dr.p, render, P * 12, cudaMemcpyHostToDevice, st.s));
        U3DG_CUDA(cudaMemcpyAsync(dt.p, target, P * 12, cudaMemcpyHostToDevice, st.s));
        LossScratch ls{dabc.p, sums.p, blocks};
        launchLoss(dr.p, dt.p, nullptr, width, height, lambda, dg.p, ls, st.s);
        launchLossFinalize(ls, width, height, lambda, nullptr, 0, nullptr, vals.p, vals.p + 3, st.s);
        U3DG_CUDA(cudaGetLastError());
        float v[4];
        U3DG_CUDA(cudaMemcpyAsync(v, vals.p, sizeof(v), cudaMemcpyDeviceToHost, st.s));
        U3DG_CUDA(cudaMemcpyAsync(grad, dg.p, P * 12, cudaMemcpyDeviceToHost, st.s));
        st.sync();
        if (out) {
            out->total = v[0];
            out->l1 = v[1];
            out->ssim = v[2];
        }
    });
}

int u3dg_psnr(const float *a, const float *b, size_t count, float *out)
{
    return guarded([&] {
        if ((count && (!a || !b)) || !out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        requireDevice();
        Stream st;
        DevBuf<float> da, db;
        DevBuf<double> sums;
        da.reserve(std::max<size_t>(count, 1), true);
        db.reserve(std::max<size_t>(count, 1), true);
        sums.reserve(297, true);
        double total = 0.0;
        if (count) {
            U3DG_CUDA(cudaMemcpyAsync(da.p, a, count * 4, cudaMemcpyHostToDevice, st.s));
            U3DG_CUDA(cudaMemcpyAsync(db.p, b, count * 4, cudaMemcpyHostToDevice, st.s));
            launchPsnrF(da.p, db.p, count, sums.p, st.s);
            U3DG_CUDA(cudaGetLastError());
            U3DG_CUDA(cudaMemcpyAsync(&total, sums.p + 296, sizeof(double), cudaMemcpyDeviceToHost, st.s));
        }
        st.sync();
        const double mse = total / double(std::max<size_t>(count, 1));
        *out = mse <= 1e-12 ? 99.0f : float(-10.0 * std::log10(mse));
    });
}

// ------------------------------------------------------------------ Adam

int u3dg_adam_create(size_t count, u3dg_adam **out)
{
    return guarded([&] {
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        *out = nullptr;
        requireDevice();
        auto a = std::make_unique<u3dg_adam>();
        U3DG_CUDA(cudaGetDevice(&a->device));
        a->count = count;
        const size_t c = std::max<size_t>(count, 1);
        a->m.reserve(14 * c, true);
        a->v.reserve(14 * c, true);
        U3DG_CUDA(cudaMemsetAsync(a->m.p, 0, 14 * c * 4, a->stream.s));
        U3DG_CUDA(cudaMemsetAsync(a->v.p, 0, 14 * c * 4, a->stream.s));
        a->stream.sync();
        *out = a.release();
    });
}

static u3dg_adam &adamOf(u3dg_adam *a)
{
    if (!a)
        throw StatusError(U3DG_ERR_INVALID_ARG, "adam is NULL");
    U3DG_CUDA(cudaSetDevice(a->device));
    return *a;
}

// Host SoA model <-> 14-float arena of capacity c.
static void uploadGroups(float *base, size_t c, const u3dg_model &m, cudaStream_t s)
{
    const Params P = paramsAt(base, c);
    const size_t n = m.count;
    if (!n)
        return;
    U3DG_CUDA(cudaMemcpyAsync(P.means, m.means, n * 12, cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.scales, m.scales, n * 12, cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.quats, m.quats, n * 16, cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.opac, m.opacities, n * 4, cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.colors, m.colors, n * 12, cudaMemcpyHostToDevice, s));
}

static void downloadGroups(const float *base, size_t c, size_t n, u3dg_model &m, cudaStream_t s)
{
    const Params P = paramsAt(const_cast<float *>(base), c);
    if (!n)
        return;
    U3DG_CUDA(cudaMemcpyAsync(m.means, P.means, n * 12, cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.scales, P.scales, n * 12, cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.quats, P.quats, n * 16, cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.opacities, P.opac, n * 4, cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.colors, P.colors, n * 12, cudaMemcpyDeviceToHost, s));
}

int u3dg_adam_step(u3dg_adam *adam, u3dg_model *params, const u3dg_model *grads, const u3dg_learning_rates *lr)
{
    return guarded([&] {
        u3dg_adam &A = adamOf(adam);
        requireModel(params, "params");
        requireModel(grads, "grads");
        if (!lr || params->count != A.count || grads->count != A.count)
            throw StatusError(U3DG_ERR_INVALID_ARG, "params / grads must have the optimizer's size");
        const size_t c = std::max<size_t>(A.count, 1), n = A.count;
        cudaStream_t s = A.stream.s;
        A.p.reserve(14 * c);
        A.g.reserve(14 * c);
        uploadGroups(A.p.p, c, *params, s);
        uploadGroups(A.g.p, c, *grads, s);
        ++A.step;
        const float bc1 = 1.0f - std::pow(0.9f, float(A.step));
        const float bc2 = 1.0f - std::pow(0.999f, float(A.step));
        const float inv = 1.0f / std::sqrt(bc2);
        const float lrs[5] = {lr->means, lr->scales, lr->quats, lr->opacities, lr->colors};
        const size_t off[5] = {0, 3 * c, 6 * c, 10 * c, 11 * c};
        const size_t len[5] = {3 * n, 3 * n, 4 * n, n, 3 * n};
        for (int k = 0; k < 5; ++k)
            launchAdamSegment(A.p.p + off[k], A.g.p + off[k], A.m.p + off[k], A.v.p + off[k], int(len[k]), lrs[k] / bc1,
                              inv, s);
        U3DG_CUDA(cudaGetLastError());
        downloadGroups(A.p.p, c, n, *params, s);
        A.stream.sync();
    });
}

int u3dg_adam_compact(u3dg_adam *adam, const uint8_t *keep, size_t count)
{
    return guarded([&] {
        u3dg_adam &A = adamOf(adam);
        if (count != A.count || (count && !keep))
            throw StatusError(U3DG_ERR_INVALID_ARG, "keep must have the optimizer's size");
        const size_t c = std::max<size_t>(A.count, 1);
        std::vector<float> hm(14 * c), hv(14 * c);
        U3DG_CUDA(cudaMemcpyAsync(hm.data(), A.m.p, 14 * c * 4, cudaMemcpyDeviceToHost, A.stream.s));
        U3DG_CUDA(cudaMemcpyAsync(hv.data(), A.v.p, 14 * c * 4, cudaMemcpyDeviceToHost, A.stream.s));
        A.stream.sync();
        size_t kept = 0;
        for (size_t i = 0; i < count; ++i)
            kept += keep[i] ? 1 : 0;
        const size_t c2 = std::max<size_t>(kept, 1);
        std::vector<float> nm(14 * c2, 0.0f), nv(14 * c2, 0.0f);
        const int dims[5] = {3, 3, 4, 1, 3};
        const size_t off[5] = {0, 3, 6, 10, 11};
        for (int gidx = 0; gidx < 5; ++gidx) {
            size_t o = 0;
            for (size_t i = 0; i < count; ++i) {
                if (!keep[i])
                    continue;
                for (int d = 0; d < dims[gidx]; ++d) {
                    nm[off[gidx] * c2 + o * dims[gidx] + d] = hm[off[gidx] * c + i * dims[gidx] + d];
                    nv[off[gidx] * c2 + o * dims[gidx] + d] = hv[off[gidx] * c + i * dims[gidx] + d];
                }
                ++o;
            }
        }
        A.m.reserve(14 * c2, true);
        A.v.reserve(14 * c2, true);
        U3DG_CUDA(cudaMemcpyAsync(A.m.p, nm.data(), 14 * c2 * 4, cudaMemcpyHostToDevice, A.stream.s));
        U3DG_CUDA(cudaMemcpyAsync(A.v.p, nv.data(), 14 * c2 * 4, cudaMemcpyHostToDevice, A.stream.s));
        A.stream.sync();
        A.count = kept;
    });
}

int u3dg_adam_grow(u3dg_adam *adam, size_t count)
{
    return guarded([&] {
        u3dg_adam &A = adamOf(adam);
        const size_t c = std::max<size_t>(A.count, 1), n2 = A.count + count, c2 = std::max<size_t>(n2, 1);
        std::vector<float> hm(14 * c), hv(14 * c), nm(14 * c2, 0.0f), nv(14 * c2, 0.0f);
        U3DG_CUDA(cudaMemcpyAsync(hm.data(), A.m.p, 14 * c * 4, cudaMemcpyDeviceToHost, A.stream.s));
        U3DG_CUDA(cudaMemcpyAsync(hv.data(), A.v.p, 14 * c * 4, cudaMemcpyDeviceToHost, A.stream.s));
        A.stream.sync();
        const int dims[5] = {3, 3, 4, 1, 3};
        const size_t off[5] = {0, 3, 6, 10, 11};
        for (int gidx = 0; gidx < 5; ++gidx)
            for (size_t k = 0; k < A.count * dims[gidx]; ++k) {
                nm[off[gidx] * c2 + k] = hm[off[gidx] * c + k];
                nv[off[gidx] * c2 + k] = hv[off[gidx] * c + k];
            }
        A.m.reserve(14 * c2, true);
        A.v.reserve(14 * c2, true);
        U3DG_CUDA(cudaMemcpyAsync(A.m.p, nm.data(), 14 * c2 * 4, cudaMemcpyHostToDevice, A.stream.s));
        U3DG_CUDA(cudaMemcpyAsync(A.v.p, nv.data(), 14 * c2 * 4, cudaMemcpyHostToDevice, A.stream.s));
        A.stream.sync();
        A.count = n2;
    });
}

int u3dg_adam_reset_opacity_moments(u3dg_adam *adam)
{
    return guarded([&] {
        u3dg_adam &A = adamOf(adam);
        const size_t c = std::max<size_t>(A.count, 1);
        if (A.count) {
            U3DG_CUDA(cudaMemsetAsync(A.m.p + 10 * c, 0, A.count * 4, A.stream.s));
            U3DG_CUDA(cudaMemsetAsync(A.v.p + 10 * c, 0, A.count * 4, A.stream.s));
        }
        A.stream.sync();
    });
}

int u3dg_adam_moments(u3dg_adam *adam, u3dg_model *m, u3dg_model *v)
{
    return guarded([&] {
        u3dg_adam &A = adamOf(adam);
        const size_t c = std::max<size_t>(A.count, 1);
        if (m) {
            requireModel(m, "m");
            downloadGroups(A.m.p, c, A.count, *m, A.stream.s);
        }
        if (v) {
            requireModel(v, "v");
            downloadGroups(A.v.p, c, A.count, *v, A.stream.s);
        }
        A.stream.sync();
    });
}

void u3dg_adam_destroy(u3dg_adam *adam)
{
    if (!adam)
        return;
    cudaSetDevice(adam->device);
    delete adam;
}

// ------------------------------------------------------------------ densification

int u3dg_densify_and_prune(u3dg_model *model, u3dg_model *adam_m, u3dg_model *adam_v, const float *grad_accum,
                           const int *grad_count, size_t capacity, float scene_extent,
                           const u3dg_train_options *options, int opacity_was_reset, unsigned int seed, size_t *count,
                           int *counts3)
{
    return guarded([&] {
        requireModel(model, "model");
        requireModel(adam_m, "adam_m");
        requireModel(adam_v, "adam_v");
        if (!options || !count || (model->count && (!grad_accum || !grad_count)))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (adam_m->count != model->count || adam_v->count != model->count)
            throw StatusError(U3DG_ERR_INVALID_ARG, "moments must have the model's size");
        requireDevice();
        u3dg_train_options o = *options;
        TrainerImpl t(*model, nullptr, 0, scene_extent, o);
        const size_t n = model->count;
        copyModelToArena(t.arena[t.cur].p + 14 * t.cap, t.cap, *adam_m, t.stream);
        copyModelToArena(t.arena[t.cur].p + 28 * t.cap, t.cap, *adam_v, t.stream);
        if (n) {
            U3DG_CUDA(cudaMemcpyAsync(t.gradAccum.p, grad_accum, n * 4, cudaMemcpyHostToDevice, t.stream));
            U3DG_CUDA(cudaMemcpyAsync(t.gradCount.p, grad_count, n * 4, cudaMemcpyHostToDevice, t.stream));
        }
        t.opacityWasReset = opacity_was_reset != 0;
        std::mt19937 rng(seed);
        const DensifyResult r = densifyOnDevice(t, rng);
        *count = size_t(r.newCount);
        if (counts3) {
            counts3[0] = r.pruned;
            counts3[1] = r.clones;
            counts3[2] = r.splits;
        }
        if (size_t(r.newCount) > capacity)
            throw StatusError(U3DG_ERR_CAPACITY, "densified model does not fit the given capacity");
        u3dg_model om = *model, mm = *adam_m, vm = *adam_v;
        om.count = mm.count = vm.count = size_t(r.newCount);
        downloadGroups(t.arena[t.cur].p, t.cap, om.count, om, t.stream);
        downloadGroups(t.arena[t.cur].p + 14 * t.cap, t.cap, mm.count, mm, t.stream);
        downloadGroups(t.arena[t.cur].p + 28 * t.cap, t.cap, vm.count, vm, t.stream);
        t.sync();
    });
}

// ------------------------------------------------------------------ host I/O and init

int u3dg_init_gaussians_from_points(const float *xyz, const float *rgb, size_t n, u3dg_model *out)
{
    return guarded([&] {
        if (n && (!xyz || !out))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (n)
            requireModel(out, "out");
        requireDevice();
        initGaussiansFromPointsDevice(xyz, rgb, n, *out);
    });
}

// ------------------------------------------------------------------ crop

static void requireBox(const u3dg_crop_box *box)
{
    if (!box)
        throw StatusError(U3DG_ERR_INVALID_ARG, "crop box is NULL");
}

int u3dg_crop_model(const u3dg_model *model, const u3dg_crop_box *box, float min_opacity, u3dg_model *out,
                    size_t capacity, size_t *count)
{
    return guarded([&] {
        requireModel(model, "model");
        requireBox(box);
        if (!count)
            throw StatusError(U3DG_ERR_INVALID_ARG, "count is NULL");
        requireDevice();
        Stream st;
        DevModel in;
        in.upload(*model, st.s);
        const int n = int(model->count);
        DevBuf<int> keep, pos, scratch;
        const size_t kept = cropKeep(in.params(), n, *box, min_opacity, keep, pos, scratch, st.s);
        *count = kept;
        if (!out)
            return;
        if (kept > capacity)
            throw StatusError(U3DG_ERR_CAPACITY, "output capacity too small");
        requireModel(out, "out");
        DevModel res;
        res.cap = std::max<size_t>(kept, 1);
        res.buf.reserve(14 * res.cap, true);
        launchCropWrite(in.buf.p, in.cap, res.buf.p, res.cap, 1, n, keep.p, pos.p, st.s);
        U3DG_CUDA(cudaGetLastError());
        res.download(*out, kept, st.s);
        st.sync();
    });
}

int u3dg_suggest_crop_box(const u3dg_model *model, float low_fraction, float high_fraction, float margin,
                          u3dg_crop_box *out)
{
    return guarded([&] {
        requireModel(model, "model");
        requireBox(out);
        requireDevice();
        Stream st;
        DevModel in;
        in.upload(*model, st.s);
        // suggestCropBox weighs towards opaque Gaussians: opacity floor 0.3 (Crop.cpp:54-57).
        *out = quantileBoxOnDevice(in.params(), int(model->count), low_fraction, high_fraction, margin, 0.3f, st.s);
    });
}

int u3dg_model_bounds(const u3dg_model *model, u3dg_crop_box *out)
{
    return guarded([&] {
        requireModel(model, "model");
        requireBox(out);
        requireDevice();
        Stream st;
        DevModel in;
        in.upload(*model, st.s);
        *out = quantileBoxOnDevice(in.params(), int(model->count), 0.005f, 0.995f, 0.1f, 0.0f, st.s); // Crop.cpp:59-62
    });
}

int u3dg_trainer_crop(u3dg_trainer *trainer, const u3dg_crop_box *box, float min_opacity)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        requireBox(box);
        t.crop(*box, min_opacity);
    });
}

int u3dg_trainer_suggest_crop_box(u3dg_trainer *trainer, float low_fraction, float high_fraction, float margin,
                                  u3dg_crop_box *out)
{
    return guarded([&] {
        TrainerImpl &t = impl(trainer);
        requireBox(out);
        t.finish();
        *out = low_fraction < 0.0f
                   ? quantileBoxOnDevice(t.params(), t.n, 0.005f, 0.995f, 0.1f, 0.0f, t.stream)
                   : quantileBoxOnDevice(t.params(), t.n, low_fraction, high_fraction, margin, 0.3f, t.stream);
    });
}

int u3dg_write_splat_ply(const char *path, const u3dg_model *model)
{
    return guarded([&] {
        if (!path)
            throw StatusError(U3DG_ERR_INVALID_ARG, "path is NULL");
        requireModel(model, "model");
        std::string err;
        if (!writeSplatPlyHost(path, *model, &err))
            throw StatusError(U3DG_ERR_IO, err);
    });
}

int u3dg_write_splat_ply_sh(const char *path, const u3dg_model *model, const float *sh_rest, int degree)
{
    return guarded([&] {
        if (!path)
            throw StatusError(U3DG_ERR_INVALID_ARG, "path is NULL");
        requireModel(model, "model");
        if (!sh_rest && model->count > 0)
            throw StatusError(U3DG_ERR_INVALID_ARG, "sh_rest is NULL");
        if (degree < 1 || degree > 3)
            throw StatusError(U3DG_ERR_INVALID_ARG, "SH degree must be 1..3");
        static const float kNone = 0.0f;
        std::string err;
        if (!writeSplatPlyHost(path, *model, &err, sh_rest ? sh_rest : &kNone, degree))
            throw StatusError(U3DG_ERR_IO, err);
    });
}

int u3dg_read_splat_ply(const char *path, u3dg_model *out, size_t capacity, size_t *count, int *is_splat)
{
    return guarded([&] {
        if (!path || !count)
            throw StatusError(U3DG_ERR_INVALID_ARG, "path and count must not be NULL");
        std::string err;
        HostModel m;
        bool splat = false;
        if (!readSplatPlyHost(path, m, &err, &splat))
            throw StatusError(U3DG_ERR_IO, err);
        *count = m.size();
        if (is_splat)
            *is_splat = splat ? 1 : 0;
        if (!out)
            return;
        if (m.size() > capacity)
            throw StatusError(U3DG_ERR_CAPACITY, "output capacity too small");
        requireModel(out, "out");
        std::copy(m.means.begin(), m.means.end(), out->means);
        std::copy(m.scales.begin(), m.scales.end(), out->scales);
        std::copy(m.quats.begin(), m.quats.end(), out->quats);
        std::copy(m.opac.begin(), m.opac.end(), out->opacities);
        std::copy(m.colors.begin(), m.colors.end(), out->colors);
    });
}

int u3dg_render_sh(const u3dg_model *model, const float *sh_rest, int degree, const u3dg_camera *camera,
                   const u3dg_raster_settings *settings, float *rgb)
{
    return guarded([&] {
        requireDevice();
        u3dg_rasterizer r;
        U3DG_CUDA(cudaGetDevice(&r.device));
        rasterForward(r, model, sh_rest, degree, camera, settings, rgb);
    });
}

int u3dg_render_views_sh(const u3dg_model *model, const float *sh_rest, int degree, const u3dg_camera *cameras,
                         int count, const u3dg_raster_settings *settings, uint8_t *rgb8)
{
    return guarded([&] {
        requireDevice();
        requireModel(model, "model");
        if (count < 0 || (count > 0 && (!cameras || !rgb8)) || !settings)
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (degree < 0 || degree > 3)
            throw StatusError(U3DG_ERR_INVALID_ARG, "SH degree must be 0..3");
        checkSettings(*settings);
        u3dg_rasterizer r;
        U3DG_CUDA(cudaGetDevice(&r.device));
        cudaStream_t s = r.stream.s;
        r.model.upload(*model, s);
        DevBuf<float> sh;
        const float *shDev = nullptr;
        if (sh_rest && degree > 0 && model->count > 0) {
            const size_t K = size_t((degree + 1) * (degree + 1) - 1);
            sh.reserve(model->count * K * 3, true);
            U3DG_CUDA(cudaMemcpyAsync(sh.p, sh_rest, model->count * K * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
            shDev = sh.p;
        }
        DevBuf<uint8_t> q;
        size_t offset = 0;
        for (int v = 0; v < count; ++v) {
            checkCamera(cameras[v]);
            const size_t P3 = size_t(cameras[v].width) * cameras[v].height * 3;
            r.ws.forwardChecked(r.model.params(), int(model->count), cameras[v], *settings, shDev, degree, s);
            q.reserve(P3);
            launchQuantize(r.ws.rgb.p, P3, q.p, s);
            U3DG_CUDA(cudaGetLastError());
            U3DG_CUDA(cudaMemcpyAsync(rgb8 + offset, q.p, P3, cudaMemcpyDeviceToHost, s));
            r.stream.sync();
            offset += P3;
        }
    });
}

} // extern "C"
