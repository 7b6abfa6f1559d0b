// batch.cu - many scenes trained at once on one GPU (C ABI: u3dg_batch_*). No reference counterpart:
// the reference trains one scene per Trainer (engine/src/splat/Trainer.cpp). Every scene keeps its own
// TrainerImpl (model, Adam state, RNG, stream); stepBatch interleaves them so the kernels of small
// scenes run concurrently, and runs without densification go through each trainer's step graph. An
// optional autotuner picks each scene's tile size (8, 16 or 32) from short timed runs.

#include "engine.h"

#include <chrono>

using namespace u3dg;

struct u3dg_batch {
    int device = 0;
    std::vector<std::unique_ptr<u3dg_trainer>> scenes;
    std::vector<RasterSchedule> schedules; // tile size, batch depths, tuned ms per step (0: not tuned)
    BatchGraph graph; // rounds of all scenes as one graph launch
    std::vector<TrainerImpl *> impls() const
    {
        std::vector<TrainerImpl *> v;
        for (const auto &s : scenes)
            v.push_back(s->impl.get());
        return v;
    }
};

namespace {

u3dg_batch &batchOf(u3dg_batch *b)
{
    if (!b)
        throw StatusError(U3DG_ERR_INVALID_ARG, "batch is NULL");
    U3DG_CUDA(cudaSetDevice(b->device));
    return *b;
}

void requireScene(const u3dg_batch &b, int scene)
{
    if (scene < 0 || scene >= int(b.scenes.size()))
        throw StatusError(U3DG_ERR_INVALID_ARG, "scene index out of range");
}

} // namespace

extern "C" {

int u3dg_batch_create(const u3dg_model *initial, const u3dg_image *const *images, const int *image_counts,
                      const float *extents, const u3dg_train_options *options, int scenes, int autotune,
                      u3dg_batch **out)
{
    return guardedCall([&] {
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        *out = nullptr;
        if (scenes <= 0 || !initial || !images || !image_counts || !extents || !options)
            throw StatusError(U3DG_ERR_INVALID_ARG, "invalid batch arguments");
        int devices = 0;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
            cudaGetLastError();
            throw StatusError(U3DG_ERR_NO_DEVICE, "no CUDA device is available");
        }
        auto b = std::make_unique<u3dg_batch>();
        U3DG_CUDA(cudaGetDevice(&b->device));
        for (int s = 0; s < scenes; ++s) {
            if (initial[s].count > 0 && (!initial[s].means || !initial[s].scales || !initial[s].quats ||
                                         !initial[s].opacities || !initial[s].colors))
                throw StatusError(U3DG_ERR_INVALID_ARG, "scene " + std::to_string(s) + ": model has NULL arrays");
            u3dg_train_options o = options[s];
            RasterSchedule rs{o.raster.tile_size, 8, 1, 1, 0.0f};
            if (autotune)
                rs = autotuneSchedule(initial[s], images[s], image_counts[s], extents[s], options[s]);
            o.raster.tile_size = rs.tileSize;
            auto t = std::make_unique<u3dg_trainer>();
            t->impl = std::make_unique<TrainerImpl>(initial[s], images[s], image_counts[s], extents[s], o);
            t->impl->ws.forwardBlock = rs.forwardBlock;
            t->impl->ws.forwardDepth = rs.forwardDepth;
            t->impl->ws.backwardDepth = rs.backwardDepth;
            t->ownedByBatch = true;
            b->schedules.push_back(rs);
            b->scenes.push_back(std::move(t));
        }
        *out = b.release();
    });
}

int u3dg_batch_step(u3dg_batch *batch, int count)
{
    return guardedCall([&] {
        u3dg_batch &b = batchOf(batch);
        if (count > 0)
            stepBatch(b.impls(), count, &b.graph);
    });
}

int u3dg_batch_time_steps(u3dg_batch *batch, int count, float *ms)
{
    return guardedCall([&] {
        u3dg_batch &b = batchOf(batch);
        if (!ms)
            throw StatusError(U3DG_ERR_INVALID_ARG, "ms is NULL");
        std::vector<TrainerImpl *> ts = b.impls();
        for (TrainerImpl *t : ts)
            t->finish();
        // One start event that every scene stream waits on, one end event per stream that the first
        // stream waits on: the elapsed time spans all streams' work on the device.
        cudaStream_t s0 = ts[0]->stream;
        cudaEvent_t start, stop;
        U3DG_CUDA(cudaEventCreate(&start));
        U3DG_CUDA(cudaEventCreate(&stop));
        std::vector<cudaEvent_t> ends(ts.size());
        for (auto &e : ends)
            U3DG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        U3DG_CUDA(cudaEventRecord(start, s0));
        for (TrainerImpl *t : ts)
            U3DG_CUDA(cudaStreamWaitEvent(t->stream, start, 0));
        if (count > 0)
            stepBatch(ts, count, &b.graph);
        for (size_t i = 0; i < ts.size(); ++i) {
            U3DG_CUDA(cudaEventRecord(ends[i], ts[i]->stream));
            U3DG_CUDA(cudaStreamWaitEvent(s0, ends[i], 0));
        }
        U3DG_CUDA(cudaEventRecord(stop, s0));
        U3DG_CUDA(cudaEventSynchronize(stop));
        U3DG_CUDA(cudaEventElapsedTime(ms, start, stop));
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        for (auto &e : ends)
            cudaEventDestroy(e);
    });
}

int u3dg_batch_size(u3dg_batch *batch, int *scenes)
{
    return guardedCall([&] {
        u3dg_batch &b = batchOf(batch);
        if (!scenes)
            throw StatusError(U3DG_ERR_INVALID_ARG, "scenes is NULL");
        *scenes = int(b.scenes.size());
    });
}

int u3dg_batch_trainer(u3dg_batch *batch, int scene, u3dg_trainer **out)
{
    return guardedCall([&] {
        u3dg_batch &b = batchOf(batch);
        requireScene(b, scene);
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        *out = b.scenes[size_t(scene)].get();
    });
}

int u3dg_batch_tile_size(u3dg_batch *batch, int scene, int *tile, float *tuned_ms_per_step)
{
    return u3dg_batch_schedule(batch, scene, tile, nullptr, nullptr, nullptr, tuned_ms_per_step);
}

int u3dg_batch_schedule(u3dg_batch *batch, int scene, int *tile, int *forward_block, int *forward_depth,
                        int *backward_depth, float *tuned_ms_per_step)
{
    return guardedCall([&] {
        u3dg_batch &b = batchOf(batch);
        requireScene(b, scene);
        const RasterSchedule &rs = b.schedules[size_t(scene)];
        if (tile)
            *tile = rs.tileSize;
        if (forward_block)
            *forward_block = rs.forwardBlock;
        if (forward_depth)
            *forward_depth = rs.forwardDepth;
        if (backward_depth)
            *backward_depth = rs.backwardDepth;
        if (tuned_ms_per_step)
            *tuned_ms_per_step = rs.msPerStep;
    });
}

int u3dg_batch_graph_launches(u3dg_batch *batch, long long *launches, long long *captures)
{
    return guardedCall([&] {
        u3dg_batch &b = batchOf(batch);
        if (launches)
            *launches = b.graph.launches;
        if (captures)
            *captures = b.graph.captures;
    });
}

void u3dg_batch_destroy(u3dg_batch *batch)
{
    if (!batch)
        return;
    cudaSetDevice(batch->device);
    delete batch;
}

} // extern "C"
