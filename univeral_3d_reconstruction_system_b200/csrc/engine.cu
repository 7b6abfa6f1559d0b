// engine.cu - host orchestration of the GPU trainer: raster workspace, Trainer, densification.
//
// One CUDA stream per trainer. A step queues: projection, depth sort, per-rank tile counts + scan,
// capacity check, emission, tile sort, tile offsets, compositing forward, loss forward/backward +
// stats, compositing backward, and the chain rule fused with Adam - with no host wait inside. The
// host reads each step's bin counts back asynchronously and checks them kLag steps later; a step whose
// intersections overflowed the buffers did no update (the device skips it and every later step), so
// the host restores its own state to that step, grows the buffers and replays. Densification steps
// wait for the GPU anyway (the split count decides how many samples the host RNG draws).
// The training RNG (std::mt19937, Trainer.h:79) stays on the host so the view order and the split
// samples are the reference's exactly.
//
// Runs of 10 steps with no densification or opacity reset among them go through a CUDA graph whose
// kernels read each step's camera, target and learning rates from device descriptors (StepDesc); the
// graph is recorded once and updated in place when the model size or buffers change. A trainer keeps
// one run in flight while the host checks the previous one and prepares the next (stepTo). stepBatch
// runs several trainers this way, as one graph launch per round when all of them can. Every buffer a
// schedule needs is allocated when the trainer is created, so a schedule never waits on an allocation.

#include "engine.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>

namespace u3dg {

static std::atomic<unsigned long long> gLaunches{0};

void countLaunch() { gLaunches.fetch_add(1, std::memory_order_relaxed); }

unsigned long long launchCount() { return gLaunches.load(std::memory_order_relaxed); }

void addLaunches(long long k) { gLaunches.fetch_add((unsigned long long)k, std::memory_order_relaxed); }

static std::atomic<unsigned long long> gAllocEpoch{0};

unsigned long long allocEpoch() { return gAllocEpoch.load(std::memory_order_relaxed); }

void bumpAllocEpoch() { gAllocEpoch.fetch_add(1, std::memory_order_relaxed); }

void DeviceSlab::commit()
{
    if (items.empty())
        return;
    auto slice = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t sum = 0;
    for (const Item &it : items)
        sum += slice(it.bytes);
    void *base = nullptr;
    const cudaError_t e = cudaMalloc(&base, sum);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw StatusError(U3DG_ERR_OOM, "cudaMalloc of " + std::to_string(sum) + " bytes failed: " + cudaGetErrorString(e));
    }
    bases.push_back(base);
    total += sum;
    size_t off = 0;
    for (const Item &it : items) {
        it.adopt(it.buf, static_cast<char *>(base) + off, it.count);
        off += slice(it.bytes);
    }
    items.clear();
}

static thread_local std::string tLastError;

int setError(int code, const std::string &msg)
{
    tLastError = msg;
    return code;
}

const char *lastError() { return tLastError.c_str(); }

void checkSettings(const u3dg_raster_settings &st)
{
    if (!(st.tile_size == 8 || (st.tile_size >= 16 && st.tile_size % 16 == 0 && st.tile_size <= 256)))
        throw StatusError(U3DG_ERR_INVALID_ARG,
                          "tile_size must be 8 or a multiple of 16 up to 256, got " + std::to_string(st.tile_size));
}

void checkCamera(const u3dg_camera &cam)
{
    if (cam.width <= 0 || cam.height <= 0 || cam.width > 16384 || cam.height > 16384)
        throw StatusError(U3DG_ERR_INVALID_ARG, "camera size must be 1..16384 pixels per side");
    if (!(cam.fx != 0.0f) || !(cam.fy != 0.0f))
        throw StatusError(U3DG_ERR_INVALID_ARG, "camera focal lengths must be non-zero");
}

// ------------------------------------------------------------------ raster workspace

RasterWorkspace::RasterWorkspace()
{
    counts.reserve(1, true);
    hostCounts.reserve(1);
    BinCounts c{};
    c.abortIter = -1;
    *hostCounts.p = c;
    U3DG_CUDA(cudaMemcpy(counts.p, &c, sizeof(c), cudaMemcpyHostToDevice));
    // The compositing kernels' block counters start at zero and are reset by each launch's last CTA.
    blockCounters.reserve(4, true);
    U3DG_CUDA(cudaMemset(blockCounters.p, 0, 4 * sizeof(int)));
}

void RasterWorkspace::clearCounts(cudaStream_t stream)
{
    BinCounts c{};
    c.abortIter = -1;
    // A kernel-free, stream-ordered reset: copy from a pinned value that is never modified afterwards.
    static thread_local HostPinned<BinCounts> zero;
    if (!zero.p) {
        zero.reserve(1);
        *zero.p = c;
    }
    U3DG_CUDA(cudaMemcpyAsync(counts.p, zero.p, sizeof(BinCounts), cudaMemcpyHostToDevice, stream));
}

size_t RasterWorkspace::checkedIntersections(size_t capacity)
{
    capacity = std::max<size_t>(capacity, 1024);
    if (capacity > size_t(INT_MAX / 16))
        throw StatusError(U3DG_ERR_CAPACITY, "tile-Gaussian intersections exceed the supported 1.3e8");
    return capacity;
}

template <class F>
void RasterWorkspace::eachIntersectionBuffer(size_t capacity, F &&f)
{
    f(iKeys0, capacity);
    f(iKeys1, capacity);
    f(iVals0, capacity);
    f(iVals1, capacity);
    f(emitGid, capacity);
    f(entries, capacity);
    f(partial, capacity * kG2d * size_t(partialSlots));
}

void RasterWorkspace::reserveIntersections(size_t capacity)
{
    capacity = checkedIntersections(capacity);
    if (int(capacity) <= icap && iKeys0.p)
        return;
    eachIntersectionBuffer(capacity, [](auto &b, size_t c) { b.reserve(c, true); });
    icap = int(capacity);
}

void RasterWorkspace::planIntersections(DeviceSlab &slab, size_t capacity)
{
    capacity = checkedIntersections(capacity);
    eachIntersectionBuffer(capacity, [&](auto &b, size_t c) { slab.add(b, c); });
    icap = std::max(icap, int(capacity));
}

void RasterWorkspace::project(const Params &P, int count, const u3dg_camera &c, const u3dg_raster_settings &s,
                              const float *shRest, int shDegree, cudaStream_t stream, const StepDesc *desc)
{
    checkSettings(s);
    checkCamera(c);
    cam = c;
    st = s;
    n = count;
    tilesX = (cam.width + st.tile_size - 1) / st.tile_size;
    tilesY = (cam.height + st.tile_size - 1) / st.tile_size;
    const size_t nn = size_t(std::max(n, 1));
    reserveGaussians(nn);
    if (icap == 0)
        reserveIntersections(std::max<size_t>(size_t(1) << 20, 16 * nn));
    const int per = st.tile_size > 16 ? st.tile_size / 16 : 1;
    if (per * per > partialSlots) { // a tile size spanning more backward CTAs than before
        partialSlots = per * per;
        partial.reserve(size_t(icap) * kG2d * size_t(partialSlots), true);
    }
    ProjOut out{rec.p, depthKey.p, depth.p, rect.p, radius.p, flags.p, cov2d.p, cnt.p, rowTab.p, culled() ? 1 : 0};
    launchProject(P, n, cam, st, tilesX, tilesY, shRest, shDegree, out, stream, desc);
}

template <class F>
void RasterWorkspace::eachGaussianBuffer(size_t nn, F &&f)
{
    f(rec, nn);
    f(depthKey, nn);
    f(depthPairs[0], nn);
    f(depthPairs[1], nn);
    f(depthOrder, nn);
    f(depth, nn);
    f(rect, nn);
    f(radius, nn);
    f(rowTab, cullRowEntries(nn));
    f(cnt, nn);
    f(offs, nn + 1);
    f(scanPartial, scanPartialEntries(int(nn)) + 1);
    f(flags, nn);
    f(cov2d, nn);
    f(g2d, nn * kG2d);
    f(hist, std::max(radixHistEntries(std::max(int(nn), icap)), size_t(256)));
}

void RasterWorkspace::reserveGaussians(size_t nn)
{
    eachGaussianBuffer(std::max<size_t>(nn, 1), [](auto &b, size_t c) { b.reserve(c); });
}

void RasterWorkspace::planGaussians(DeviceSlab &slab, size_t nn)
{
    eachGaussianBuffer(std::max<size_t>(nn, 1), [&](auto &b, size_t c) { slab.add(b, c); });
}

void RasterWorkspace::planPixels(DeviceSlab &slab, size_t pixels, int tx, int ty, int tileSize)
{
    // The sizes bin() and composite() reserve for such a view.
    slab.add(rgb, pixels * 3);
    slab.add(finalT, pixels);
    slab.add(nContrib, pixels);
    slab.add(tileOffsets, size_t(tx) * ty + 1);
    slab.add(rowTotals, size_t(radixDigits()));
    const int pb = tileSize <= 8 ? 8 : 16;
    const int per = tileSize > pb ? tileSize / pb : 1;
    slab.add(blockOrder, size_t(std::max(1, tx * per * ty * per)));
}

void RasterWorkspace::bin(cudaStream_t stream, int iteration, const StepDesc *desc)
{
    const int tiles = tilesX * tilesY;
    hist.reserve(std::max(radixHistEntries(std::max(n, icap)), size_t(256)));
    rowTotals.reserve(size_t(radixDigits()));
    tileOffsets.reserve(size_t(tiles) + 1);
    uint32_t *keysOut = nullptr, *valsOut = nullptr;
    radixSortDepth(depthKey.p, depthPairs[0].p, depthPairs[1].p, depthOrder.p, n, hist.p, rowTotals.p, stream);
    sortedIds = depthOrder.p;
    // The projection counted each Gaussian's tiles (and, culling, its row table); the scan takes the
    // counts in depth-rank order.
    const SplatRec *cullRec = culled() ? rec.p : nullptr;
    exclusiveScanChecked(cnt.p, sortedIds, offs.p, n, scanPartial.p, ScanCapacity{icap, counts.p, iteration, desc},
                         stream);
    launchEmit(sortedIds, offs.p, rect.p, n, counts.p, icap, tilesX, cullRec, st.tile_size, rowTab.p, iKeys0.p,
               emitGid.p, stream);
    int bits = 0;
    while ((1 << bits) < tiles)
        ++bits;
    bits = std::max(bits, 1);
    // Up to 2048 tiles: one pass whose scatter also writes the lists' entries and the tile offsets.
    const TileFinish fin{emitGid.p, entries.p, tileOffsets.p, tiles};
    const int tilePasses = radixSortPairs(iKeys0.p, iKeys1.p, iVals0.p, iVals1.p, &counts.p->effTotal, icap, bits,
                                          hist.p, rowTotals.p, &keysOut, &valsOut, stream, &fin);
    if (tilePasses != 1)
        launchFinalizeBins(keysOut, valsOut, emitGid.p, counts.p, icap, tiles, entries.p, tileOffsets.p, stream);
}

void RasterWorkspace::forwardChecked(const Params &P, int count, const u3dg_camera &c, const u3dg_raster_settings &s,
                                     const float *shRest, int shDegree, cudaStream_t stream)
{
    for (int attempt = 0; attempt < 8; ++attempt) {
        clearCounts(stream);
        forward(P, count, c, s, shRest, shDegree, stream, 0);
        U3DG_CUDA(cudaMemcpyAsync(hostCounts.p, counts.p, sizeof(BinCounts), cudaMemcpyDeviceToHost, stream));
        U3DG_CUDA(cudaStreamSynchronize(stream));
        if (hostCounts.p->abortIter < 0)
            return;
        reserveIntersections(size_t(hostCounts.p->need) + size_t(hostCounts.p->need) / 4);
    }
    throw StatusError(U3DG_ERR_CAPACITY, "intersection buffers could not be sized");
}

RasterArgs RasterWorkspace::rasterArgs() const
{
    RasterArgs a;
    a.tileOffsets = tileOffsets.p;
    a.entries = entries.p;
    a.rec = rec.p;
    a.width = cam.width;
    a.height = cam.height;
    a.tileSize = st.tile_size;
    a.tilesX = tilesX;
    for (int k = 0; k < 3; ++k)
        a.bg[k] = st.background[k];
    a.minAlpha = st.min_alpha;
    a.minTransmittance = st.min_transmittance;
    const int pb = st.tile_size <= 8 ? 8 : 16;
    // Whole tiles of pixel blocks: a block past the image edge composites nothing, but (for tiles of
    // several blocks) still writes its slot of every entry of its tile.
    const int per = st.tile_size > pb ? st.tile_size / pb : 1;
    a.blocksX = tilesX * per;
    a.blocksY = tilesY * per;
    a.subSlots = per * per;
    a.subStride = size_t(icap) * kG2d;
    a.blockOrder = blockOrder.p;
    a.counters = blockCounters.p;
    a.forwardBlock = forwardBlock;
    a.forwardDepth = forwardDepth;
    a.backwardDepth = backwardDepth;
    return a;
}

void RasterWorkspace::composite(cudaStream_t stream)
{
    const size_t P = size_t(cam.width) * cam.height;
    rgb.reserve(P * 3);
    finalT.reserve(P);
    nContrib.reserve(P);
    const int pb = st.tile_size <= 8 ? 8 : 16;
    const int per = st.tile_size > pb ? st.tile_size / pb : 1;
    blockOrder.reserve(size_t(std::max(1, tilesX * per * tilesY * per)));
    const RasterArgs a = rasterArgs();
    launchBlockOrder(a, blockOrder.p, stream);
    launchCompositeForward(a, rgb.p, finalT.p, nContrib.p, stream);
}

void RasterWorkspace::backwardComposite(const float *dLdRgb, cudaStream_t stream)
{
    launchCompositeBackward(rasterArgs(), dLdRgb, finalT.p, nContrib.p, partial.p, stream);
}

ChainArgs RasterWorkspace::chainArgs(const Params &P) const
{
    ChainArgs a{};
    a.params = P;
    a.n = n;
    a.cam = cam;
    a.st = st;
    a.radius = radius.p;
    a.rec = rec.p;
    a.flags = flags.p;
    a.offs = offs.p;
    a.sortedIds = sortedIds;
    a.partial = partial.p;
    const int per = st.tile_size > 16 ? st.tile_size / 16 : 1;
    a.subSlots = per * per;
    a.subStride = size_t(icap) * kG2d;
    a.g2d = g2d.p;
    a.counts = counts.p;
    return a;
}

// ------------------------------------------------------------------ trainer

void copyModelToArena(float *base, size_t cap, const u3dg_model &m, cudaStream_t s)
{
    const Params P = paramsAt(base, cap);
    const size_t n = m.count;
    if (n == 0)
        return;
    U3DG_CUDA(cudaMemcpyAsync(P.means, m.means, n * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.scales, m.scales, n * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.quats, m.quats, n * 4 * sizeof(float), cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.opac, m.opacities, n * sizeof(float), cudaMemcpyHostToDevice, s));
    U3DG_CUDA(cudaMemcpyAsync(P.colors, m.colors, n * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
}

static void copyArenaToModel(const float *base, size_t cap, size_t n, u3dg_model &m, cudaStream_t s)
{
    const Params P = paramsAt(const_cast<float *>(base), cap);
    if (n == 0)
        return;
    U3DG_CUDA(cudaMemcpyAsync(m.means, P.means, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.scales, P.scales, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.quats, P.quats, n * 4 * sizeof(float), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.opacities, P.opac, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(m.colors, P.colors, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
}

TrainerImpl::TrainerImpl(const u3dg_model &initial, const u3dg_image *imgs, int count, float sceneExtent,
                         const u3dg_train_options &opt, bool backgroundUpload)
    : o(opt), rng(opt.seed)
{
    checkSettings(o.raster);
    if (count < 0 || (count > 0 && imgs == nullptr))
        throw StatusError(U3DG_ERR_INVALID_ARG, "image list is invalid");
    if (initial.count > 0 && (!initial.means || !initial.scales || !initial.quats || !initial.opacities || !initial.colors))
        throw StatusError(U3DG_ERR_INVALID_ARG, "initial model has null arrays");
    if (initial.count > size_t(INT_MAX / 64))
        throw StatusError(U3DG_ERR_CAPACITY, "too many Gaussians");
    if (o.refine_interval <= 0)
        throw StatusError(U3DG_ERR_INVALID_ARG, "refine_interval must be positive");
    U3DG_CUDA(cudaGetDevice(&device));
    U3DG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    extent = std::max(sceneExtent, 1e-6f);
    ws.cullTiles = true;
    n = int(initial.count);
    cap = std::max<size_t>(size_t(std::max(o.max_gaussians, 0)), initial.count);
    cap = std::max<size_t>(cap, 1);
    size_t total = 0, maxP = 1;
    int maxTx = 1, maxTy = 1, maxLossBlocks = 1;
    const int ts = o.raster.tile_size;
    for (int k = 0; k < count; ++k) {
        checkCamera(imgs[k].camera);
        if (!imgs[k].rgb)
            throw StatusError(U3DG_ERR_INVALID_ARG, "image " + std::to_string(k) + " has no pixels");
        const u3dg_camera &c = imgs[k].camera;
        cams.push_back(c);
        imageOffset.push_back(total);
        const size_t P = size_t(c.width) * c.height;
        total += P * 3;
        maxP = std::max(maxP, P);
        maxTx = std::max(maxTx, (c.width + ts - 1) / ts);
        maxTy = std::max(maxTy, (c.height + ts - 1) / ts);
        maxLossBlocks = std::max(maxLossBlocks, lossBlocks(c.width, c.height));
    }
    // Everything a step, an evaluation or a densification needs, sized for the capacity and the
    // largest view, in one device allocation: nothing is allocated during a schedule (allocations wait
    // for the device), and creation pays for one cudaMalloc instead of one per buffer. Intersection
    // buffers start at 16 tiles per Gaussian at the capacity and grow on demand.
    for (auto &a : arena)
        slab.add(a, 42 * cap);
    slab.add(gradAccum, cap);
    slab.add(gradCount, cap);
    slab.add(images, std::max<size_t>(total, 1));
    slab.add(dLoss, maxP * 3);
    slab.add(abc, maxP * 9);
    slab.add(lossBlockSums, size_t(maxLossBlocks) * 3);
    slab.add(dStats, 1);
    slab.add(descDev, kGraphSteps);
    slab.add(statusDev, kGraphSteps);
    const int per = ts > 16 ? ts / 16 : 1;
    ws.partialSlots = std::max(ws.partialSlots, per * per);
    ws.planIntersections(slab, std::max<size_t>(size_t(1) << 20, 16 * cap));
    ws.planGaussians(slab, cap);
    ws.planPixels(slab, maxP, maxTx, maxTy, ts);
    for (DevBuf<int> *b : {&keep, &cost, &costScan, &accCost, &accScan, &isSplit, &splitScan, &keepScan})
        slab.add(*b, cap + 1);
    slab.add(firstSecond, 2);
    slab.add(dScanPartial, scanPartialEntries(int(cap)) + 1);
    slab.add(normals, 6 * cap);
    slab.commit();
    U3DG_CUDA(cudaMemsetAsync(arena[cur].p, 0, 42 * cap * sizeof(float), stream));
    copyModelToArena(arena[cur].p, cap, initial, stream);
    U3DG_CUDA(cudaMemsetAsync(gradAccum.p, 0, cap * sizeof(float), stream));
    U3DG_CUDA(cudaMemsetAsync(gradCount.p, 0, cap * sizeof(int), stream));
    if (!backgroundUpload || count == 0) {
        for (int k = 0; k < count; ++k) {
            const size_t P = size_t(imgs[k].camera.width) * imgs[k].camera.height;
            U3DG_CUDA(cudaMemcpyAsync(images.p + imageOffset[size_t(k)], imgs[k].rgb, P * 3, cudaMemcpyHostToDevice,
                                      stream));
        }
    }
    hStats.reserve(1);
    U3DG_CUDA(cudaMemsetAsync(dStats.p, 0, sizeof(DevStats), stream));
    std::memset(hStats.p, 0, sizeof(DevStats));
    statusSlots.reserve(kSlots);
    uniformViews = !cams.empty();
    for (const u3dg_camera &c : cams)
        uniformViews = uniformViews && c.width == cams[0].width && c.height == cams[0].height;
    descHost.reserve(2 * kGraphSteps);
    graphStatus.reserve(2 * kGraphSteps);
    for (cudaEvent_t &e : chunkDone)
        U3DG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    hCounts.reserve(4);
    hNormals.reserve(6 * cap);
    if (backgroundUpload && count > 0)
        startUploads(imgs, count);
    // The model's host buffers may be released after this call returns (and the images' too, unless
    // they are uploaded in the background).
    U3DG_CUDA(cudaStreamSynchronize(stream));
}

void TrainerImpl::startUploads(const u3dg_image *imgs, int count)
{
    auto up = std::make_unique<ImageUploader>();
    U3DG_CUDA(cudaStreamCreateWithFlags(&up->copy, cudaStreamNonBlocking));
    up->ready.assign(size_t(count), nullptr);
    for (cudaEvent_t &e : up->ready)
        U3DG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    up->waited.assign(size_t(count), 0);
    // The first epoch's view order, as nextStep will draw it from the same generator state.
    std::vector<int> first(static_cast<size_t>(count));
    for (int k = 0; k < count; ++k)
        first[size_t(k)] = k;
    std::mt19937 r = rng;
    std::shuffle(first.begin(), first.end(), r);
    up->position.assign(size_t(count), 0);
    for (int k = 0; k < count; ++k)
        up->position[size_t(first[size_t(k)])] = k;
    std::vector<const uint8_t *> src(static_cast<size_t>(count));
    for (int k = 0; k < count; ++k)
        src[size_t(k)] = imgs[k].rgb;
    ImageUploader *u = up.get();
    const int dev = device;
    uint8_t *dst = images.p;
    std::vector<size_t> offsets = imageOffset, bytes(static_cast<size_t>(count));
    for (int k = 0; k < count; ++k)
        bytes[size_t(k)] = size_t(imgs[k].camera.width) * imgs[k].camera.height * 3;
    up->thread = std::thread([u, dev, dst, first, src, offsets, bytes] {
        std::string err;
        if (cudaSetDevice(dev) != cudaSuccess)
            err = "cudaSetDevice failed in the image upload thread";
        for (size_t k = 0; k < first.size() && err.empty(); ++k) {
            const size_t v = size_t(first[k]);
            cudaError_t e = cudaMemcpyAsync(dst + offsets[v], src[v], bytes[v], cudaMemcpyHostToDevice, u->copy);
            if (e == cudaSuccess)
                e = cudaEventRecord(u->ready[v], u->copy);
            if (e != cudaSuccess) {
                err = std::string("image upload: ") + cudaGetErrorString(e);
                break;
            }
            std::lock_guard<std::mutex> lock(u->m);
            u->issued = int(k) + 1;
            u->cv.notify_all();
        }
        std::lock_guard<std::mutex> lock(u->m);
        if (!err.empty())
            u->error = err;
        u->cv.notify_all();
    });
    uploader = std::move(up);
}

void TrainerImpl::requireView(size_t v)
{
    ImageUploader *u = uploader.get();
    if (!u || u->waited[v])
        return;
    {
        std::unique_lock<std::mutex> lock(u->m);
        u->cv.wait(lock, [&] { return u->issued > u->position[v] || !u->error.empty(); });
        if (u->issued <= u->position[v])
            throw StatusError(U3DG_ERR_CUDA, u->error);
    }
    U3DG_CUDA(cudaStreamWaitEvent(stream, u->ready[v], 0));
    u->waited[v] = 1;
}

void TrainerImpl::waitUploads()
{
    ImageUploader *u = uploader.get();
    if (!u || u->joined)
        return;
    if (u->thread.joinable())
        u->thread.join();
    u->joined = true;
    U3DG_CUDA(cudaStreamSynchronize(u->copy));
    if (!u->error.empty())
        throw StatusError(U3DG_ERR_CUDA, u->error);
    // Every image is in place: later steps need not wait for anything.
    for (size_t v = 0; v < u->waited.size(); ++v)
        if (!u->waited[v]) {
            U3DG_CUDA(cudaStreamWaitEvent(stream, u->ready[v], 0));
            u->waited[v] = 1;
        }
}

TrainerImpl::~TrainerImpl()
{
    if (uploader) {
        // The copies read the caller's buffers and write `images`: finish them first.
        if (uploader->thread.joinable())
            uploader->thread.join();
        cudaStreamSynchronize(uploader->copy);
        for (cudaEvent_t e : uploader->ready)
            if (e)
                cudaEventDestroy(e);
        cudaStreamDestroy(uploader->copy);
    }
    if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
    for (InFlight &f : inflight)
        cudaEventDestroy(f.done);
    for (cudaEvent_t e : freeEvents)
        cudaEventDestroy(e);
    for (cudaEvent_t e : chunkDone)
        if (e)
            cudaEventDestroy(e);
    delete timer;
}

void TrainerImpl::sync() { U3DG_CUDA(cudaStreamSynchronize(stream)); }

HostSnapshot TrainerImpl::snapshot() const
{
    HostSnapshot s;
    s.iteration = iteration;
    s.orderPos = orderPos;
    s.order = order;
    s.rng = rng;
    s.adamStep = adamStep;
    s.opacityWasReset = opacityWasReset;
    return s;
}

void TrainerImpl::restore(const HostSnapshot &s)
{
    iteration = s.iteration;
    orderPos = s.orderPos;
    order = s.order;
    rng = s.rng;
    adamStep = s.adamStep;
    opacityWasReset = s.opacityWasReset;
}

bool TrainerImpl::checkOldest()
{
    InFlight f = inflight.front();
    inflight.erase(inflight.begin());
    U3DG_CUDA(cudaEventSynchronize(f.done));
    freeEvents.push_back(f.done);
    const BinCounts c = statusSlots.p[f.slot];
    if (c.abortIter < 0) {
        // Grow ahead of need: keep a quarter of headroom over the largest pass seen.
        if (size_t(c.total) + size_t(c.total) / 4 > size_t(ws.icap)) {
            sync();
            ws.reserveIntersections(size_t(c.total) + size_t(c.total) / 2);
        }
        return true;
    }
    // This step overflowed: it and every step queued after it did nothing on the device.
    sync();
    for (InFlight &g : inflight)
        freeEvents.push_back(g.done);
    inflight.clear();
    restore(f.snap);
    ws.reserveIntersections(size_t(c.need) + size_t(c.need) / 2);
    ws.clearCounts(stream);
    ++replays;
    return false;
}

void TrainerImpl::step()
{
    if (cams.empty() || done())
        return;
    while (int(inflight.size()) >= kLag)
        if (!checkOldest())
            return; // rolled back; the caller's loop replays from the restored iteration
    enqueueStep();
}

void TrainerImpl::stepTo(int target)
{
    target = std::min(target, o.iterations);
    // Graph runs are pipelined: the next run is launched (from the other slot) before the host waits
    // for the previous one, so the GPU is not idle while the host checks statuses and prepares
    // descriptors. A run that overflowed rolls the host state back to its failing step; the run
    // launched after it did nothing on the device (the abort is sticky) and is dropped.
    int pending = -1; // slot of the run launched but not yet checked
    while (iteration < target && !cams.empty()) {
        if (graphEligible(target)) {
            if (pending < 0) {
                // Record the run's graph first if it needs one: the capture executes nothing, so it
                // overlaps the single steps still running on the device instead of following them.
                primeGraph(target);
                finish(); // graph runs start with no single step in flight
                if (!graphEligible(target))
                    continue;
            }
            const int slot = pending < 0 ? 0 : 1 - pending;
            const bool launched = beginGraphChunk(slot);
            if (pending >= 0 && !endGraphChunk(pending, false)) {
                if (launched)
                    dropGraphChunk(slot);
                pending = -1;
                continue;
            }
            pending = launched ? slot : -1;
            continue;
        }
        if (pending >= 0) { // the steps after the graph runs start from their checked state
            endGraphChunk(pending, false);
            pending = -1;
            continue;
        }
        step();
    }
    if (pending >= 0) {
        const int last = pending;
        pending = -1;
        if (!endGraphChunk(last, false))
            stepTo(target); // replay the rolled-back steps
    }
}

void TrainerImpl::finish()
{
    const int target = iteration;
    for (;;) {
        bool ok = true;
        while (!inflight.empty())
            if (!checkOldest()) {
                ok = false;
                break;
            }
        if (ok)
            return;
        stepTo(target);
    }
}

StepValues TrainerImpl::nextStep()
{
    StepValues sv;
    // View order: one shuffle of all views per epoch (Trainer.cpp:57-64).
    if (orderPos >= order.size()) {
        order.resize(cams.size());
        for (size_t k = 0; k < order.size(); ++k)
            order[k] = int(k);
        std::shuffle(order.begin(), order.end(), rng);
        orderPos = 0;
    }
    sv.view = size_t(order[orderPos++]);
    requireView(sv.view);
    sv.d.cam = cams[sv.view];
    sv.d.target = images.p + imageOffset[sv.view];
    sv.d.iteration = iteration;
    // Means learning rate decays exponentially and scales with the scene (Trainer.cpp:81-85);
    // Adam bias corrections as Adam::step (Adam.cpp:68-71), all in host float like the reference.
    const float t = float(iteration) / float(std::max(1, o.iterations - 1));
    const float lrMeans = std::exp(std::log(o.lr.means) * (1 - t) + std::log(o.means_lr_final) * t) * extent;
    ++adamStep;
    const float bc1 = 1.0f - std::pow(0.9f, float(adamStep));
    const float bc2 = 1.0f - std::pow(0.999f, float(adamStep));
    const float lrs[5] = {lrMeans, o.lr.scales, o.lr.quats, o.lr.opacities, o.lr.colors};
    for (int k = 0; k < 5; ++k)
        sv.d.stepSize[k] = lrs[k] / bc1;
    sv.d.invSqrtBc2 = 1.0f / std::sqrt(bc2);
    return sv;
}

void TrainerImpl::launchStep(const StepValues &sv, const StepDesc *desc, BinCounts *statusDst)
{
    const u3dg_camera &cam = sv.d.cam;
    const int W = cam.width, H = cam.height;
    PhaseTimer *tm = (profiling && !desc) ? timer : nullptr;
    if (tm)
        tm->mark(0, stream);
    ws.project(params(), n, cam, o.raster, nullptr, 0, stream, desc);
    if (tm)
        tm->mark(1, stream);
    ws.bin(stream, sv.d.iteration, desc);
    if (tm)
        tm->mark(2, stream);
    ws.composite(stream);
    if (tm)
        tm->mark(3, stream);
    // Loss (Trainer.cpp:67-71) and the step's stats (Trainer.cpp:88-92).
    const int lb = lossBlocks(W, H);
    lossBlockSums.reserve(size_t(lb) * 3);
    LossScratch ls{abc.p, lossBlockSums.p, lb};
    launchLoss(ws.rgb.p, nullptr, sv.d.target, W, H, o.ssim_lambda, dLoss.p, ls, stream, desc);
    launchLossFinalize(ls, W, H, o.ssim_lambda, dStats.p, sv.d.iteration + 1, ws.counts.p, nullptr, nullptr, stream,
                       desc);
    if (tm)
        tm->mark(4, stream);
    ws.backwardComposite(dLoss.p, stream);
    if (tm)
        tm->mark(5, stream);
    ChainArgs a = ws.chainArgs(params());
    a.gradAccum = gradAccum.p;
    a.gradCount = gradCount.p;
    a.m = moment1();
    a.v = moment2();
    for (int k = 0; k < 5; ++k)
        a.stepSize[k] = sv.d.stepSize[k];
    a.invSqrtBc2 = sv.d.invSqrtBc2;
    a.desc = desc;
    launchChain(a, true, stream);
    U3DG_CUDA(cudaGetLastError());
    if (tm)
        tm->mark(6, stream);
    // statusDst: pinned host memory (single steps) or device memory (graph runs).
    U3DG_CUDA(cudaMemcpyAsync(statusDst, ws.counts.p, sizeof(BinCounts), cudaMemcpyDefault, stream));
}

void TrainerImpl::enqueueStep()
{
    InFlight f;
    f.snap = snapshot();
    const StepValues sv = nextStep();
    f.slot = nextSlot;
    nextSlot = (nextSlot + 1) % kSlots;
    launchStep(sv, nullptr, statusSlots.p + f.slot);
    ++normalSteps;
    ++iteration;
    if (freeEvents.empty()) {
        cudaEvent_t e;
        U3DG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        freeEvents.push_back(e);
    }
    f.done = freeEvents.back();
    freeEvents.pop_back();
    U3DG_CUDA(cudaEventRecord(f.done, stream));
    inflight.push_back(f);
    if (iteration >= o.refine_start && iteration < o.refine_stop && iteration % o.refine_interval == 0) {
        // The densification decision needs this step's statistics: finish (and replay) first. A replay
        // inside finish() reaches this iteration again and densifies there; do not densify twice.
        finish();
        if (densifiedAt != iteration) {
            densifyAndPrune();
            densifiedAt = iteration;
        }
    }
    if (o.opacity_reset_interval > 0 && iteration < o.refine_stop && iteration % o.opacity_reset_interval == 0)
        resetOpacity();
    U3DG_CUDA(cudaMemcpyAsync(hStats.p, dStats.p, sizeof(DevStats), cudaMemcpyDeviceToHost, stream));
    PhaseTimer *tm = profiling ? timer : nullptr;
    if (tm) {
        tm->mark(7, stream);
        U3DG_CUDA(cudaEventSynchronize(tm->ev[7]));
        u3dg_phase_times &acc = tm->acc;
        acc.steps += 1;
        acc.project_ms += tm->between(0, 1);
        acc.sort_ms += tm->between(1, 2);
        acc.forward_ms += tm->between(2, 3);
        acc.loss_ms += tm->between(3, 4);
        acc.backward_ms += tm->between(4, 5);
        acc.update_ms += tm->between(5, 6);
        acc.densify_ms += tm->between(6, 7);
        acc.total_ms += tm->between(0, 7);
        U3DG_CUDA(cudaMemcpy(ws.hostCounts.p, ws.counts.p, sizeof(BinCounts), cudaMemcpyDeviceToHost));
        acc.intersections += uint64_t(std::max(ws.hostCounts.p->effTotal, 0));
        acc.gaussians += uint64_t(ws.n);
        acc.pixels += uint64_t(sv.d.cam.width) * uint64_t(sv.d.cam.height);
    }
}

bool TrainerImpl::graphEligible(int target) const
{
    if (!useGraphs || profiling || !uniformViews || normalSteps == 0 || iteration + kGraphSteps > target)
        return false;
    for (int j = 1; j <= kGraphSteps; ++j) {
        const int it = iteration + j;
        if (it >= o.refine_start && it < o.refine_stop && it % o.refine_interval == 0)
            return false;
        if (o.opacity_reset_interval > 0 && it < o.refine_stop && it % o.opacity_reset_interval == 0)
            return false;
    }
    return true;
}

bool TrainerImpl::runGraphChunk()
{
    if (!beginGraphChunk())
        return false;
    return endGraphChunk();
}

void TrainerImpl::prepareGraphChunk(StepValues *vals, int slot)
{
    constexpr int K = kGraphSteps;
    std::vector<HostSnapshot> &snaps = pendingSnaps[slot];
    snaps.assign(K, HostSnapshot{});
    for (int k = 0; k < K; ++k) {
        snaps[k] = snapshot();
        vals[k] = nextStep();
        descHost.p[slot * K + k] = vals[k].d;
        ++iteration;
    }
}

void TrainerImpl::recordGraphChunk(const StepValues *vals)
{
    for (int k = 0; k < kGraphSteps; ++k)
        launchStep(vals[k], descDev.p + k, statusDev.p + k);
    U3DG_CUDA(cudaMemcpyAsync(hStats.p, dStats.p, sizeof(DevStats), cudaMemcpyDeviceToHost, stream));
}

void TrainerImpl::uploadGraphChunk(cudaStream_t s, int slot)
{
    constexpr int K = kGraphSteps;
    U3DG_CUDA(cudaMemcpyAsync(descDev.p, descHost.p + slot * K, K * sizeof(StepDesc), cudaMemcpyHostToDevice, s));
}

void TrainerImpl::downloadGraphStatus(cudaStream_t s, int slot)
{
    constexpr int K = kGraphSteps;
    U3DG_CUDA(cudaMemcpyAsync(graphStatus.p + slot * K, statusDev.p, K * sizeof(BinCounts), cudaMemcpyDeviceToHost, s));
}

void TrainerImpl::abandonGraphChunk(int slot)
{
    restore(pendingSnaps[slot][0]);
    pendingSnaps[slot].clear();
}

void TrainerImpl::dropGraphChunk(int slot)
{
    // The host state was already rolled back past this run; its device work did nothing (sticky
    // abort), and the stream order puts any later work after it.
    pendingSnaps[slot].clear();
}

// Makes `exec` run `graph`: an in-place update when the topology allows it, else a new instance.
static void applyGraph(cudaGraphExec_t &exec, cudaGraph_t graph)
{
    bool updated = false;
    if (exec) {
        cudaGraphExecUpdateResultInfo info{};
        updated = cudaGraphExecUpdate(exec, graph, &info) == cudaSuccess && info.result == cudaGraphExecUpdateSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
    }
    if (!updated)
        U3DG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
}

bool TrainerImpl::graphStale() const
{
    return stepGraph.exec == nullptr || stepGraph.n != n || stepGraph.cur != cur || stepGraph.icap != ws.icap ||
           stepGraph.epoch != allocEpoch();
}

bool TrainerImpl::captureStepGraph(const StepValues *vals)
{
    // Keep the instantiated graph: a re-capture with the same topology (only kernel arguments and
    // grid sizes change after a densification) updates it in place, cheaper than instantiating.
    if (stepGraph.graph) {
        cudaGraphDestroy(stepGraph.graph);
        stepGraph.graph = nullptr;
    }
    const unsigned long long epoch0 = allocEpoch();
    const unsigned long long launches0 = launchCount();
    U3DG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    try {
        recordGraphChunk(vals);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(stream, &g);
        if (g)
            cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    U3DG_CUDA(cudaStreamEndCapture(stream, &stepGraph.graph));
    // The captured kernels ran no work yet: count them when the graph runs.
    stepGraph.kernels = (long long)(launchCount() - launches0);
    addLaunches(-stepGraph.kernels);
    if (allocEpoch() != epoch0) {
        // A buffer moved while the steps were being recorded: the graph may hold stale addresses.
        stepGraph.reset();
        return false;
    }
    applyGraph(stepGraph.exec, stepGraph.graph);
    ++stepGraph.captures;
    stepGraph.n = n;
    stepGraph.cur = cur;
    stepGraph.icap = ws.icap;
    stepGraph.epoch = allocEpoch();
    return true;
}

void TrainerImpl::primeGraph(int target)
{
    if (!graphEligible(target) || !graphStale())
        return;
    // Record the next run's graph with the values its steps would have, then put the host state back:
    // a capture executes nothing, so the run itself later launches the same graph unchanged.
    const HostSnapshot s = snapshot();
    StepValues vals[kGraphSteps];
    for (int k = 0; k < kGraphSteps; ++k) {
        vals[k] = nextStep();
        ++iteration;
    }
    try {
        captureStepGraph(vals);
    } catch (...) {
        restore(s);
        throw;
    }
    restore(s);
}

bool TrainerImpl::beginGraphChunk(int slot)
{
    constexpr int K = kGraphSteps;
    // This slot's pinned descriptors are rewritten below: its previous run (checked already, or dropped
    // after an overflow without a wait) must have finished reading them.
    U3DG_CUDA(cudaEventSynchronize(chunkDone[slot]));
    StepValues vals[K];
    prepareGraphChunk(vals, slot);
    if (graphStale() && !captureStepGraph(vals)) {
        abandonGraphChunk(slot);
        return false;
    }
    // One graph serves both slots: the device-side descriptors and statuses are rewritten and read
    // in stream order, and each slot keeps its own host copies.
    uploadGraphChunk(stream, slot);
    U3DG_CUDA(cudaGraphLaunch(stepGraph.exec, stream));
    downloadGraphStatus(stream, slot);
    U3DG_CUDA(cudaEventRecord(chunkDone[slot], stream));
    addLaunches(stepGraph.kernels);
    ++graphChunks;
    return true;
}

bool TrainerImpl::endGraphChunk(int slot, bool wholeStream)
{
    if (wholeStream)
        sync();
    else
        U3DG_CUDA(cudaEventSynchronize(chunkDone[slot]));
    std::vector<HostSnapshot> &snaps = pendingSnaps[slot];
    const int K = int(snaps.size());
    for (int k = 0; k < K; ++k) {
        const BinCounts c = graphStatus.p[slot * kGraphSteps + k];
        if (c.abortIter >= 0) {
            // Step k overflowed: it and every step queued after it did nothing on the device.
            restore(snaps[k]);
            snaps.clear();
            if (!wholeStream)
                sync(); // the next run, already queued, still uses the buffers about to be replaced
            ws.reserveIntersections(size_t(c.need) + size_t(c.need) / 2);
            ws.clearCounts(stream);
            ++replays;
            return false;
        }
        if (size_t(c.total) + size_t(c.total) / 4 > size_t(ws.icap)) {
            if (!wholeStream)
                sync();
            ws.reserveIntersections(size_t(c.total) + size_t(c.total) / 2);
        }
    }
    snaps.clear();
    return true;
}

BatchGraph::~BatchGraph()
{
    if (exec)
        cudaGraphExecDestroy(exec);
    if (graph)
        cudaGraphDestroy(graph);
    for (cudaEvent_t e : events)
        cudaEventDestroy(e);
}

std::vector<long long> BatchGraph::keyOf(const std::vector<TrainerImpl *> &ts)
{
    std::vector<long long> k;
    for (TrainerImpl *t : ts) {
        k.push_back(reinterpret_cast<long long>(t));
        k.push_back(t->n);
        k.push_back(t->cur);
        k.push_back(t->ws.icap);
    }
    k.push_back((long long)allocEpoch());
    return k;
}

// One round of kGraphSteps steps of every trainer in `ts` as ONE graph launch: the scenes' step
// chunks are recorded on their own streams, forked from and joined into the first trainer's stream,
// so the graph runs them concurrently. Returns false (state untouched) if the capture had to be
// dropped because a buffer moved.
static bool runCombinedRound(const std::vector<TrainerImpl *> &ts, BatchGraph &bg)
{
    constexpr int K = TrainerImpl::kGraphSteps;
    std::vector<std::vector<StepValues>> vals(ts.size(), std::vector<StepValues>(K));
    for (size_t i = 0; i < ts.size(); ++i)
        ts[i]->prepareGraphChunk(vals[i].data());
    cudaStream_t s0 = ts[0]->stream;
    const std::vector<long long> key = BatchGraph::keyOf(ts);
    if (bg.exec == nullptr || key != bg.key) {
        if (bg.graph) {
            cudaGraphDestroy(bg.graph);
            bg.graph = nullptr;
        }
        while (bg.events.size() < ts.size()) {
            cudaEvent_t e;
            U3DG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            bg.events.push_back(e);
        }
        const unsigned long long epoch0 = allocEpoch();
        const unsigned long long launches0 = launchCount();
        U3DG_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed));
        try {
            U3DG_CUDA(cudaEventRecord(bg.events[0], s0)); // fork
            for (size_t i = 1; i < ts.size(); ++i)
                U3DG_CUDA(cudaStreamWaitEvent(ts[i]->stream, bg.events[0], 0));
            for (size_t i = 0; i < ts.size(); ++i)
                ts[i]->recordGraphChunk(vals[i].data());
            for (size_t i = 1; i < ts.size(); ++i) { // join
                U3DG_CUDA(cudaEventRecord(bg.events[i], ts[i]->stream));
                U3DG_CUDA(cudaStreamWaitEvent(s0, bg.events[i], 0));
            }
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s0, &g);
            if (g)
                cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        U3DG_CUDA(cudaStreamEndCapture(s0, &bg.graph));
        bg.kernels = (long long)(launchCount() - launches0);
        addLaunches(-bg.kernels);
        if (allocEpoch() != epoch0) {
            cudaGraphDestroy(bg.graph);
            bg.graph = nullptr;
            bg.key.clear();
            for (TrainerImpl *t : ts)
                t->abandonGraphChunk();
            return false;
        }
        applyGraph(bg.exec, bg.graph);
        bg.key = key;
        ++bg.captures;
    }
    for (TrainerImpl *t : ts)
        t->uploadGraphChunk(s0);
    U3DG_CUDA(cudaGraphLaunch(bg.exec, s0));
    for (TrainerImpl *t : ts)
        t->downloadGraphStatus(s0);
    addLaunches(bg.kernels);
    ++bg.launches;
    U3DG_CUDA(cudaStreamSynchronize(s0));
    for (TrainerImpl *t : ts) {
        ++t->graphChunks;
        t->endGraphChunk();
    }
    return true;
}

void stepBatch(const std::vector<TrainerImpl *> &trainers, int count, BatchGraph *bg)
{
    const size_t S = trainers.size();
    std::vector<int> target(S);
    for (size_t i = 0; i < S; ++i)
        target[i] = std::min(trainers[i]->iteration + std::max(count, 0), trainers[i]->o.iterations);
    std::vector<char> launched(S);
    for (;;) {
        // Every unfinished scene can run a graph chunk and all are on one device: one launch for all of
        // them, once their buffers have stayed put for a round (otherwise each densification of any
        // scene would re-record the whole graph).
        std::vector<TrainerImpl *> active;
        std::vector<int> activeTarget;
        bool allEligible = true;
        for (size_t i = 0; i < S; ++i) {
            TrainerImpl &t = *trainers[i];
            if (t.iteration >= target[i] || t.cams.empty())
                continue;
            active.push_back(&t);
            activeTarget.push_back(target[i]);
            allEligible = allEligible && t.graphEligible(target[i]) && t.device == trainers[0]->device;
        }
        if (active.empty())
            break;
        if (bg != nullptr && active.size() >= 2 && allEligible) {
            U3DG_CUDA(cudaSetDevice(active[0]->device));
            for (TrainerImpl *t : active)
                t->finish();
            bool still = true;
            for (size_t i = 0; i < active.size(); ++i)
                still = still && active[i]->graphEligible(activeTarget[i]);
            const std::vector<long long> key = BatchGraph::keyOf(active);
            if (still && (key == bg->key || key == bg->lastKey)) {
                runCombinedRound(active, *bg);
                continue;
            }
            bg->lastKey = key;
        }
        std::fill(launched.begin(), launched.end(), 0);
        for (size_t i = 0; i < S; ++i) {
            TrainerImpl &t = *trainers[i];
            if (t.iteration >= target[i] || t.cams.empty())
                continue;
            U3DG_CUDA(cudaSetDevice(t.device));
            if (t.graphEligible(target[i])) {
                t.finish();
                if (t.graphEligible(target[i]) && t.beginGraphChunk())
                    launched[i] = 1;
                continue;
            }
            const int stop = std::min(target[i], t.iteration + TrainerImpl::kGraphSteps);
            while (t.iteration < stop && !t.graphEligible(target[i]))
                t.step();
        }
        for (size_t i = 0; i < S; ++i)
            if (launched[i]) {
                U3DG_CUDA(cudaSetDevice(trainers[i]->device));
                trainers[i]->endGraphChunk();
            }
    }
    for (TrainerImpl *t : trainers) {
        U3DG_CUDA(cudaSetDevice(t->device));
        t->finish();
    }
}

RasterSchedule autotuneSchedule(const u3dg_model &initial, const u3dg_image *imgs, int count, float extent,
                                const u3dg_train_options &opt)
{
    // Every candidate is deterministic: tile 32 spans four backward CTAs per tile, each with its own
    // partial slots, added in a fixed order by the chain rule.
    static const int kTiles[3] = {16, 8, 32};
    RasterSchedule best{opt.raster.tile_size, 8, 1, 1, 0.0f};
    for (int tile : kTiles) {
        // Two runs per tile: forward 16x16 blocks at depth 1 with the backward at depth 1, and forward
        // 8x8 blocks at depth 2 with the backward at depth 2 (tile 8: both forwards use 8x8 blocks, at
        // depth 1 and 2). Each times graph runs of whole steps, then profiled steps for the compositing
        // kernels' own times; the forward and backward settings are picked independently (the kernels
        // do not interact) and the tile's step time is the first run's corrected by their gains.
        float stepMs[2] = {}, fwdMs[2] = {}, bwdMs[2] = {};
        for (int d = 0; d < 2; ++d) {
            u3dg_train_options o = opt;
            o.raster.tile_size = tile;
            o.iterations = std::max(o.iterations, 64);
            TrainerImpl t(initial, imgs, count, extent, o);
            t.ws.forwardBlock = d == 0 ? 16 : 8;
            t.ws.forwardDepth = t.ws.backwardDepth = d + 1;
            t.stepTo(3 + TrainerImpl::kGraphSteps); // warm-up, including the first graph capture
            t.finish();
            cudaEvent_t e0, e1;
            U3DG_CUDA(cudaEventCreate(&e0));
            U3DG_CUDA(cudaEventCreate(&e1));
            U3DG_CUDA(cudaEventRecord(e0, t.stream));
            t.stepTo(t.iteration + 2 * TrainerImpl::kGraphSteps);
            t.finish();
            U3DG_CUDA(cudaEventRecord(e1, t.stream));
            U3DG_CUDA(cudaEventSynchronize(e1));
            U3DG_CUDA(cudaEventElapsedTime(&stepMs[d], e0, e1));
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            stepMs[d] /= float(2 * TrainerImpl::kGraphSteps);
            t.timer = new PhaseTimer();
            t.profiling = true;
            t.stepTo(t.iteration + TrainerImpl::kGraphSteps);
            t.sync();
            const u3dg_phase_times &acc = t.timer->acc;
            fwdMs[d] = acc.steps ? acc.forward_ms / float(acc.steps) : 0.0f;
            bwdMs[d] = acc.steps ? acc.backward_ms / float(acc.steps) : 0.0f;
        }
        const int f = fwdMs[1] < fwdMs[0] ? 1 : 0, b = bwdMs[1] < bwdMs[0] ? 1 : 0;
        const float ms = stepMs[0] - (fwdMs[0] - fwdMs[f]) - (bwdMs[0] - bwdMs[b]);
        if (best.msPerStep == 0.0f || ms < best.msPerStep)
            best = RasterSchedule{tile, f == 0 && tile > 8 ? 16 : 8, f + 1, b + 1, ms};
    }
    return best;
}

DensifyResult densifyOnDevice(TrainerImpl &t, std::mt19937 &rng)
{
    cudaStream_t s = t.stream;
    const int n = t.n;
    const u3dg_train_options &o = t.o;
    DensifyResult r{n, 0, 0, 0};
    if (n <= 0)
        return r;
    const size_t nn = size_t(n) + 1;
    for (DevBuf<int> *b : {&t.keep, &t.cost, &t.costScan, &t.accCost, &t.accScan, &t.isSplit, &t.splitScan, &t.keepScan})
        b->reserve(nn);
    t.firstSecond.reserve(2);
    t.dScanPartial.reserve(scanPartialEntries(n) + 1);
    const float splitScale = o.percent_dense * t.extent;
    const long long budget = o.max_gaussians > n ? (long long)o.max_gaussians - n : 0;
    const Params P = t.params();
    launchDensifyClassify(P, n, t.gradAccum.p, t.gradCount.p, t.extent, splitScale, o.prune_opacity,
                          o.densify_grad_threshold, t.opacityWasReset ? 1 : 0, t.keep.p, t.cost.p, s);
    exclusiveScan(t.cost.p, t.costScan.p, n, t.dScanPartial.p, s);
    U3DG_CUDA(cudaMemsetAsync(t.firstSecond.p, 0x7F, 2 * sizeof(int), s)); // 0x7F7F7F7F: "none" (>= n)
    launchDensifySelect(n, t.cost.p, t.costScan.p, budget, t.firstSecond.p, t.keep.p, t.accCost.p, t.isSplit.p, s);
    exclusiveScan(t.keep.p, t.keepScan.p, n, t.dScanPartial.p, s);
    exclusiveScan(t.accCost.p, t.accScan.p, n, t.dScanPartial.p, s);
    exclusiveScan(t.isSplit.p, t.splitScan.p, n, t.dScanPartial.p, s);
    t.hCounts.reserve(4);
    U3DG_CUDA(cudaMemcpyAsync(t.hCounts.p + 0, t.keepScan.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(t.hCounts.p + 1, t.accScan.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaMemcpyAsync(t.hCounts.p + 2, t.splitScan.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    U3DG_CUDA(cudaStreamSynchronize(s));
    const int kept = t.hCounts.p[0], added = t.hCounts.p[1], splits = t.hCounts.p[2];
    // Split samples: 6 per accepted split, in index order, c = 0..1, k = 0..2 (Trainer.cpp:114,145-150).
    // A fresh distribution per call, as the reference constructs one per densifyAndPrune.
    std::normal_distribution<float> normal(0.0f, 1.0f);
    const size_t ns = size_t(splits) * 6;
    t.hNormals.resize(std::max<size_t>(ns, 1));
    for (size_t k = 0; k < ns; ++k)
        t.hNormals[k] = normal(rng);
    t.normals.reserve(std::max<size_t>(ns, 1));
    if (ns > 0)
        U3DG_CUDA(cudaMemcpyAsync(t.normals.p, t.hNormals.data(), ns * sizeof(float), cudaMemcpyHostToDevice, s));
    const int other = 1 - t.cur;
    launchDensifyWrite(P, t.moment1(), t.moment2(), t.paramsOf(other, 0), t.paramsOf(other, 1), t.paramsOf(other, 2), n,
                       t.keep.p, t.keepScan.p, t.accCost.p, t.accScan.p, t.isSplit.p, t.splitScan.p, kept, t.normals.p,
                       std::log(1.6f), s);
    U3DG_CUDA(cudaGetLastError());
    t.cur = other;
    r.newCount = kept + added;
    r.splits = splits;
    r.clones = added - 2 * splits;
    r.pruned = n - kept - splits;
    t.n = r.newCount;
    U3DG_CUDA(cudaMemsetAsync(t.gradAccum.p, 0, size_t(t.n) * sizeof(float), s));
    U3DG_CUDA(cudaMemsetAsync(t.gradCount.p, 0, size_t(t.n) * sizeof(int), s));
    // hNormals is read by the copy above; keep it valid until the copy is done.
    U3DG_CUDA(cudaStreamSynchronize(s));
    return r;
}

void TrainerImpl::densifyAndPrune()
{
    const DensifyResult r = densifyOnDevice(*this, rng);
    lastPruned = r.pruned;
    lastClones = r.clones;
    lastSplits = r.splits;
    // More Gaussians usually means more intersections: keep 16 per Gaussian of headroom.
    if (size_t(ws.icap) < 16 * size_t(n))
        ws.reserveIntersections(16 * size_t(n));
}

void TrainerImpl::crop(const u3dg_crop_box &box, float minOpacity)
{
    finish();
    const int other = 1 - cur;
    const size_t kept = cropKeep(params(), n, box, minOpacity, keep, keepScan, dScanPartial, stream);
    // Parameters and both moments (three consecutive arenas) into the other arena set, then flip.
    launchCropWrite(arena[cur].p, cap, arena[other].p, cap, 3, n, keep.p, keepScan.p, stream);
    U3DG_CUDA(cudaGetLastError());
    cur = other;
    n = int(kept);
    U3DG_CUDA(cudaMemsetAsync(gradAccum.p, 0, size_t(std::max(n, 1)) * sizeof(float), stream));
    U3DG_CUDA(cudaMemsetAsync(gradCount.p, 0, size_t(std::max(n, 1)) * sizeof(int), stream));
    sync();
}

void TrainerImpl::resetOpacity()
{
    // logit(0.01f) in host float arithmetic (GaussianModel.h:13, Trainer.cpp:173).
    const float cap01 = std::log(0.01f / (1.0f - 0.01f));
    launchOpacityReset(params().opac, moment1().opac, moment2().opac, n, cap01, ws.counts.p, stream);
    opacityWasReset = true;
}

float TrainerImpl::evaluatePsnr()
{
    finish();
    waitUploads();
    if (cams.empty())
        return 0.0f;
    constexpr int kSq = 297; // sqDiff partial blocks + 1 (loss.cu)
    psnrSums.reserve(cams.size() * kSq);
    for (size_t v = 0; v < cams.size(); ++v) {
        ws.forwardChecked(params(), n, cams[v], o.raster, nullptr, 0, stream);
        const size_t count = size_t(cams[v].width) * cams[v].height * 3;
        launchPsnrU8(ws.rgb.p, images.p + imageOffset[v], count, psnrSums.p + v * kSq, stream);
    }
    std::vector<double> sums(cams.size() * kSq);
    U3DG_CUDA(cudaMemcpyAsync(sums.data(), psnrSums.p, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    double total = 0;
    for (size_t v = 0; v < cams.size(); ++v) {
        const size_t count = size_t(cams[v].width) * cams[v].height * 3;
        const double mse = sums[v * kSq + kSq - 1] / double(std::max<size_t>(count, 1));
        total += mse <= 1e-12 ? 99.0f : float(-10.0 * std::log10(mse)); // psnr, Loss.cpp:187-196
    }
    return float(total / double(cams.size()));
}

void TrainerImpl::render(const u3dg_camera &c, float *hostRgb)
{
    finish();
    ws.forwardChecked(params(), n, c, o.raster, nullptr, 0, stream);
    U3DG_CUDA(cudaMemcpyAsync(hostRgb, ws.rgb.p, size_t(c.width) * c.height * 3 * sizeof(float), cudaMemcpyDeviceToHost,
                              stream));
    sync();
}

void TrainerImpl::download(u3dg_model &out)
{
    finish();
    copyArenaToModel(arena[cur].p, cap, size_t(n), out, stream);
    sync();
}

} // namespace u3dg
