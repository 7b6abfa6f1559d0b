// engine.h - host-side objects behind the C ABI: device buffers, the raster workspace and the trainer.
#pragma once

#include "kernels.h"

#include <condition_variable>
#include <cstdio>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace u3dg {

// A failed CUDA call, carried to the C ABI boundary and turned into a status code there.
struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char *expr, const char *file, int line)
        : std::runtime_error(std::string(expr) + ": " + cudaGetErrorString(c) + " (" + file + ":" + std::to_string(line) + ")"),
          code(c)
    {
    }
};

struct StatusError : std::runtime_error {
    int status;
    StatusError(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

// Thread-local message behind u3dg_last_error; returns `code`.
int setError(int code, const std::string &msg);
const char *lastError();

// Runs f, turning every C++ exception into a status code and a message (the C ABI never throws).
template <class F>
int guardedCall(F &&f)
{
    try {
        f();
        return U3DG_OK;
    } catch (const StatusError &e) {
        return setError(e.status, e.what());
    } catch (const CudaError &e) {
        const int code = (e.code == cudaErrorMemoryAllocation) ? U3DG_ERR_OOM
                         : (e.code == cudaErrorNoDevice || e.code == cudaErrorInsufficientDriver) ? U3DG_ERR_NO_DEVICE
                                                                                                   : U3DG_ERR_CUDA;
        return setError(code, e.what());
    } catch (const std::bad_alloc &) {
        return setError(U3DG_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return setError(U3DG_ERR_STATE, e.what());
    }
}

#define U3DG_CUDA(x)                                                   \
    do {                                                               \
        cudaError_t e_ = (x);                                          \
        if (e_ != cudaSuccess)                                         \
            throw ::u3dg::CudaError(e_, #x, __FILE__, __LINE__);       \
    } while (0)

// Counts device and pinned allocations in this process. A captured CUDA graph bakes buffer addresses
// into its nodes; it is reused only while this count is unchanged since its capture.
unsigned long long allocEpoch();
void bumpAllocEpoch();

// Device array with capacity growth (cudaMalloc only when it has to grow). A buffer may instead hold a
// slice of a DeviceSlab (owned false): the slab frees it, and a growth past the slice moves the buffer
// to an allocation of its own.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    bool owned = true;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) {
            if (owned)
                cudaFree(p);
            bumpAllocEpoch();
        }
        p = nullptr;
        cap = 0;
        owned = true;
    }
    // Takes n elements at mem, which the caller keeps alive (a slab slice).
    void adopt(void *mem, size_t n)
    {
        release();
        p = static_cast<T *>(mem);
        cap = n;
        owned = false;
        bumpAllocEpoch();
    }
    // Ensures room for n elements; contents are NOT preserved when it grows.
    void reserve(size_t n, bool exact = false)
    {
        if (n <= cap && p)
            return;
        release();
        size_t c = exact ? n : std::max(n, cap + cap / 2);
        if (c == 0)
            c = 1;
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&p), c * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            throw StatusError(U3DG_ERR_OOM, "cudaMalloc of " + std::to_string(c * sizeof(T)) + " bytes failed: " +
                                                cudaGetErrorString(e));
        }
        cap = c;
        bumpAllocEpoch();
    }
};

// One device allocation carved into many buffers. A cudaMalloc that has to map new device memory costs
// about 0.3 ms whatever its size, so a trainer plans its ~40 buffers (add) and allocates them together
// (commit) instead of paying that once per buffer. Slices start on 256-byte boundaries. The slab must
// outlive the buffers' use of their slices (declare it before them).
class DeviceSlab {
  public:
    DeviceSlab() = default;
    DeviceSlab(const DeviceSlab &) = delete;
    DeviceSlab &operator=(const DeviceSlab &) = delete;
    ~DeviceSlab()
    {
        for (void *b : bases)
            cudaFree(b);
    }
    // Plans n elements for b (nothing if b already holds that many).
    template <class T>
    void add(DevBuf<T> &b, size_t n)
    {
        n = std::max<size_t>(n, 1);
        if (b.p && b.cap >= n)
            return;
        items.push_back({&b, n * sizeof(T), n, [](void *buf, void *mem, size_t k) { static_cast<DevBuf<T> *>(buf)->adopt(mem, k); }});
    }
    // Allocates everything planned since the last commit and hands out the slices.
    void commit();
    size_t bytes() const { return total; }

  private:
    struct Item {
        void *buf;
        size_t bytes, count;
        void (*adopt)(void *, void *, size_t);
    };
    std::vector<Item> items;
    std::vector<void *> bases;
    size_t total = 0;
};

// Pinned host array (for asynchronous device->host reads).
template <class T>
struct HostPinned {
    T *p = nullptr;
    size_t cap = 0;
    ~HostPinned()
    {
        if (p)
            cudaFreeHost(p);
    }
    // Grows geometrically: page-locking is slow and cudaFreeHost waits for the device.
    void reserve(size_t n)
    {
        if (n <= cap && p)
            return;
        if (p)
            cudaFreeHost(p);
        p = nullptr;
        const size_t c = std::max<size_t>(std::max(n, cap * 2), 1);
        U3DG_CUDA(cudaMallocHost(reinterpret_cast<void **>(&p), c * sizeof(T)));
        cap = c;
        bumpAllocEpoch();
    }
};

unsigned long long launchCount();
void addLaunches(long long k);
void checkSettings(const u3dg_raster_settings &st);
// Uploads a host model into the params slot of an arena of capacity `cap`.
void copyModelToArena(float *base, size_t cap, const u3dg_model &m, cudaStream_t s);
void checkCamera(const u3dg_camera &cam);

// Everything Rasterizer::forward keeps between forward and backward (Rasterizer.h:57-89), on the GPU.
struct RasterWorkspace {
    // per Gaussian
    DevBuf<SplatRec> rec;
    DevBuf<uint32_t> depthKey, depthOrder; // depth sort key per Gaussian; Gaussian ids in depth order
    DevBuf<uint2> depthPairs[2];           // the depth sort's (key, id) pairs between passes
    DevBuf<float> depth;
    DevBuf<int4> rect;
    DevBuf<int> radius, cnt, offs, scanPartial, hist, rowTotals; // cnt: tiles per Gaussian (projection)
    DevBuf<uint32_t> rowTab; // tile culling: per Gaussian, the first rows' spans (emission lookup)
    DevBuf<uint8_t> flags;
    DevBuf<float4> cov2d;
    DevBuf<float> g2d; // per Gaussian: summed 2D gradients (chain-rule input)
    // per intersection (capacity icap)
    DevBuf<uint32_t> iKeys0, iKeys1, iVals0, iVals1;
    DevBuf<int> emitGid;
    DevBuf<int2> entries; // per tile-sorted entry: Gaussian id, emission index
    DevBuf<float> partial;             // partialSlots arrays of icap * 9 floats
    int icap = 0;
    int partialSlots = 1;              // slot arrays the backward needs: (tile size / 16)^2 above 16
    // per tile / pixel
    DevBuf<int> tileOffsets, nContrib;
    DevBuf<int> blockOrder, blockCounters; // compositing schedule: pixel blocks by list length, counters
    DevBuf<float> rgb, finalT;
    // device-side sizes of the last pass and their pinned host copy
    DevBuf<BinCounts> counts;
    HostPinned<BinCounts> hostCounts;

    int n = 0, tilesX = 0, tilesY = 0;
    // Compositing schedule (none changes a result): the forward kernel's pixel block edge (8 or 16,
    // for tiles of 16 and 32 pixels) and the list entries each compositing thread stages per
    // shared-memory batch (1 or 2).
    int forwardBlock = 8, forwardDepth = 1, backwardDepth = 1;
    // Tile culling: list a Gaussian only in the tiles of its rectangle that its contributing ellipse
    // can reach (trainers; the rasterizer unit boundary keeps the reference's lists).
    bool cullTiles = false;
    // Culling applies while tile rows fit the row table's 16-bit cumulative counts (< 8192 tiles).
    bool culled() const { return cullTiles && tilesX < 8192; }
    u3dg_camera cam{};
    u3dg_raster_settings st{};
    uint32_t *sortedIds = nullptr;

    RasterWorkspace();
    // Sizes the intersection buffers for `capacity` entries (waits for the device if they grow).
    void reserveIntersections(size_t capacity);
    // Sizes the per-Gaussian buffers for `count` Gaussians (project() grows them on demand otherwise).
    void reserveGaussians(size_t count);
    // The same sizes (and the per-pixel buffers for views of up to `pixels` pixels and `tiles` tiles at
    // the tile size st.tile_size), planned into a slab instead of allocated one by one.
    void planIntersections(DeviceSlab &slab, size_t capacity);
    void planGaussians(DeviceSlab &slab, size_t count);
    void planPixels(DeviceSlab &slab, size_t pixels, int tilesX, int tilesY, int tileSize);
    // Clears the overflow / abort record (stream-ordered).
    void clearCounts(cudaStream_t stream);
    // desc (may be null): the camera of a graph-captured step (see StepDesc).
    void project(const Params &P, int count, const u3dg_camera &c, const u3dg_raster_settings &s, const float *shRest,
                 int shDegree, cudaStream_t stream, const StepDesc *desc = nullptr);
    // Depth sort + tile binning from depthKey / rect / radius. Never waits for the device: an overflow of
    // the intersection buffers is recorded in `counts` (tagged with `iteration`) and bins nothing.
    void bin(cudaStream_t stream, int iteration, const StepDesc *desc = nullptr);
    void composite(cudaStream_t stream);
    void forward(const Params &P, int count, const u3dg_camera &c, const u3dg_raster_settings &s, const float *shRest,
                 int shDegree, cudaStream_t stream, int iteration)
    {
        project(P, count, c, s, shRest, shDegree, stream);
        bin(stream, iteration);
        composite(stream);
    }
    // A forward that is complete when it returns: waits, and on an overflow grows the intersection
    // buffers and runs again. For the unit entry points and evaluation, not the training loop.
    void forwardChecked(const Params &P, int count, const u3dg_camera &c, const u3dg_raster_settings &s,
                        const float *shRest, int shDegree, cudaStream_t stream);
    // Intersections binned by the last completed pass (valid after a wait).
    int total() const { return hostCounts.p->effTotal; }
    // Compositing backward into `partial`.
    void backwardComposite(const float *dLdRgb, cudaStream_t stream);
    RasterArgs rasterArgs() const;
    ChainArgs chainArgs(const Params &P) const;

  private:
    // Calls f(buffer, elements) for every per-Gaussian / per-intersection buffer at the given size.
    template <class F>
    void eachGaussianBuffer(size_t nn, F &&f);
    template <class F>
    void eachIntersectionBuffer(size_t capacity, F &&f);
    static size_t checkedIntersections(size_t capacity);
};

// CUDA events around the phases of a profiled step.
struct PhaseTimer {
    static constexpr int kEvents = 8;
    cudaEvent_t ev[kEvents];
    u3dg_phase_times acc{};
    PhaseTimer()
    {
        for (auto &e : ev)
            U3DG_CUDA(cudaEventCreate(&e));
    }
    ~PhaseTimer()
    {
        for (auto &e : ev)
            cudaEventDestroy(e);
    }
    void mark(int k, cudaStream_t s) { U3DG_CUDA(cudaEventRecord(ev[k], s)); }
    float between(int a, int b)
    {
        float ms = 0;
        U3DG_CUDA(cudaEventElapsedTime(&ms, ev[a], ev[b]));
        return ms;
    }
};

// Host-side trainer state before a step: what a replay restores.
struct HostSnapshot {
    int iteration = 0;
    size_t orderPos = 0;
    std::vector<int> order;
    std::mt19937 rng;
    int adamStep = 0;
    bool opacityWasReset = false;
};

// The host-side values of one step (what StepDesc carries to a graph-captured step).
struct StepValues {
    size_t view = 0;
    StepDesc d{};
};

// A CUDA graph of kGraphSteps consecutive training steps, and what it was captured for.
struct StepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long epoch = 0;
    long long kernels = 0;  // kernel nodes per launch
    long long captures = 0; // captures so far (instantiated, or applied to the instance as an update)
    int n = -1, cur = -1, icap = -1;
    void reset()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        n = cur = icap = -1;
    }
    ~StepGraph() { reset(); }
};

// A queued step whose device-side status has not been checked yet.
struct InFlight {
    HostSnapshot snap;
    cudaEvent_t done = nullptr;
    int slot = 0; // pinned status slot
};

// Training images copied to the device by a host thread while training starts (trainers created
// with background upload). Views are copied in the order the first epoch will use them (the first
// shuffle of the view order, computed from a copy of the trainer's generator), each on the copy
// stream followed by an event; a step makes its stream wait for its view's event first, so no step
// reads an image before it has arrived and the results are the same as with images uploaded at
// creation.
struct ImageUploader {
    std::thread thread;
    cudaStream_t copy = nullptr;
    std::vector<cudaEvent_t> ready; // per view
    std::vector<int> position;      // per view: its place in the upload order
    std::vector<char> waited;       // per view: the trainer's stream already waits for it
    std::mutex m;
    std::condition_variable cv;
    int issued = 0;                 // copies issued so far, in upload order (guarded by m)
    std::string error;              // first failure of the thread (guarded by m)
    bool joined = false;
};

// The GPU Trainer (Trainer.h:47-93, Trainer.cpp).
struct TrainerImpl {
    int device = 0;
    cudaStream_t stream = nullptr;
    u3dg_train_options o{};
    float extent = 1.0f;
    size_t cap = 0;
    int n = 0;
    int cur = 0;                      // which arena holds the live model
    DeviceSlab slab;                  // the buffers sized at creation (declared first: freed last)
    DevBuf<float> arena[2];           // params, m, v: 3 * 14 * cap floats each
    DevBuf<float> gradAccum;
    DevBuf<int> gradCount;
    std::vector<u3dg_camera> cams;
    std::vector<size_t> imageOffset;
    DevBuf<uint8_t> images;
    RasterWorkspace ws;
    DevBuf<float> dLoss, abc;
    DevBuf<double> lossBlockSums, psnrSums;
    DevBuf<DevStats> dStats;
    HostPinned<DevStats> hStats;
    // densification scratch
    DevBuf<int> keep, cost, costScan, accCost, accScan, isSplit, splitScan, keepScan, firstSecond, dScanPartial;
    DevBuf<float> normals;
    HostPinned<int> hCounts;
    std::vector<float> hNormals; // split samples drawn on the host (pageable: copied once per densification)

    std::mt19937 rng;
    std::vector<int> order;
    size_t orderPos = 0;
    int iteration = 0;
    int adamStep = 0;
    bool opacityWasReset = false;
    int lastPruned = 0, lastClones = 0, lastSplits = 0;
    int replays = 0;                  // steps replayed after an intersection-buffer overflow
    int densifiedAt = -1;             // iteration of the last densification

    // Steps run ahead of their status check by at most kLag steps.
    static constexpr int kLag = 2;
    static constexpr int kSlots = 8;
    std::vector<InFlight> inflight;
    std::vector<cudaEvent_t> freeEvents;
    HostPinned<BinCounts> statusSlots; // kSlots pinned copies of the bin counts, one per queued step
    int nextSlot = 0;

    bool profiling = false;
    PhaseTimer *timer = nullptr;

    // Graph execution of runs of steps without densification, opacity reset or profiling, when every
    // view has the same size: kGraphSteps steps per launch, their values in descriptors on the device.
    static constexpr int kGraphSteps = 10;
    bool useGraphs = true;
    bool uniformViews = false;
    // Graph runs of kGraphSteps steps. A trainer keeps one run in flight while the host prepares and
    // launches the next (stepTo), alternating two slots of host-side descriptors and statuses; the
    // graph reads its descriptors from, and writes its statuses to, device buffers that each launch
    // refills and copies out in stream order. Batches use slot 0.
    StepGraph stepGraph;
    DevBuf<StepDesc> descDev;          // kGraphSteps
    HostPinned<StepDesc> descHost;     // 2 * kGraphSteps
    DevBuf<BinCounts> statusDev;       // kGraphSteps
    HostPinned<BinCounts> graphStatus; // 2 * kGraphSteps
    cudaEvent_t chunkDone[2] = {nullptr, nullptr};
    void resetGraphs() { stepGraph.reset(); }
    long long graphChunks = 0;        // graph launches so far
    long long normalSteps = 0;        // steps launched one by one (the first step is never a graph)

    // backgroundUpload: the images are copied by a host thread while the first steps run (the
    // caller's pixel buffers must stay valid until waitUploads() returns or the trainer is gone).
    TrainerImpl(const u3dg_model &initial, const u3dg_image *imgs, int count, float sceneExtent,
                const u3dg_train_options &opt, bool backgroundUpload = false);
    ~TrainerImpl();
    // Blocks until every image is on the device (no-op without background upload); afterwards the
    // caller's pixel buffers may be released.
    void waitUploads();
    std::unique_ptr<ImageUploader> uploader;
    // Makes the trainer's stream wait until view v's image has arrived (background upload).
    void requireView(size_t v);

    Params params() { return paramsAt(arena[cur].p, cap); }
    Params moment1() { return paramsAt(arena[cur].p + 14 * cap, cap); }
    Params moment2() { return paramsAt(arena[cur].p + 28 * cap, cap); }
    Params paramsOf(int which, int k) { return paramsAt(arena[which].p + size_t(k) * 14 * cap, cap); }

    bool done() const { return iteration >= o.iterations; }
    // Trainer::step: queues one step (after checking the step kLag before it).
    void step();
    // Runs steps until `target` iterations are reached (or done), replaying after overflows.
    void stepTo(int target);
    // Waits for every queued step and replays any that overflowed; afterwards the state is final.
    void finish();
    void densifyAndPrune();
    void resetOpacity();
    // cropModel (Crop.cpp:44-52) of the live model with its Adam moments; statistics restart at zero.
    void crop(const u3dg_crop_box &box, float minOpacity);
    float evaluatePsnr();
    void render(const u3dg_camera &c, float *hostRgb);
    void download(u3dg_model &out);
    void sync();

private:
    void startUploads(const u3dg_image *imgs, int count);
    HostSnapshot snapshot() const;
    void restore(const HostSnapshot &s);
    void enqueueStep();
    // Advances the host state by one step (view order, learning rates, Adam step) and returns its values.
    StepValues nextStep();
    // Queues the device work of one step; desc (may be null) is where graph-captured kernels read the values.
    void launchStep(const StepValues &sv, const StepDesc *desc, BinCounts *statusDst);
public:
    // Whether the next kGraphSteps steps can run as one graph launch.
    bool graphEligible(int target) const;
    // Runs kGraphSteps steps through the step graph (capturing it when stale). Returns false after an
    // overflow (the state is rolled back to the overflowed step, as checkOldest does).
    bool runGraphChunk();
    // runGraphChunk in two halves, so several trainers can have a chunk in flight at once: begin
    // advances the host state, captures the graph if stale and launches it (no wait; false when a
    // capture had to be discarded, with the state restored); end waits and checks the statuses.
    // Launches the next 10 steps as one graph run in `slot` (false: nothing launched, the host state
    // is back where it was). endGraphChunk waits for the slot's run (the whole stream when
    // `wholeStream`) and checks its statuses; false means a step overflowed and the host state was
    // rolled back to it (a run launched after it in the other slot then did nothing on the device and
    // must be dropped with dropGraphChunk).
    bool beginGraphChunk(int slot = 0);
    // Whether the step graph must be recorded again before its next launch.
    bool graphStale() const;
    // Records (and instantiates) the step graph for steps with these values; false when a buffer moved
    // during the recording (the graph is dropped).
    bool captureStepGraph(const StepValues *vals);
    // Records the graph the next run toward `target` will launch, without running anything and with
    // the host state unchanged (so a timed run does not include the recording).
    void primeGraph(int target);
    bool endGraphChunk(int slot = 0, bool wholeStream = true);
    void dropGraphChunk(int slot);
    // The parts of beginGraphChunk, for a graph that holds several trainers' chunks (stepBatch, slot 0):
    // advance the host state by kGraphSteps steps, record their launches on this trainer's stream
    // (inside a capture), upload their descriptors on stream s, or undo the host-state advance.
    void prepareGraphChunk(StepValues *vals, int slot = 0);
    void recordGraphChunk(const StepValues *vals);
    void uploadGraphChunk(cudaStream_t s, int slot = 0);
    // After a launch: the run's statuses into the slot's host copy (stream order).
    void downloadGraphStatus(cudaStream_t s, int slot = 0);
    void abandonGraphChunk(int slot = 0);

private:
    std::vector<HostSnapshot> pendingSnaps[2]; // host state before each step of the slot's run
    // Checks the oldest queued step; returns false (after rolling back) when it had overflowed.
    bool checkOldest();
};

// crop.cu: cropModel / suggestCropBox / modelBounds (Crop.cpp:12-62) on device arrays. cropKeep fills
// keep[i] and its exclusive scan pos (n + 1 entries) and returns the kept count (waits for the stream);
// launchCropWrite copies the kept rows of `arenas` consecutive 14-float arenas; quantileBoxOnDevice is
// quantileBox (Crop.cpp:12-40) with the per-axis quantiles taken by a device sort.
size_t cropKeep(const Params &P, int n, const u3dg_crop_box &box, float minOpacity, DevBuf<int> &keep,
                DevBuf<int> &pos, DevBuf<int> &scratch, cudaStream_t s);
void launchCropWrite(const float *src, size_t srcCap, float *dst, size_t dstCap, int arenas, int n, const int *keep,
                     const int *pos, cudaStream_t s);
u3dg_crop_box quantileBoxOnDevice(const Params &P, int n, float lo, float hi, float margin, float minOpacity,
                                  cudaStream_t s);

// Densification on device arrays (shared by the trainer and the unit entry point).
struct DensifyResult {
    int newCount;
    int pruned, clones, splits;
};
DensifyResult densifyOnDevice(TrainerImpl &t, std::mt19937 &rng);

// One CUDA graph holding a round of kGraphSteps steps of several trainers (stepBatch), with what it
// was recorded for.
struct BatchGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> key, lastKey; // trainers, their sizes and buffers, allocation count
    std::vector<cudaEvent_t> events;     // fork / join events of the recording
    long long kernels = 0, captures = 0, launches = 0;
    static std::vector<long long> keyOf(const std::vector<TrainerImpl *> &ts);
    BatchGraph() = default;
    BatchGraph(const BatchGraph &) = delete;
    BatchGraph &operator=(const BatchGraph &) = delete;
    ~BatchGraph();
};

// Steps every trainer by `count` iterations (or to its end), interleaving them on their own streams:
// each round launches a graph chunk (or up to kGraphSteps single steps) per trainer before waiting
// for any, so small scenes run concurrently on the GPU. When every unfinished trainer can run a graph
// chunk and their buffers have not moved since the previous round, the round is ONE launch of a
// graph holding all of their chunks (bg, may be null: no combined graph).
void stepBatch(const std::vector<TrainerImpl *> &trainers, int count, BatchGraph *bg = nullptr);

// Tile size (8 or 16: the sizes whose results are deterministic), forward pixel block (8 or 16) and
// compositing batch depths (1 or 2 staged list entries per thread per batch, for the forward and the
// backward kernel) with the shortest step time for a scene, timed on throwaway trainers started from
// the same model.
struct RasterSchedule {
    int tileSize, forwardBlock, forwardDepth, backwardDepth;
    float msPerStep;
};
RasterSchedule autotuneSchedule(const u3dg_model &initial, const u3dg_image *imgs, int count, float extent,
                                const u3dg_train_options &opt);

} // namespace u3dg

// The C ABI's trainer handle (include/u3dg.h). Handles owned by a batch are borrowed by callers.
struct u3dg_trainer {
    std::unique_ptr<u3dg::TrainerImpl> impl;
    bool ownedByBatch = false;
};
