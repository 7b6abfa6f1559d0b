// kernels.h - host-side launch interface of the CUDA kernels (no torch, plain pointers).
#pragma once

#include "common.cuh"

#include <utility>

namespace u3dg {

// Programmatic dependent launch (sm_90+): the kernels of a training step are launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, so the GPU may launch a kernel as soon as every CTA
// of the previous kernel in the stream has exited, before that kernel's completion and memory flush are
// signalled to the stream; each such kernel starts with pdlEntry(), which waits until the previous
// kernel has completed and its memory is visible (griddepcontrol.wait). No kernel triggers its
// dependents early (griddepcontrol.launch_dependents): measured on a 300k-Gaussian 640x480 step, an
// early trigger let waiting CTAs occupy SM slots the running kernel's tail still needed (1.297 ms per
// step against 1.276 without it). Ordering is the plain stream order's; what overlaps is one kernel's
// launch and CTA set-up with the previous one's completion. In a kernel launched without the attribute
// the instruction does nothing.
__device__ __forceinline__ void pdlEntry()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launches `kernel` on stream s with programmatic stream serialisation (see pdlEntry; the kernel must
// call pdlEntry() before it reads anything an earlier kernel wrote).
template <typename... KArgs, typename... Args>
inline void launchPdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Device-side sizes of one bin pass. The host never waits for them inside a step: it reads the
// struct back asynchronously and checks it one step later.
struct BinCounts {
    int total;     // tile-Gaussian intersections found by the scan
    int effTotal;  // intersections actually binned: total, or 0 after an overflow / abort
    int abortIter; // -1, or the first step whose intersections did not fit (sticky until cleared)
    int need;      // largest intersection count that did not fit
    int pad[4];
};

// The values of one training step that change from step to step (view, target image, iteration,
// Adam step sizes). Launches given a StepDesc read them from device memory instead of their by-value
// arguments, so a captured CUDA graph of training steps serves any views and learning rates.
struct StepDesc {
    u3dg_camera cam;
    const uint8_t *target; // the view's uint8 image
    int iteration;         // iteration count before the step (0-based step index)
    float stepSize[5];     // Adam: lr / bc1 per group
    float invSqrtBc2;
    int pad[2];
};

// Outputs of the projection kernel, one entry per Gaussian.
struct ProjOut {
    SplatRec *rec;      // raster record (valid where radius > 0)
    uint32_t *depthKey; // float bits of the camera-space depth; 0xFFFFFFFF when not visible
    float *depth;       // camera-space depth (valid where radius > 0)
    int4 *rect;         // tile rectangle x0, y0, x1, y1 (exclusive)
    int *radius;        // 0 = not visible
    uint8_t *flags;     // bit0/1: J clamped in x/y; bit2..4: colour clamped
    float4 *cov2d;      // 2D covariance a, b, c (including eps2d), for inspection
    int *tileCount;     // tiles the Gaussian is listed in (0 when not visible)
    uint32_t *rowTab;   // tile culling: the first rows' spans (tile_cull.cuh, listedTiles); may be null
    int cullTiles;      // 1: list only the tiles the contributing ellipse reaches (then rowTab is set)
};

// Arguments of the chain-rule kernel (backward pass 2), optionally fused with Adam.
struct ChainArgs {
    Params params;
    int n;
    u3dg_camera cam;
    u3dg_raster_settings st;
    const int *radius;
    const SplatRec *rec;
    const uint8_t *flags;
    const int *offs;      // per rank: first intersection in emission order (n + 1 entries)
    const uint32_t *sortedIds; // Gaussian id per depth rank
    const float *partial; // per intersection, in emission order: 9 summed 2D gradients (subSlots arrays)
    int subSlots;         // slot arrays of partial (RasterArgs::subSlots), subStride floats apart
    size_t subStride;
    float *g2d;           // per Gaussian: the 9 partials summed (written by launchChain's first kernel)
    const BinCounts *counts; // the kernel does nothing when counts->abortIter >= 0
    float *gradAccum;     // |dL/dmean2d| NDC statistic (may be null)
    int *gradCount;       // visibility count (may be null)
    Params grads;         // non-Adam mode: gradients are added here
    Params m, v;          // Adam mode: moments
    float stepSize[5];    // Adam mode: lr / bc1 per group
    float invSqrtBc2;
    const StepDesc *desc; // when set: cam, stepSize and invSqrtBc2 come from here
};

// gaussian.cu
// desc (may be null): the camera comes from desc->cam (no spherical harmonics in that mode).
void launchProject(const Params &P, int n, const u3dg_camera &cam, const u3dg_raster_settings &st, int tilesX,
                   int tilesY, const float *shRest, int shDegree, const ProjOut &out, cudaStream_t s,
                   const StepDesc *desc = nullptr);
void launchChain(const ChainArgs &a, bool adam, cudaStream_t s);
void launchAdamSegment(float *p, const float *g, float *m, float *v, int len, float stepSize, float invSqrtBc2,
                       cudaStream_t s);
void launchDensifyClassify(const Params &P, int n, const float *gradAccum, const int *gradCount, float extent,
                           float splitScale, float pruneOpacity, float gradThreshold, int opacityWasReset, int *keep,
                           int *cost, cudaStream_t s);
void launchDensifySelect(int n, const int *cost, const int *costScan, long long budget, int *firstSecond, int *keep,
                         int *accCost, int *isSplit, cudaStream_t s);
void launchDensifyWrite(const Params &P, const Params &M, const Params &V, const Params &P2, const Params &M2,
                        const Params &V2, int n, const int *keep, const int *keepScan, const int *accCost,
                        const int *accScan, const int *isSplit, const int *splitScan, int keptTotal,
                        const float *normals, float log16, cudaStream_t s);
// Skipped when counts (may be null) records an aborted step.
void launchOpacityReset(float *opac, float *mOpac, float *vOpac, int n, float cap, const BinCounts *counts,
                        cudaStream_t s);

// binning.cu
// Blocks of a radix pass sized for at most nMax items, and the histogram entries it needs.
int radixBlocks(int nMax);
size_t radixHistEntries(int nMax);
// Outputs of a tile sort done in one pass (keys of at most 11 bits, digit = tile): instead of the
// sorted keys and values, the scatter writes every sorted entry as one 8-byte pair (entries[pos] =
// (Gaussian id = emitGid[emission index], emission index)), and the tile offsets (tiles + 1 entries;
// the last is the item count). One scattered 8-byte store per entry instead of two 4-byte ones: the
// scatter's cost is its scattered stores.
struct TileFinish {
    const int *emitGid;
    int2 *entries;
    int *tileOffsets;
    int tiles;
};
// Stable LSD radix sort of (key, value) pairs on key bits [0, bits); the item count is read on the
// device from *nDev (at most nMax), or, with nDev null, is nHost (known on the host; at most nMax);
// the initial values are the item indices. Result in *keysOut / *valsOut (one of the two buffers).
// Returns the number of passes; rowTotals needs radixDigits() entries. fin (may be null) applies when
// bits <= 11 (one pass): the sorted keys and values are then not written (fin->entries instead).
int radixSortPairs(uint32_t *keysA, uint32_t *keysB, uint32_t *valsA, uint32_t *valsB, const int *nDev, int nMax,
                   int bits, int *hist, int *rowTotals, uint32_t **keysOut, uint32_t **valsOut, cudaStream_t s,
                   const TileFinish *fin = nullptr, int nHost = 0);
int radixDigits();
// The depth sort: stable sort of the n 32-bit keys (four 8-bit passes; ties keep index order), items
// kept as (key, index) pairs between passes (pairsA / pairsB: n each); sortedIds receives the
// indices in key order.
void radixSortDepth(const uint32_t *keys, uint2 *pairsA, uint2 *pairsB, uint32_t *sortedIds, int n, int *hist,
                    int *rowTotals, cudaStream_t s);
// Exclusive prefix sum of n ints: out[0..n], out[n] = total. partial needs scanPartialEntries(n).
size_t scanPartialEntries(int n);
void exclusiveScan(const int *in, int *out, int n, int *partial, cudaStream_t s);
// The scan of in[perm[i]] (the per-Gaussian tile counts in depth-rank order), fused with the bin pass's
// capacity check (launchCapacityCheck on the total out[n], done by the scan's last kernel).
struct ScanCapacity {
    int capacity;
    BinCounts *counts;
    int iteration;
    const StepDesc *desc;
};
void exclusiveScanChecked(const int *in, const uint32_t *perm, int *out, int n, int *partial, const ScanCapacity &cap,
                          cudaStream_t s);
// Entries of the per-Gaussian row table of tile culling (ProjOut::rowTab) for n Gaussians.
size_t cullRowEntries(size_t n);
// Checks *total against the intersection capacity (see BinCounts); exclusiveScanChecked does the same
// inside its last kernel.
void launchCapacityCheck(const int *total, int capacity, BinCounts *c, int iteration, cudaStream_t s,
                         const StepDesc *desc = nullptr);
// Emission of the intersections in depth-rank order: tile key and Gaussian id per intersection (the
// same tiles as launchRankCounts counted).
void launchEmit(const uint32_t *sortedIds, const int *offs, const int4 *rect, int n, const BinCounts *c, int capacity,
                int tilesX, const SplatRec *cullRec, int tileSize, const uint32_t *rowTab, uint32_t *keys, int *emitGid,
                cudaStream_t s);
// After a tile sort of several passes (more than 2048 tiles): the (Gaussian id, emission index) pair of
// every sorted entry and the tile offsets (a binary search in the sorted keys). A one-pass tile sort
// writes both itself (TileFinish).
void launchFinalizeBins(const uint32_t *sortedKeys, const uint32_t *sortedEmit, const int *emitGid, const BinCounts *c,
                        int capacity, int tiles, int2 *entries, int *tileOffsets, cudaStream_t s);

// raster.cu
struct RasterArgs {
    const int *tileOffsets;
    const int2 *entries; // per tile-sorted entry: Gaussian id, emission index (where backward stores partials)
    const SplatRec *rec;
    int width, height, tileSize, tilesX;
    float bg[3];
    float minAlpha, minTransmittance;
    // Persistent scheduling over the pixel blocks (PB x PB, PB = 8 for tile size 8, else 16).
    int blocksX, blocksY;
    const int *blockOrder; // pixel blocks, heaviest tile list first (launchBlockOrder)
    int *counters;         // 4 ints, zero between launches: forward [0..1], backward [2..3]
    int forwardBlock;      // pixel block edge of the forward kernel: 8 or 16 (tiles > 8 only; same results)
    int forwardDepth;      // list entries staged per thread per batch, forward: 1 or 2 (same results)
    int backwardDepth;     // the same for the backward kernel
    // Tiles larger than the backward's 16x16 pixel block are covered by several CTAs: each writes its
    // sums into its own slot array (slot = the block's position in its tile, row-major), subSlots
    // arrays of subStride floats apart, and the chain rule adds a Gaussian's slots in slot order.
    int subSlots;
    size_t subStride;
};
// Orders the pixel blocks by the list length of their tile, longest first (log-scale buckets), into
// order[blocksX * blocksY].
void launchBlockOrder(const RasterArgs &a, int *order, cudaStream_t s);
void launchCompositeForward(const RasterArgs &a, float *rgb, float *finalT, int *nContrib, cudaStream_t s);
// partial: 9 floats per intersection in emission order, in a.subSlots slot arrays (every slot of every
// entry is written: no zeroing needed).
void launchCompositeBackward(const RasterArgs &a, const float *dLdRgb, const float *finalT, const int *nContrib,
                             float *partial, cudaStream_t s);

// loss.cu
struct LossScratch {
    float *abc;        // 3 maps x 3 channels x P
    double *blockSums; // 3 doubles per block: l1, ssim, squared error
    int blocks;
};
int lossBlocks(int width, int height);
// target is either float (targetF) or uint8 (targetU8, converted as float(u8) * (1/255f)).
// desc (may be null): the uint8 target comes from desc->target.
void launchLoss(const float *render, const float *targetF, const uint8_t *targetU8, int width, int height, float lambda,
                float *grad, const LossScratch &ls, cudaStream_t s, const StepDesc *desc = nullptr);
// Reduces the block sums into the step's LossValue / PSNR and updates the EMA stats
// (Trainer.cpp:88-92) unless counts (may be null) records an aborted step. out3 (may be null) gets
// total, l1, ssim; psnrOut (may be null) the PSNR.
// desc (may be null): iteration is desc->iteration + 1.
void launchLossFinalize(const LossScratch &ls, int width, int height, float lambda, DevStats *stats, int iteration,
                        const BinCounts *counts, float *out3, float *psnrOut, cudaStream_t s,
                        const StepDesc *desc = nullptr);
// PSNR of the render against a uint8 target, accumulated in double (evaluatePsnr).
void launchPsnrU8(const float *render, const uint8_t *target, size_t count, double *sumOut, cudaStream_t s);
void launchPsnrF(const float *a, const float *b, size_t count, double *sumOut, cudaStream_t s);
// TrainImage::quantize on the device: lround(clamp(v, 0, 1) * 255) per value.
void launchQuantize(const float *rgb, size_t count, uint8_t *out, cudaStream_t s);

} // namespace u3dg
