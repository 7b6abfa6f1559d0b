// binning.cu - tile binning on the GPU (Rasterizer::binTiles, Rasterizer.cpp:206-261).
//
// The reference sorts the visible Gaussians by the float bits of their depth with a stable LSD
// radix sort (ties keep index order), then buckets them per tile in that order, so every tile list
// is depth-sorted. Here the same order comes from two stable radix sorts:
//   1. (depth bits, Gaussian id) over all Gaussians -> depth rank; invisible ones get key
//      0xFFFFFFFF and sort last;
//   2. intersections are emitted in depth-rank order (an exclusive scan of per-rank tile counts
//      gives each Gaussian its slots), keyed by tile id, and sorted stably by the tile id only.
// Within a tile the emission order, i.e. (depth bits, id), survives, which is exactly the
// reference's list.
//
// The intersection count is only known on the device, so nothing here waits for the host: the tile
// sort reads its item count from device memory (the depth sort takes the host-known Gaussian count),
// grids are sized for the capacity, and a capacity check (in the scan of the per-rank tile counts)
// turns an overflow into an empty bin list plus a flag the host reads later (it then grows the
// buffers and replays the step).
//
// Sorting: stable LSD passes, 8-bit digits for the depth keys and one 11-bit pass for tile ids (up to
// 2048 tiles; that pass's scatter also writes the tile lists' Gaussian ids and, in block 0, the tile
// offsets, which are the exclusive scan of its digit totals). A pass is
// three kernels: per-block digit histograms, a per-digit scan over the blocks, and a scatter whose
// in-block ranks come from warp match-any votes. Every block owns one contiguous chunk of the items
// and walks it in rounds of kTile items.

#include "tile_cull.cuh"

#include <algorithm>
#include <climits>

namespace u3dg {

namespace {

constexpr int kThreads = 256;
constexpr int kItemsPerThread = 4;
constexpr int kTile = kThreads * kItemsPerThread; // items per block round
constexpr int kWarps = kThreads / 32;
// Blocks of a radix pass at most (each owns a contiguous chunk of the items in rounds of kTile).
#ifndef U3DG_RADIX_MAX_BLOCKS
#define U3DG_RADIX_MAX_BLOCKS (148 * 6)
#endif
constexpr int kMaxBlocks = U3DG_RADIX_MAX_BLOCKS;
constexpr int kWideBits = 11; // one pass sorts tile ids up to 2048; other sorts use 8-bit digits

// Block-wide exclusive scan of one int per thread (blockDim == 256); returns the block total.
__device__ __forceinline__ int blockExclusiveScan(int v, int &total)
{
    __shared__ int warpSums[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kWarps ? warpSums[lane] : 0;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o)
                w += y;
        }
        if (lane < kWarps)
            warpSums[lane] = w; // inclusive
    }
    __syncthreads();
    total = warpSums[kWarps - 1];
    const int before = warp > 0 ? warpSums[warp - 1] : 0;
    __syncthreads();
    return before + x - v;
}

// The contiguous item range of block b when n items are split over G blocks in rounds of kTile.
__device__ __forceinline__ void chunkOf(int n, int G, int b, int &begin, int &end)
{
    const long long per = (long long)G * kTile;
    const int rounds = int((n + per - 1) / per);
    const long long chunk = (long long)rounds * kTile;
    begin = int(std::min<long long>(n, b * chunk));
    end = int(std::min<long long>(n, begin + chunk));
}

template <int DB>
// keys, or with pairs set the (key, value) pairs' keys.
__global__ void __launch_bounds__(kThreads) radixHistKernel(const uint32_t *keys, const uint2 *pairs, const int *nPtr,
                                                            int nHost, int shift, int *hist, int G)
{
    pdlEntry();
    constexpr int R = 1 << DB;
    __shared__ int counts[R];
    for (int d = threadIdx.x; d < R; d += kThreads)
        counts[d] = 0;
    __syncthreads();
    int begin, end;
    chunkOf(nPtr ? *nPtr : nHost, G, blockIdx.x, begin, end);
    for (int i = begin + threadIdx.x; i < end; i += kThreads)
        atomicAdd(&counts[((pairs ? pairs[i].x : keys[i]) >> shift) & uint32_t(R - 1)], 1);
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kThreads)
        hist[size_t(d) * G + blockIdx.x] = counts[d];
}

// One block per digit: exclusive scan of that digit's row of G block counts; rowTotals[d] = sum.
__global__ void __launch_bounds__(kThreads) radixRowScanKernel(int *hist, int G, int *rowTotals)
{
    pdlEntry();
    int *row = hist + size_t(blockIdx.x) * G;
    int carry = 0;
    for (int c0 = 0; c0 < G; c0 += kThreads) {
        const int i = c0 + threadIdx.x;
        const int v = i < G ? row[i] : 0;
        int total;
        const int ex = blockExclusiveScan(v, total);
        if (i < G)
            row[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0)
        rowTotals[blockIdx.x] = carry;
}

// Stable scatter of one pass with 2^DB digits. Per round of kTile items, each warp ranks its items
// among equal digits with match-any votes and keeps per-digit counts (at most 128, one byte) in shared
// memory; an item's position is its digit's base + the counts of the warps before it (they hold
// earlier items) + its rank in its warp. After the round the last item of each (warp, digit) advances
// the digit's base and clears that count, so only the touched counts are reset.
// kTiles (the single pass of a tile sort, digit = tile): instead of the sorted keys and values, the
// scatter writes each entry's (Gaussian id, emission index) pair (fin.entries[pos]), and block 0
// writes the tile offsets, which are the digit bases it starts from.
// Where a pass of the depth sort keeps its items: (key, value) pairs in and out, so each item is one
// load and one scattered 8-byte store; the last pass writes the values only (the keys are done).
struct PairIO {
    const uint2 *in;    // when set: the items (keysIn / valsIn unused)
    uint2 *out;         // when set: write (key, value) pairs
    uint32_t *valsOnly; // when set: write the values only
};

template <int DB, bool kTiles = false>
__global__ void __launch_bounds__(kThreads) radixScatterKernel(const uint32_t *keysIn, const uint32_t *valsIn,
                                                               uint32_t *keysOut, uint32_t *valsOut, const int *nPtr,
                                                               int nHost, int shift, const int *hist, const int *rowTotals,
                                                               int G, TileFinish fin, PairIO io)
{
    pdlEntry();
    const int n = nPtr ? *nPtr : nHost;
    constexpr int R = 1 << DB;
    __shared__ uint8_t warpCounts[kWarps][R];
    __shared__ int base[R];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int begin, end;
    chunkOf(n, G, blockIdx.x, begin, end);
    for (int k = threadIdx.x; k < kWarps * R; k += kThreads)
        (&warpCounts[0][0])[k] = 0;
    {
        // Digit base: exclusive scan of the digit totals, plus this block's row prefix.
        int carry = 0;
        for (int c0 = 0; c0 < R; c0 += kThreads) {
            const int d = c0 + threadIdx.x;
            int total;
            const int ex = blockExclusiveScan(rowTotals[d], total);
            base[d] = carry + ex + hist[size_t(d) * G + blockIdx.x];
            carry += total;
        }
    }
    __syncthreads();
    if (kTiles && blockIdx.x == 0) {
        for (int d = threadIdx.x; d < fin.tiles; d += kThreads)
            fin.tileOffsets[d] = base[d]; // block 0's row prefix is zero
        if (threadIdx.x == 0)
            fin.tileOffsets[fin.tiles] = n;
    }
    const uint32_t lanesBelow = (1u << lane) - 1u;
    uint8_t *myCounts = warpCounts[warp];
    for (int r0 = begin; r0 < end; r0 += kTile) {
        const int first = r0 + warp * (32 * kItemsPerThread);
        uint32_t key[kItemsPerThread], val[kItemsPerThread];
        int digit[kItemsPerThread], local[kItemsPerThread];
#pragma unroll
        for (int r = 0; r < kItemsPerThread; ++r) {
            const int i = first + r * 32 + lane;
            const bool valid = i < end;
            if (io.in) {
                const uint2 kv = valid ? io.in[i] : make_uint2(0u, 0u);
                key[r] = kv.x;
                val[r] = kv.y;
            } else {
                key[r] = valid ? keysIn[i] : 0u;
                val[r] = valid ? (valsIn ? valsIn[i] : uint32_t(i)) : 0u;
            }
            const int d = valid ? int((key[r] >> shift) & uint32_t(R - 1)) : R;
            digit[r] = d;
            local[r] = 0;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            int before = 0;
            if (valid) {
                before = myCounts[d];
                local[r] = before + __popc(peers & lanesBelow);
            }
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1)
                myCounts[d] = uint8_t(before + __popc(peers));
            __syncwarp();
        }
        __syncthreads();
        bool last[kItemsPerThread];
#pragma unroll
        for (int r = 0; r < kItemsPerThread; ++r) {
            const int d = digit[r];
            last[r] = false;
            if (d < R) {
                int cross = 0;
                for (int w = 0; w < warp; ++w)
                    cross += warpCounts[w][d];
                const int pos = base[d] + cross + local[r];
                if (kTiles) {
                    fin.entries[pos] = make_int2(fin.emitGid[val[r]], int(val[r]));
                } else if (io.out) {
                    io.out[pos] = make_uint2(key[r], val[r]);
                } else if (io.valsOnly) {
                    io.valsOnly[pos] = val[r];
                } else {
                    keysOut[pos] = key[r];
                    valsOut[pos] = val[r];
                }
                last[r] = local[r] == int(myCounts[d]) - 1;
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kItemsPerThread; ++r)
            if (last[r])
                atomicAdd(&base[digit[r]], int(myCounts[digit[r]]));
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kItemsPerThread; ++r)
            if (last[r])
                myCounts[digit[r]] = 0;
        __syncthreads();
    }
}

// Capacity check of a bin pass on its intersection count t: the usable count is t, or 0 when t
// exceeds the intersection buffers or a previous step already aborted (the abort is sticky until the
// host clears it). iteration identifies the aborted step for the host.
__device__ __forceinline__ void checkCapacity(int t, int capacity, BinCounts *c, int iteration, const StepDesc *desc)
{
    if (desc)
        iteration = desc->iteration;
    const bool over = t < 0 || t > capacity;
    if (over) {
        if (c->abortIter < 0)
            c->abortIter = iteration;
        c->need = max(c->need, t < 0 ? INT_MAX : t);
    }
    c->total = t;
    c->effTotal = (over || c->abortIter >= 0) ? 0 : t;
}

// Exclusive scan, reduce-then-scan over a host-known n.
constexpr int kScanTile = kThreads * 8;

// The scan's input element i: in[i], or in[perm[i]] with a permutation (the per-Gaussian tile counts
// taken in depth-rank order).
__device__ __forceinline__ int scanInput(const int *in, const uint32_t *perm, int i)
{
    return in[perm ? int(perm[i]) : i];
}

__global__ void __launch_bounds__(kThreads) scanReduceKernel(const int *in, const uint32_t *perm, int n, int *partial)
{
    pdlEntry();
    const int base = blockIdx.x * kScanTile;
    int s = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = base + r * kThreads + threadIdx.x;
        if (i < n)
            s += scanInput(in, perm, i);
    }
    int total;
    blockExclusiveScan(s, total);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads) scanPartialKernel(int *partial, int B)
{
    pdlEntry();
    int carry = 0;
    for (int c0 = 0; c0 < B; c0 += kThreads) {
        const int i = c0 + threadIdx.x;
        const int v = i < B ? partial[i] : 0;
        int total;
        const int ex = blockExclusiveScan(v, total);
        if (i < B)
            partial[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0)
        partial[B] = carry;
}

// cap.counts (may be null): block 0 also runs the bin pass's capacity check on the total.
__global__ void __launch_bounds__(kThreads) scanDownsweepKernel(const int *in, const uint32_t *perm, int *out, int n,
                                                                const int *partial, int B, ScanCapacity cap)
{
    pdlEntry();
    const int base = blockIdx.x * kScanTile + threadIdx.x * 8;
    int v[8];
    int s = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        v[r] = (base + r < n) ? scanInput(in, perm, base + r) : 0;
        s += v[r];
    }
    int total;
    int run = blockExclusiveScan(s, total) + partial[blockIdx.x];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (base + r < n)
            out[base + r] = run;
        run += v[r];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out[n] = partial[B];
        if (cap.counts != nullptr)
            checkCapacity(partial[B], cap.capacity, cap.counts, cap.iteration, cap.desc);
    }
}

// Capacity check of a bin pass on its scan total (checkCapacity), when the scan had no kernels to
// fold it into.
__global__ void capacityKernel(const int *total, int capacity, BinCounts *c, int iteration, const StepDesc *desc)
{
    pdlEntry();
    checkCapacity(*total, capacity, c, iteration, desc);
}

// One warp per 32 consecutive depth ranks (grid-stride): the warp writes its ranks' intersections in
// order, 32 at a time. Each lane finds the rank of its intersection as the last of the warp's 32 start
// offsets not above it (a binary search over lanes with shuffles; empty ranks share their start with
// the next rank, so the search lands on the rank that owns the slot), then its tile in that rank's
// rectangle (row-major, as the reference's ty/tx loops).
__global__ void __launch_bounds__(256) emitKernel(const uint32_t *sortedIds, const int *offs, const int4 *rect, int n,
                                                  const BinCounts *c, int tilesX, const SplatRec *cullRec, int tileSize,
                                                  const uint32_t *rowTab, uint32_t *keys, int *emitGid)
{
    pdlEntry();
    const int total = c->effTotal;
    if (total <= 0)
        return;
    const int lane = threadIdx.x & 31;
    const int warps = int((gridDim.x * blockDim.x) >> 5);
    for (int w = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w * 32 < n; w += warps) {
        const int r = w * 32 + lane;
        const bool valid = r < n;
        const int o = valid ? offs[r] : INT_MAX;
        int g = 0;
        int4 q = make_int4(0, 0, 1, 1);
        if (valid) {
            g = int(sortedIds[r]);
            q = rect[g];
        }
        const int first = offs[w * 32], last = min(offs[min(w * 32 + 32, n)], total);
        for (int e0 = first; e0 < last; e0 += 32) {
            const int e = e0 + lane;
            int l = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int oc = __shfl_sync(0xffffffffu, o, l + step);
                if (oc <= e)
                    l += step;
            }
            const int ol = __shfl_sync(0xffffffffu, o, l);
            const int gl = __shfl_sync(0xffffffffu, g, l);
            const int qx = __shfl_sync(0xffffffffu, q.x, l), qy = __shfl_sync(0xffffffffu, q.y, l);
            const int qz = __shfl_sync(0xffffffffu, q.z, l), qw = __shfl_sync(0xffffffffu, q.w, l);
            if (e < last) {
                int k = e - ol;
                int ty, tx;
                if (cullRec == nullptr) {
                    const int wdt = qz - qx;
                    ty = qy + k / wdt;
                    tx = qx + k % wdt;
                } else {
                    // The k-th reachable tile in row-major order: the Gaussian's row table, then (rows
                    // beyond it) the rows' spans.
                    // One 32-byte row (two vector loads) per Gaussian; entries past its rows are unused.
                    const uint4 *tab = reinterpret_cast<const uint4 *>(rowTab + size_t(gl) * kCullRows);
                    const uint4 t0 = tab[0], t1 = tab[1];
                    const uint32_t tv[kCullRows] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w};
                    const int rows = qw - qy;
                    ty = -1;
                    tx = qx;
                    int before = 0;
#pragma unroll
                    for (int i = 0; i < kCullRows; ++i) {
                        if (i >= rows)
                            break;
                        const uint32_t v = tv[i];
                        const int through = int(v & 0xffffu);
                        if (k < through) {
                            ty = qy + i;
                            tx = int(v >> 16) + (k - before);
                            break;
                        }
                        before = through;
                    }
                    if (ty < 0) { // rare: more rows than the table holds
                        k -= before;
                        const CullShape csl = cullShape(cullRec, gl);
                        const int4 qq = make_int4(qx, qy, qz, qw);
                        ty = qy;
                        for (int row = qy + kCullRows; row < qw; ++row) {
                            int c0, c1;
                            cullSpan(csl, qq, row, tileSize, c0, c1);
                            if (k < c1 - c0) {
                                ty = row;
                                tx = c0 + k;
                                break;
                            }
                            k -= c1 - c0;
                        }
                    }
                }
                keys[e] = uint32_t(ty * tilesX + tx);
                emitGid[e] = gl;
            }
        }
    }
}

__global__ void finalizeKernel(const uint32_t *sortedEmit, const int *emitGid, const BinCounts *c, int2 *entries)
{
    pdlEntry();
    const int total = c->effTotal;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
        const uint32_t e = sortedEmit[s];
        entries[s] = make_int2(emitGid[e], int(e));
    }
}

__global__ void tileOffsetsKernel(const uint32_t *sortedKeys, const BinCounts *c, int tiles, int *tileOffsets)
{
    pdlEntry();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > tiles)
        return;
    const int total = c->effTotal;
    int lo = 0, hi = total; // first s with key >= t
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (int(sortedKeys[mid]) < t)
            lo = mid + 1;
        else
            hi = mid;
    }
    tileOffsets[t] = (t == tiles) ? total : lo;
}

inline int grid(long long n, int t) { return int((n + t - 1) / t); }

} // namespace

int radixBlocks(int nMax) { return std::max(1, std::min(kMaxBlocks, (nMax + kTile - 1) / kTile)); }

size_t radixHistEntries(int nMax) { return size_t(1 << kWideBits) * size_t(radixBlocks(nMax)); }

int radixDigits() { return 1 << kWideBits; }

int radixSortPairs(uint32_t *keysA, uint32_t *keysB, uint32_t *valsA, uint32_t *valsB, const int *nDev, int nMax,
                   int bits, int *hist, int *rowTotals, uint32_t **keysOut, uint32_t **valsOut, cudaStream_t s,
                   const TileFinish *fin, int nHost)
{
    uint32_t *kin = keysA, *kout = keysB, *vout = valsB;
    const uint32_t *vin = nullptr;
    const int G = radixBlocks(nMax);
    // Keys of up to 11 bits (tile ids) in one pass of 2048 digits; longer keys in 8-bit passes (three
    // 11-bit passes over 32-bit depth keys measured slower than four 8-bit ones).
    const bool wide = bits <= kWideBits;
    if (!wide)
        fin = nullptr;
    const int db = wide ? kWideBits : 8;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += db, ++passes) {
        if (wide) {
            { launchPdl(radixHistKernel<kWideBits>, G, kThreads, 0, s, kin, nullptr, nDev, nHost, shift, hist, G); countLaunch(); }
            { launchPdl(radixRowScanKernel, 1 << kWideBits, kThreads, 0, s, hist, G, rowTotals); countLaunch(); }
            if (fin != nullptr)
                { launchPdl(radixScatterKernel<kWideBits, true>, G, kThreads, 0, s, kin, vin, kout, vout, nDev, nHost, shift, hist, rowTotals, G, *fin, PairIO{}); countLaunch(); }
            else
                { launchPdl(radixScatterKernel<kWideBits>, G, kThreads, 0, s, kin, vin, kout, vout, nDev, nHost, shift, hist, rowTotals, G, TileFinish{}, PairIO{}); countLaunch(); }
        } else {
            { launchPdl(radixHistKernel<8>, G, kThreads, 0, s, kin, nullptr, nDev, nHost, shift, hist, G); countLaunch(); }
            { launchPdl(radixRowScanKernel, 1 << 8, kThreads, 0, s, hist, G, rowTotals); countLaunch(); }
            { launchPdl(radixScatterKernel<8>, G, kThreads, 0, s, kin, vin, kout, vout, nDev, nHost, shift, hist, rowTotals, G, TileFinish{}, PairIO{}); countLaunch(); }
        }
        uint32_t *nk = kin;
        kin = kout;
        kout = nk;
        vin = vout;
        vout = (vout == valsB) ? valsA : valsB;
    }
    *keysOut = kin;
    *valsOut = const_cast<uint32_t *>(vin);
    return passes;
}

void radixSortDepth(const uint32_t *keys, uint2 *pairsA, uint2 *pairsB, uint32_t *sortedIds, int n, int *hist,
                    int *rowTotals, cudaStream_t s)
{
    const int G = radixBlocks(std::max(n, 1));
    const uint2 *pin = nullptr;
    uint2 *bufs[2] = {pairsA, pairsB};
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        const PairIO io{pin, pass < 3 ? bufs[pass & 1] : nullptr, pass < 3 ? nullptr : sortedIds};
        { launchPdl(radixHistKernel<8>, G, kThreads, 0, s, keys, pin, nullptr, n, shift, hist, G); countLaunch(); }
        { launchPdl(radixRowScanKernel, 1 << 8, kThreads, 0, s, hist, G, rowTotals); countLaunch(); }
        { launchPdl(radixScatterKernel<8>, G, kThreads, 0, s, keys, nullptr, nullptr, nullptr, nullptr, n, shift, hist, rowTotals, G, TileFinish{}, io); countLaunch(); }
        pin = io.out;
    }
}

size_t scanPartialEntries(int n) { return size_t((n + kScanTile - 1) / kScanTile) + 1; }

static void scanLaunches(const int *in, const uint32_t *perm, int *out, int n, int *partial, const ScanCapacity &cap,
                         cudaStream_t s)
{
    const int B = (n + kScanTile - 1) / kScanTile;
    { launchPdl(scanReduceKernel, B, kThreads, 0, s, in, perm, n, partial); countLaunch(); }
    { launchPdl(scanPartialKernel, 1, kThreads, 0, s, partial, B); countLaunch(); }
    { launchPdl(scanDownsweepKernel, B, kThreads, 0, s, in, perm, out, n, partial, B, cap); countLaunch(); }
}

void exclusiveScan(const int *in, int *out, int n, int *partial, cudaStream_t s)
{
    if (n <= 0) {
        cudaMemsetAsync(out, 0, sizeof(int), s);
        return;
    }
    scanLaunches(in, nullptr, out, n, partial, ScanCapacity{0, nullptr, 0, nullptr}, s);
}

void exclusiveScanChecked(const int *in, const uint32_t *perm, int *out, int n, int *partial, const ScanCapacity &cap,
                          cudaStream_t s)
{
    if (n <= 0) {
        cudaMemsetAsync(out, 0, sizeof(int), s);
        launchCapacityCheck(out, cap.capacity, cap.counts, cap.iteration, s, cap.desc);
        return;
    }
    scanLaunches(in, perm, out, n, partial, cap, s);
}

size_t cullRowEntries(size_t n) { return n * kCullRows; }


void launchCapacityCheck(const int *total, int capacity, BinCounts *c, int iteration, cudaStream_t s,
                         const StepDesc *desc)
{
    { launchPdl(capacityKernel, 1, 1, 0, s, total, capacity, c, iteration, desc); countLaunch(); }
}

void launchEmit(const uint32_t *sortedIds, const int *offs, const int4 *rect, int n, const BinCounts *c, int capacity,
                int tilesX, const SplatRec *cullRec, int tileSize, const uint32_t *rowTab, uint32_t *keys, int *emitGid,
                cudaStream_t s)
{
    if (n > 0 && capacity > 0)
        { launchPdl(emitKernel, std::min(grid((long long)(n + 31) / 32 * 32, 256), 148 * 16), 256, 0, s, sortedIds, offs, rect, n, c, tilesX, cullRec, tileSize, rowTab, keys, emitGid); countLaunch(); }
}

void launchFinalizeBins(const uint32_t *sortedKeys, const uint32_t *sortedEmit, const int *emitGid, const BinCounts *c,
                        int capacity, int tiles, int2 *entries, int *tileOffsets, cudaStream_t s)
{
    if (capacity > 0)
        { launchPdl(finalizeKernel, std::min(grid(capacity, 256), 148 * 16), 256, 0, s, sortedEmit, emitGid, c, entries); countLaunch(); }
    { launchPdl(tileOffsetsKernel, grid(tiles + 1, 256), 256, 0, s, sortedKeys, c, tiles, tileOffsets); countLaunch(); }
}

} // namespace u3dg
