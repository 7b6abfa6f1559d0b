// init.cu - initGaussiansFromPoints (GaussianModel.cpp:68-144) with its neighbour search on the GPU.
//
// The reference sizes each initial Gaussian from the mean squared distance to its 3 nearest
// neighbours, found through a hash grid: every point scans the buckets of the 27 cells around its
// own, where a bucket holds every point whose cell hashes to that key (hash collisions included, and
// a key met twice among the 27 is scanned twice). That search is O(27 x bucket) per point and takes
// 2 s on the host for 300k points. Here the host builds the grid exactly as the reference does
// (buildInitGrid: bounds, cell size, cell keys, key-sorted index) and finishes the model
// (finishInitFromNeighbours: mean, square root, log, colours); one GPU thread per point runs the
// 27-cell scan in the same order with the same comparisons, each squared distance rounded like the
// host's ((ex ex + ey ey) + ez ez, no fused multiply-add), so the result is bit-identical to the
// host version.

#include "engine.h"
#include "host_io.h"

#include <cfloat>
#include <climits>

namespace u3dg {

namespace {

__global__ void __launch_bounds__(256) initNeighboursKernel(const float *xyz, const int *cell, const long long *keys,
                                                            const uint32_t *ids, int n, float *best)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
    const int cx = cell[3 * i], cy = cell[3 * i + 1], cz = cell[3 * i + 2];
    float b0 = FLT_MAX, b1 = FLT_MAX, b2 = FLT_MAX;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                const long long key = (static_cast<long long>(cx + dx) * 73856093LL) ^
                                      (static_cast<long long>(cy + dy) * 19349663LL) ^
                                      (static_cast<long long>(cz + dz) * 83492791LL);
                int lo = 0, hi = n; // first sorted key >= key
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (keys[mid] < key)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                for (int it = lo; it < n && keys[it] == key; ++it) {
                    const int j = int(ids[it]);
                    if (j == i)
                        continue;
                    const float ex = __fsub_rn(xyz[3 * j], xi), ey = __fsub_rn(xyz[3 * j + 1], yi),
                                ez = __fsub_rn(xyz[3 * j + 2], zi);
                    float d2 = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
                    // Insertion into the three smallest, as the reference's swap chain.
                    if (d2 < b0) {
                        const float t = b0;
                        b0 = d2;
                        d2 = t;
                    }
                    if (d2 < b1) {
                        const float t = b1;
                        b1 = d2;
                        d2 = t;
                    }
                    if (d2 < b2)
                        b2 = d2;
                }
            }
    best[3 * i] = b0;
    best[3 * i + 1] = b1;
    best[3 * i + 2] = b2;
}

} // namespace

void initGaussiansFromPointsDevice(const float *xyz, const float *rgb, size_t n, u3dg_model &out)
{
    if (n == 0)
        return;
    if (n > size_t(INT_MAX / 3))
        throw StatusError(U3DG_ERR_CAPACITY, "too many points");
    InitGrid g;
    buildInitGrid(xyz, n, g);
    std::vector<int> cell(n * 3);
    for (size_t i = 0; i < n; ++i) {
        cell[3 * i] = g.cx[i];
        cell[3 * i + 1] = g.cy[i];
        cell[3 * i + 2] = g.cz[i];
    }
    struct Stream {
        cudaStream_t s = nullptr;
        ~Stream()
        {
            if (s)
                cudaStreamDestroy(s);
        }
    } st;
    U3DG_CUDA(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    const cudaStream_t s = st.s;
    std::vector<float> best(n * 3);
    {
        DevBuf<float> dXyz, dBest;
        DevBuf<int> dCell;
        DevBuf<long long> dKeys;
        DevBuf<uint32_t> dIds;
        dXyz.reserve(n * 3, true);
        dBest.reserve(n * 3, true);
        dCell.reserve(n * 3, true);
        dKeys.reserve(n, true);
        dIds.reserve(n, true);
        U3DG_CUDA(cudaMemcpyAsync(dXyz.p, xyz, n * 3 * sizeof(float), cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(dCell.p, cell.data(), n * 3 * sizeof(int), cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(dKeys.p, g.keys.data(), n * sizeof(long long), cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(dIds.p, g.ids.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        { initNeighboursKernel<<<int((n + 255) / 256), 256, 0, s>>>(dXyz.p, dCell.p, dKeys.p, dIds.p, int(n), dBest.p); countLaunch(); }
        U3DG_CUDA(cudaGetLastError());
        U3DG_CUDA(cudaMemcpyAsync(best.data(), dBest.p, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaStreamSynchronize(s));
    }
    finishInitFromNeighbours(xyz, rgb, n, g.cell, best.data(), out);
}

} // namespace u3dg
