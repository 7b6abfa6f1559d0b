// noalloc.cu - the photometric loss on caller-owned device buffers, with no allocation in the call.
//
// No reference counterpart. u3dg_photometric_loss (photometricLoss, Loss.cpp:47-184) takes host
// images and allocates its device buffers and SSIM scratch on every call. This variant runs the same
// two loss kernels and the same finalize kernel (loss.cu) on device pointers the caller owns; its
// temporaries live in one file-scope device array, so the call makes no cudaMalloc, no cudaFree and
// no call into an allocating library routine.
//
// Scratch (gNoAllocScratch, 11.2 MB per device context that uses this entry point):
//   [0, 3 * kMaxBlocks) doubles      per-block sums (L1, SSIM, squared error), 3 per loss block
//   next 4 floats                    total, L1, SSIM, PSNR from the finalize kernel
//   from a 256-byte boundary         the SSIM partial maps, 9 floats per pixel
// Nothing in it has to start at zero: every element a call reads was written earlier in that call
// (each loss block writes its three sums; with lambda > 0 the forward kernel writes all nine maps
// of every pixel before the backward kernel reads them, and with lambda = 0 no kernel reads them;
// the finalize kernel writes the four values).
//
// Limits: width * height <= kMaxPixels (640 x 480) and at most 2048 blocks of 32 x 16 pixels (the
// loss kernels run one CTA per block and channel: kMaxBlocks = 3 x 2048); larger requests are
// rejected with U3DG_ERR_CAPACITY before anything is launched.
//
// Set-up: the first call in each device context, with that device current, resolves the array's
// address there with cudaGetSymbolAddress (which loads this module into the context) and keeps it
// with the context's id. A later call in a different context of that device (after cudaDeviceReset
// destroyed the old one) resolves it again. Make the first call on a device, and the first after a
// reset, before any stream capture on that device begins.
//
// Overlapping calls: all calls on one device share the one scratch array. Each call holds a
// per-device lock from its first launch until it has synchronised `stream`, so calls from several
// host threads run one after another instead of overwriting each other's scratch; two processes have
// separate contexts and separate copies of the array.
//
// The call returns the loss values on the host, so it waits for `stream` to finish the loss before
// it returns (and before it releases the lock); the four result floats are read back on `stream`
// into the caller's stack, which needs no pinned buffer because the wait follows at once.

#include "engine.h"
#include "kernels.h"

#include <cudaTypedefs.h>

#include <mutex>

using namespace u3dg;

namespace {

constexpr size_t kMaxPixels = 640 * 480;
constexpr int kMaxBlocks = 3 * 2048; // 2048 tiles of 32x16 pixels, one loss block per tile and channel
constexpr size_t kSumsDoubles = 3 * size_t(kMaxBlocks);
constexpr size_t kValsOffset = kSumsDoubles;                           // in doubles; 4 floats = 2 doubles
constexpr size_t kMapsOffset = (kValsOffset + 2 + 31) / 32 * 32;       // 256-byte boundary, in doubles
constexpr size_t kScratchDoubles = kMapsOffset + (9 * kMaxPixels + 1) / 2;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double gNoAllocScratch[kScratchDoubles];

std::mutex gDeviceLock[kMaxDevices];
// The array's address in each device's context, and the id of the context it was resolved in; read
// and written under that device's lock.
double *gScratchAddress[kMaxDevices] = {};
unsigned long long gScratchContext[kMaxDevices] = {};

// Id of the calling thread's current context (cuCtxGetId through the runtime's driver entry point);
// 0 when no context is current yet.
unsigned long long currentContextId()
{
    static PFN_cuCtxGetId getId = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuCtxGetId>(fn);
    }();
    if (!getId)
        throw StatusError(U3DG_ERR_CUDA, "cuCtxGetId is not available from the CUDA driver");
    unsigned long long id = 0;
    return getId(nullptr, &id) == CUDA_SUCCESS ? id : 0;
}

} // namespace

extern "C" int u3dg_photometric_loss_noalloc(const float *render, const float *target, int width, int height,
                                             float lambda, float *grad, u3dg_loss_value *out, void *stream)
{
    return guardedCall([&] {
        if (!render || !target || !grad || width <= 0 || height <= 0)
            throw StatusError(U3DG_ERR_INVALID_ARG, "invalid loss arguments");
        const size_t pixels = size_t(width) * size_t(height);
        if (pixels > kMaxPixels)
            throw StatusError(U3DG_ERR_CAPACITY, "image larger than the 307200-pixel (640x480) no-allocation scratch");
        const int blocks = lossBlocks(width, height);
        if (blocks > kMaxBlocks)
            throw StatusError(U3DG_ERR_CAPACITY, "image needs more than 2048 loss blocks of 32x16 pixels");
        int device = -1;
        U3DG_CUDA(cudaGetDevice(&device));
        if (device < 0 || device >= kMaxDevices)
            throw StatusError(U3DG_ERR_INVALID_ARG, "device index out of range");
        std::lock_guard<std::mutex> lock(gDeviceLock[device]);
        unsigned long long ctx = currentContextId();
        if (ctx == 0) {
            U3DG_CUDA(cudaSetDevice(device)); // creates and binds the device's primary context (CUDA 12)
            ctx = currentContextId();
            if (ctx == 0)
                throw StatusError(U3DG_ERR_CUDA, "no CUDA context is current on the device");
        }
        if (!gScratchAddress[device] || gScratchContext[device] != ctx) {
            void *p = nullptr;
            U3DG_CUDA(cudaGetSymbolAddress(&p, gNoAllocScratch));
            gScratchAddress[device] = static_cast<double *>(p);
            gScratchContext[device] = ctx;
        }
        double *base = gScratchAddress[device];
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        const LossScratch ls{reinterpret_cast<float *>(base + kMapsOffset), base, blocks};
        float *vals = reinterpret_cast<float *>(base + kValsOffset);
        launchLoss(render, target, nullptr, width, height, lambda, grad, ls, s);
        launchLossFinalize(ls, width, height, lambda, nullptr, 0, nullptr, vals, vals + 3, s);
        U3DG_CUDA(cudaGetLastError());
        float v[4] = {0, 0, 0, 0};
        if (out)
            U3DG_CUDA(cudaMemcpyAsync(v, vals, sizeof(v), cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaStreamSynchronize(s));
        if (out) {
            out->total = v[0];
            out->l1 = v[1];
            out->ssim = v[2];
        }
    });
}
