// warmstart_host.cu - the learned warm-start behind the C ABI: the MLP object (parameters, Adam
// state, forward, gradients, training on the GPU) and the initialisation of a GaussianModel from an
// SfM point cloud through it.

#include "engine.h"
#include "host_io.h"
#include "warmstart.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>

using namespace u3dg;

namespace {

struct LayerOffsets {
    size_t w[kWarmLayers], b[kWarmLayers];
    LayerOffsets()
    {
        size_t o = 0;
        for (int l = 0; l < kWarmLayers; ++l) {
            w[l] = o;
            o += size_t(kWarmOut[l]) * kWarmIn[l];
            b[l] = o;
            o += size_t(kWarmOut[l]);
        }
    }
};

const LayerOffsets &offsets()
{
    static const LayerOffsets lo;
    return lo;
}

void requireGpu()
{
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess || c == 0) {
        cudaGetLastError();
        throw StatusError(U3DG_ERR_NO_DEVICE, "no CUDA device is available");
    }
}

} // namespace

// Default output weighting of the training loss: log-scales, quaternion, logit opacity, DC colour.
static const float kDefaultLossWeights[kWarmOutputs] = {1, 1, 1, 0.5f, 0.5f, 0.5f, 0.5f, 0.25f, 1, 1, 1};

struct u3dg_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevBuf<float> params, m, v, grad;
    int step = 0;
    size_t cap = 0; // rows the activation scratch holds
    DevBuf<float> x, h1, h2, h3, y, t, dy, dh, dh2, w11, lossDev;
    DevBuf<double> partial;

    u3dg_mlp()
    {
        U3DG_CUDA(cudaGetDevice(&device));
        U3DG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        params.reserve(kWarmParams, true);
        m.reserve(kWarmParams, true);
        v.reserve(kWarmParams, true);
        grad.reserve(kWarmParams, true);
        w11.reserve(kWarmOutputs, true);
        lossDev.reserve(1, true);
        partial.reserve(size_t(mseBlocks()), true);
        U3DG_CUDA(cudaMemsetAsync(m.p, 0, kWarmParams * sizeof(float), stream));
        U3DG_CUDA(cudaMemsetAsync(v.p, 0, kWarmParams * sizeof(float), stream));
    }
    ~u3dg_mlp()
    {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
    void sync() { U3DG_CUDA(cudaStreamSynchronize(stream)); }
    void scratch(size_t n)
    {
        if (n <= cap)
            return;
        cap = std::max(n, cap + cap / 2);
        x.reserve(cap * kWarmInputs, true);
        h1.reserve(cap * kWarmHidden, true);
        h2.reserve(cap * kWarmHidden, true);
        h3.reserve(cap * kWarmHidden, true);
        y.reserve(cap * kWarmOutputs, true);
        t.reserve(cap * kWarmOutputs, true);
        dy.reserve(cap * kWarmOutputs, true);
        dh.reserve(cap * kWarmHidden, true);
        dh2.reserve(cap * kWarmHidden, true);
    }
    const float *W(int l) const { return params.p + offsets().w[l]; }
    const float *B(int l) const { return params.p + offsets().b[l]; }
    float *act(int l) // input activation of layer l (0 = features)
    {
        return l == 0 ? x.p : (l == 1 ? h1.p : (l == 2 ? h2.p : h3.p));
    }
    // Forward of rows already in x: activations h1..h3 and outputs y.
    void forward(int n)
    {
        for (int l = 0; l < kWarmLayers; ++l) {
            const int in = kWarmIn[l], out = kWarmOut[l];
            float *dst = (l == kWarmLayers - 1) ? y.p : act(l + 1);
            launchGemm(act(l), in, 1, W(l), 1, in, dst, out, n, out, in, B(l), l < kWarmLayers - 1, stream);
        }
    }
    // Gradient of the weighted MSE against t (rows in x / t): loss into lossDev, gradients into grad.
    void lossGrad(int n)
    {
        forward(n);
        launchMse(y.p, t.p, w11.p, n, dy.p, partial.p, lossDev.p, stream);
        float *dOut = dy.p;
        for (int l = kWarmLayers - 1; l >= 0; --l) {
            const int in = kWarmIn[l], out = kWarmOut[l];
            const LayerOffsets &o = offsets();
            // dW = dOut^T In (out x in), db = column sums of dOut.
            launchGemm(dOut, 1, out, act(l), in, 1, grad.p + o.w[l], in, out, in, n, nullptr, false, stream);
            launchColumnSum(dOut, n, out, grad.p + o.b[l], stream);
            if (l > 0) {
                float *dIn = (dOut == dh.p) ? dh2.p : dh.p;
                launchGemm(dOut, out, 1, W(l), in, 1, dIn, in, n, in, out, nullptr, false, stream);
                launchReluBackward(dIn, act(l), size_t(n) * in, stream);
                dOut = dIn;
            }
        }
    }
    void adam(float lr)
    {
        ++step;
        const float bc1 = 1.0f - std::pow(0.9f, float(step));
        const float bc2 = 1.0f - std::pow(0.999f, float(step));
        launchAdamFlat(params.p, grad.p, m.p, v.p, kWarmParams, lr / bc1, 1.0f / std::sqrt(bc2), 1e-8f, stream);
    }
};

namespace {

// He-uniform weights, zero biases except the output layer's, which starts at the plain initialisation
// (zero residuals, identity quaternion, opacity logit(0.1)), so an untrained network is the plain init.
std::vector<float> initialParams(unsigned seed)
{
    std::vector<float> p(kWarmParams, 0.0f);
    std::mt19937 rng(seed);
    const LayerOffsets &o = offsets();
    for (int l = 0; l < kWarmLayers; ++l) {
        const float a = std::sqrt(6.0f / float(kWarmIn[l])) * (l == kWarmLayers - 1 ? 0.01f : 1.0f);
        std::uniform_real_distribution<float> u(-a, a);
        for (size_t k = 0; k < size_t(kWarmOut[l]) * kWarmIn[l]; ++k)
            p[o.w[l] + k] = u(rng);
    }
    float *b3 = p.data() + o.b[kWarmLayers - 1];
    b3[3] = 1.0f;
    b3[7] = std::log(0.1f / (1.0f - 0.1f));
    return p;
}

template <class F>
int guardedW(F &&f)
{
    return guardedCall(std::forward<F>(f));
}

u3dg_mlp &mlpOf(u3dg_mlp *m)
{
    if (!m)
        throw StatusError(U3DG_ERR_INVALID_ARG, "network is NULL");
    U3DG_CUDA(cudaSetDevice(m->device));
    return *m;
}

// Device copies of the views for feature extraction.
struct DeviceViews {
    DevBuf<uint8_t> pixels;
    DevBuf<uint8_t> refs;
    int count = 0;
    void upload(const u3dg_image *images, int n, cudaStream_t s)
    {
        count = n;
        size_t total = 0;
        for (int k = 0; k < n; ++k) {
            checkCamera(images[k].camera);
            if (!images[k].rgb)
                throw StatusError(U3DG_ERR_INVALID_ARG, "image without pixels");
            total += size_t(images[k].camera.width) * images[k].camera.height * 3;
        }
        pixels.reserve(std::max<size_t>(total, 1), true);
        std::vector<uint8_t> refsHost(warmViewRefBytes() * size_t(std::max(n, 1)));
        size_t off = 0;
        for (int k = 0; k < n; ++k) {
            const size_t sz = size_t(images[k].camera.width) * images[k].camera.height * 3;
            U3DG_CUDA(cudaMemcpyAsync(pixels.p + off, images[k].rgb, sz, cudaMemcpyHostToDevice, s));
            fillWarmViewRef(refsHost.data() + warmViewRefBytes() * size_t(k), images[k].camera, pixels.p + off);
            off += sz;
        }
        refs.reserve(refsHost.size(), true);
        U3DG_CUDA(cudaMemcpyAsync(refs.p, refsHost.data(), refsHost.size(), cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaStreamSynchronize(s)); // refsHost is a local
    }
};

// Features of n points on the device (xyz, rgb device arrays; base sigma per point).
void computeFeatures(const float *xyzDev, const float *rgbDev, int n, const float *baseSigmaDev,
                     const DeviceViews &views, float *featDev, cudaStream_t s)
{
    DevBuf<int> nbr;
    DevBuf<float> nd2;
    nbr.reserve(size_t(std::max(n, 1)) * kWarmNeighbours, true);
    nd2.reserve(size_t(std::max(n, 1)) * kWarmNeighbours, true);
    launchKnn(xyzDev, n, xyzDev, n, kWarmNeighbours, 1, nbr.p, nd2.p, s);
    launchWarmFeatures(xyzDev, rgbDev, n, nbr.p, nd2.p, baseSigmaDev, views.refs.p, views.count, featDev, s);
    U3DG_CUDA(cudaGetLastError());
    U3DG_CUDA(cudaStreamSynchronize(s));
}

// The plain initialisation and the per-point sigma it implies (exp of its log-scale).
void plainInit(const float *xyz, const float *rgb, size_t n, HostModel &base, std::vector<float> &sigma)
{
    base.resize(n);
    u3dg_model v{base.means.data(), base.scales.data(), base.quats.data(), base.opac.data(), base.colors.data(), n};
    initGaussiansFromPointsDevice(xyz, rgb, n, v);
    sigma.resize(n);
    for (size_t i = 0; i < n; ++i)
        sigma[i] = std::exp(base.scales[3 * i]);
}

} // namespace

extern "C" {

int u3dg_mlp_param_count(void) { return kWarmParams; }

int u3dg_mlp_create(const float *params, unsigned int seed, u3dg_mlp **out)
{
    return guardedW([&] {
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        *out = nullptr;
        requireGpu();
        auto m = std::make_unique<u3dg_mlp>();
        std::vector<float> p = params ? std::vector<float>(params, params + kWarmParams) : initialParams(seed);
        U3DG_CUDA(cudaMemcpyAsync(m->params.p, p.data(), kWarmParams * sizeof(float), cudaMemcpyHostToDevice,
                                  m->stream));
        U3DG_CUDA(cudaMemcpyAsync(m->w11.p, kDefaultLossWeights, sizeof(kDefaultLossWeights), cudaMemcpyHostToDevice,
                                  m->stream));
        m->sync();
        *out = m.release();
    });
}

int u3dg_mlp_params(u3dg_mlp *mlp, float *out)
{
    return guardedW([&] {
        u3dg_mlp &m = mlpOf(mlp);
        if (!out)
            throw StatusError(U3DG_ERR_INVALID_ARG, "out is NULL");
        U3DG_CUDA(cudaMemcpyAsync(out, m.params.p, kWarmParams * sizeof(float), cudaMemcpyDeviceToHost, m.stream));
        m.sync();
    });
}

int u3dg_mlp_forward(u3dg_mlp *mlp, const float *x, size_t n, float *y)
{
    return guardedW([&] {
        u3dg_mlp &m = mlpOf(mlp);
        if (n && (!x || !y))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (n > size_t(INT_MAX / kWarmInputs))
            throw StatusError(U3DG_ERR_CAPACITY, "too many rows");
        if (!n)
            return;
        m.scratch(n);
        U3DG_CUDA(cudaMemcpyAsync(m.x.p, x, n * kWarmInputs * sizeof(float), cudaMemcpyHostToDevice, m.stream));
        m.forward(int(n));
        U3DG_CUDA(cudaGetLastError());
        U3DG_CUDA(cudaMemcpyAsync(y, m.y.p, n * kWarmOutputs * sizeof(float), cudaMemcpyDeviceToHost, m.stream));
        m.sync();
    });
}

int u3dg_mlp_loss_grad(u3dg_mlp *mlp, const float *x, const float *t, const float *weights, size_t n, float *loss,
                       float *grad)
{
    return guardedW([&] {
        u3dg_mlp &m = mlpOf(mlp);
        if (!x || !t || !n)
            throw StatusError(U3DG_ERR_INVALID_ARG, "x, t must be non-empty");
        if (n > size_t(INT_MAX / kWarmInputs))
            throw StatusError(U3DG_ERR_CAPACITY, "too many rows");
        m.scratch(n);
        U3DG_CUDA(cudaMemcpyAsync(m.x.p, x, n * kWarmInputs * sizeof(float), cudaMemcpyHostToDevice, m.stream));
        U3DG_CUDA(cudaMemcpyAsync(m.t.p, t, n * kWarmOutputs * sizeof(float), cudaMemcpyHostToDevice, m.stream));
        U3DG_CUDA(cudaMemcpyAsync(m.w11.p, weights ? weights : kDefaultLossWeights, kWarmOutputs * sizeof(float),
                                  cudaMemcpyHostToDevice, m.stream));
        m.lossGrad(int(n));
        U3DG_CUDA(cudaGetLastError());
        if (loss)
            U3DG_CUDA(cudaMemcpyAsync(loss, m.lossDev.p, sizeof(float), cudaMemcpyDeviceToHost, m.stream));
        if (grad)
            U3DG_CUDA(cudaMemcpyAsync(grad, m.grad.p, kWarmParams * sizeof(float), cudaMemcpyDeviceToHost, m.stream));
        m.sync();
    });
}

int u3dg_mlp_train(u3dg_mlp *mlp, const float *x, const float *t, const float *weights, size_t n, int epochs,
                   int batch, float lr, unsigned int seed, float *epoch_loss)
{
    return guardedW([&] {
        u3dg_mlp &m = mlpOf(mlp);
        if (!x || !t || !n || epochs < 0 || batch <= 0 || !(lr > 0.0f))
            throw StatusError(U3DG_ERR_INVALID_ARG, "invalid training arguments");
        if (n > size_t(INT_MAX / kWarmInputs))
            throw StatusError(U3DG_ERR_CAPACITY, "too many rows");
        cudaStream_t s = m.stream;
        DevBuf<float> X, T;
        X.reserve(n * kWarmInputs, true);
        T.reserve(n * kWarmOutputs, true);
        U3DG_CUDA(cudaMemcpyAsync(X.p, x, n * kWarmInputs * sizeof(float), cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(T.p, t, n * kWarmOutputs * sizeof(float), cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(m.w11.p, weights ? weights : kDefaultLossWeights, kWarmOutputs * sizeof(float),
                                  cudaMemcpyHostToDevice, s));
        const int B = int(std::min<size_t>(size_t(batch), n));
        m.scratch(size_t(B));
        DevBuf<int> rows;
        rows.reserve(n, true);
        DevBuf<float> batchLoss;
        const size_t batches = n / size_t(B); // whole batches only
        batchLoss.reserve(std::max<size_t>(batches, 1), true);
        std::vector<int> perm(n);
        std::mt19937 rng(seed);
        for (int e = 0; e < epochs; ++e) {
            for (size_t k = 0; k < n; ++k)
                perm[k] = int(k);
            std::shuffle(perm.begin(), perm.end(), rng);
            U3DG_CUDA(cudaMemcpyAsync(rows.p, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
            for (size_t b = 0; b < batches; ++b) {
                launchGatherRows(X.p, kWarmInputs, rows.p + b * size_t(B), B, m.x.p, s);
                launchGatherRows(T.p, kWarmOutputs, rows.p + b * size_t(B), B, m.t.p, s);
                m.lossGrad(B);
                U3DG_CUDA(cudaMemcpyAsync(batchLoss.p + b, m.lossDev.p, sizeof(float), cudaMemcpyDeviceToDevice, s));
                m.adam(lr);
            }
            U3DG_CUDA(cudaGetLastError());
            std::vector<float> bl(std::max<size_t>(batches, 1));
            U3DG_CUDA(cudaMemcpyAsync(bl.data(), batchLoss.p, bl.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
            m.sync(); // also keeps perm valid for its upload
            double sum = 0;
            for (size_t b = 0; b < batches; ++b)
                sum += bl[b];
            if (epoch_loss)
                epoch_loss[e] = float(sum / double(std::max<size_t>(batches, 1)));
        }
    });
}

void u3dg_mlp_destroy(u3dg_mlp *mlp)
{
    if (!mlp)
        return;
    cudaSetDevice(mlp->device);
    delete mlp;
}

int u3dg_knn(const float *queries, size_t nq, const float *points, size_t np, int k, int exclude_self, int *idx,
             float *dist2)
{
    return guardedW([&] {
        if (!(k == 1 || k == 3 || k == 16))
            throw StatusError(U3DG_ERR_INVALID_ARG, "k must be 1, 3 or 16");
        if ((nq && (!queries || !idx || !dist2)) || (np && !points))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (nq > size_t(INT_MAX / 16) || np > size_t(INT_MAX / 3))
            throw StatusError(U3DG_ERR_CAPACITY, "too many points");
        requireGpu();
        cudaStream_t s;
        U3DG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        DevBuf<float> q, p, d;
        DevBuf<int> id;
        q.reserve(std::max<size_t>(nq, 1) * 3, true);
        p.reserve(std::max<size_t>(np, 1) * 3, true);
        d.reserve(std::max<size_t>(nq, 1) * size_t(k), true);
        id.reserve(std::max<size_t>(nq, 1) * size_t(k), true);
        if (nq)
            U3DG_CUDA(cudaMemcpyAsync(q.p, queries, nq * 12, cudaMemcpyHostToDevice, s));
        if (np)
            U3DG_CUDA(cudaMemcpyAsync(p.p, points, np * 12, cudaMemcpyHostToDevice, s));
        launchKnn(q.p, int(nq), p.p, int(np), k, exclude_self, id.p, d.p, s);
        U3DG_CUDA(cudaGetLastError());
        if (nq) {
            U3DG_CUDA(cudaMemcpyAsync(idx, id.p, nq * size_t(k) * sizeof(int), cudaMemcpyDeviceToHost, s));
            U3DG_CUDA(cudaMemcpyAsync(dist2, d.p, nq * size_t(k) * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        U3DG_CUDA(cudaStreamSynchronize(s));
        cudaStreamDestroy(s);
    });
}

int u3dg_warmstart_features(const float *xyz, const float *rgb, size_t n, const u3dg_image *images, int count,
                            float *features)
{
    return guardedW([&] {
        if (n && (!xyz || !features))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (count < 0 || (count && !images))
            throw StatusError(U3DG_ERR_INVALID_ARG, "invalid images");
        if (n > size_t(INT_MAX / kWarmInputs))
            throw StatusError(U3DG_ERR_CAPACITY, "too many points");
        requireGpu();
        if (!n)
            return;
        HostModel base;
        std::vector<float> sigma;
        plainInit(xyz, rgb, n, base, sigma);
        cudaStream_t s;
        U3DG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        DevBuf<float> dx, dc, ds, f;
        dx.reserve(n * 3, true);
        dc.reserve(n * 3, true);
        ds.reserve(n, true);
        f.reserve(n * kWarmInputs, true);
        U3DG_CUDA(cudaMemcpyAsync(dx.p, xyz, n * 12, cudaMemcpyHostToDevice, s));
        if (rgb)
            U3DG_CUDA(cudaMemcpyAsync(dc.p, rgb, n * 12, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(ds.p, sigma.data(), n * 4, cudaMemcpyHostToDevice, s));
        DeviceViews views;
        views.upload(images, count, s);
        computeFeatures(dx.p, rgb ? dc.p : nullptr, int(n), ds.p, views, f.p, s);
        U3DG_CUDA(cudaMemcpyAsync(features, f.p, n * kWarmInputs * sizeof(float), cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaStreamSynchronize(s));
        cudaStreamDestroy(s);
    });
}

int u3dg_warmstart_init(u3dg_mlp *mlp, const float *xyz, const float *rgb, size_t n, const u3dg_image *images,
                        int count, u3dg_model *out)
{
    return guardedW([&] {
        if (n && (!xyz || !out || !out->means || !out->scales || !out->quats || !out->opacities || !out->colors))
            throw StatusError(U3DG_ERR_INVALID_ARG, "NULL argument");
        if (n > size_t(INT_MAX / kWarmInputs))
            throw StatusError(U3DG_ERR_CAPACITY, "too many points");
        HostModel base;
        std::vector<float> sigma;
        plainInit(xyz, rgb, n, base, sigma);
        auto copyOut = [&] {
            std::copy(base.means.begin(), base.means.end(), out->means);
            std::copy(base.scales.begin(), base.scales.end(), out->scales);
            std::copy(base.quats.begin(), base.quats.end(), out->quats);
            std::copy(base.opac.begin(), base.opac.end(), out->opacities);
            std::copy(base.colors.begin(), base.colors.end(), out->colors);
        };
        if (!mlp || !n) { // no network: the plain initialisation
            copyOut();
            return;
        }
        u3dg_mlp &m = mlpOf(mlp);
        cudaStream_t s = m.stream;
        DevBuf<float> dx, dc, ds, sc, qu, op, co;
        dx.reserve(n * 3, true);
        dc.reserve(n * 3, true);
        ds.reserve(n, true);
        U3DG_CUDA(cudaMemcpyAsync(dx.p, xyz, n * 12, cudaMemcpyHostToDevice, s));
        if (rgb)
            U3DG_CUDA(cudaMemcpyAsync(dc.p, rgb, n * 12, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(ds.p, sigma.data(), n * 4, cudaMemcpyHostToDevice, s));
        DeviceViews views;
        views.upload(images, count, s);
        m.scratch(n);
        computeFeatures(dx.p, rgb ? dc.p : nullptr, int(n), ds.p, views, m.x.p, s);
        m.forward(int(n));
        sc.reserve(n * 3, true);
        qu.reserve(n * 4, true);
        op.reserve(n, true);
        co.reserve(n * 3, true);
        U3DG_CUDA(cudaMemcpyAsync(sc.p, base.scales.data(), n * 12, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(qu.p, base.quats.data(), n * 16, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(op.p, base.opac.data(), n * 4, cudaMemcpyHostToDevice, s));
        U3DG_CUDA(cudaMemcpyAsync(co.p, base.colors.data(), n * 12, cudaMemcpyHostToDevice, s));
        launchWarmCombine(m.y.p, int(n), sc.p, qu.p, op.p, co.p, s);
        U3DG_CUDA(cudaGetLastError());
        U3DG_CUDA(cudaMemcpyAsync(base.scales.data(), sc.p, n * 12, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(base.quats.data(), qu.p, n * 16, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(base.opac.data(), op.p, n * 4, cudaMemcpyDeviceToHost, s));
        U3DG_CUDA(cudaMemcpyAsync(base.colors.data(), co.p, n * 12, cudaMemcpyDeviceToHost, s));
        m.sync();
        copyOut();
    });
}

} // extern "C"
