// mlp.cu -- the learned cost model: a small MLP trained on the GPU by
// hand-written kernels, used to choose how (never what) each request is
// computed.
//
// Network: x (MELA_MLP_IN features) -> 32 ReLU -> 32 ReLU -> MELA_MLP_OUT
// outputs, the predicted log2 running time (microseconds) of each
// configuration of the request's op (dispatch.cu lists them: ten
// elimination configurations, six product configurations, three batch
// engines).  Parameters are one flat float array:
//   W1[IN][H1] b1[H1] W2[H1][H2] b2[H2] W3[H2][OUT] b3[OUT]
// Loss: mean squared error over the observed (sample, configuration) pairs.
//
// Kernels: forward (one thread per sample), backward (one thread per sample,
// per-block gradient sums in shared memory, then one global atomic per
// parameter and block), Adam update (one thread per parameter).
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>

#include "mela_common.cuh"
#include "mela_internal.h"
#include "mela_host.h"

namespace mela {

constexpr int kIn = MELA_MLP_IN, kH1 = MELA_MLP_H1, kH2 = MELA_MLP_H2, kOut = MELA_MLP_OUT;
constexpr int oW1 = 0, ob1 = oW1 + kIn * kH1, oW2 = ob1 + kH1, ob2 = oW2 + kH1 * kH2,
              oW3 = ob2 + kH2, ob3 = oW3 + kH2 * kOut, kParams = ob3 + kOut;
static_assert(kParams == MELA_MLP_PARAMS, "parameter count");

__device__ __forceinline__ void mlp_fwd(const float *P, const float *x, float *h1, float *h2, float *y)
{
#pragma unroll 4
    for (int j = 0; j < kH1; ++j) {
        float a = P[ob1 + j];
#pragma unroll
        for (int i = 0; i < kIn; ++i) a += x[i] * P[oW1 + i * kH1 + j];
        h1[j] = a > 0.f ? a : 0.f;
    }
#pragma unroll 4
    for (int k = 0; k < kH2; ++k) {
        float a = P[ob2 + k];
        for (int j = 0; j < kH1; ++j) a += h1[j] * P[oW2 + j * kH2 + k];
        h2[k] = a > 0.f ? a : 0.f;
    }
#pragma unroll
    for (int o = 0; o < kOut; ++o) {
        float a = P[ob3 + o];
        for (int k = 0; k < kH2; ++k) a += h2[k] * P[oW3 + k * kOut + o];
        y[o] = a;
    }
}

__global__ void __launch_bounds__(256) mlp_forward_kernel(const float *__restrict__ params,
                                                          const float *__restrict__ X, long long N,
                                                          float *__restrict__ Y)
{
    __shared__ float P[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= N) return;
    float x[kIn], h1[kH1], h2[kH2], y[kOut];
#pragma unroll
    for (int i = 0; i < kIn; ++i) x[i] = X[s * kIn + i];
    mlp_fwd(P, x, h1, h2, y);
#pragma unroll
    for (int o = 0; o < kOut; ++o) Y[s * kOut + o] = y[o];
}

// grad += d(loss)/d(params); loss_sum += sum of masked squared errors.
// `inv_count` = 1 / (number of observed outputs).
__global__ void __launch_bounds__(256) mlp_backward_kernel(const float *__restrict__ params,
                                                           const float *__restrict__ X,
                                                           const float *__restrict__ T,
                                                           const float *__restrict__ Mk, long long N,
                                                           float inv_count, float *__restrict__ grad,
                                                           float *loss_sum)
{
    __shared__ float P[kParams];
    __shared__ float G[kParams];
    __shared__ float Ls;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        P[i] = params[i];
        G[i] = 0.f;
    }
    if (threadIdx.x == 0) Ls = 0.f;
    __syncthreads();
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s < N) {
        float x[kIn], h1[kH1], h2[kH2], y[kOut], dy[kOut];
#pragma unroll
        for (int i = 0; i < kIn; ++i) x[i] = X[s * kIn + i];
        mlp_fwd(P, x, h1, h2, y);
        float l = 0.f;
#pragma unroll
        for (int o = 0; o < kOut; ++o) {
            const float mk = Mk[s * kOut + o];
            const float e = mk != 0.f ? (y[o] - T[s * kOut + o]) : 0.f;
            l += e * e;
            dy[o] = 2.f * e * inv_count;
        }
        atomicAdd(&Ls, l);
        // layer 3
        float dh2[kH2];
        for (int k = 0; k < kH2; ++k) {
            float a = 0.f;
#pragma unroll
            for (int o = 0; o < kOut; ++o) {
                atomicAdd(&G[oW3 + k * kOut + o], h2[k] * dy[o]);
                a += dy[o] * P[oW3 + k * kOut + o];
            }
            dh2[k] = h2[k] > 0.f ? a : 0.f;
        }
#pragma unroll
        for (int o = 0; o < kOut; ++o) atomicAdd(&G[ob3 + o], dy[o]);
        // layer 2
        float dh1[kH1];
        for (int j = 0; j < kH1; ++j) {
            float a = 0.f;
            for (int k = 0; k < kH2; ++k) {
                if (dh2[k] != 0.f) atomicAdd(&G[oW2 + j * kH2 + k], h1[j] * dh2[k]);
                a += dh2[k] * P[oW2 + j * kH2 + k];
            }
            dh1[j] = h1[j] > 0.f ? a : 0.f;
        }
        for (int k = 0; k < kH2; ++k)
            if (dh2[k] != 0.f) atomicAdd(&G[ob2 + k], dh2[k]);
        // layer 1
        for (int j = 0; j < kH1; ++j) {
            if (dh1[j] == 0.f) continue;
#pragma unroll
            for (int i = 0; i < kIn; ++i) atomicAdd(&G[oW1 + i * kH1 + j], x[i] * dh1[j]);
            atomicAdd(&G[ob1 + j], dh1[j]);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
        if (G[i] != 0.f) atomicAdd(&grad[i], G[i]);
    if (threadIdx.x == 0 && loss_sum) atomicAdd(loss_sum, Ls);
}

__global__ void adam_kernel(float *__restrict__ params, const float *__restrict__ grad,
                            float *__restrict__ m1, float *__restrict__ m2, int n, float lr, float b1,
                            float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i];
    const float a = b1 * m1[i] + (1.f - b1) * g;
    const float b = b2 * m2[i] + (1.f - b2) * g * g;
    m1[i] = a;
    m2[i] = b;
    params[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// ---------------------------------------------------------------- host-side model
// The dispatch copy of the trained parameters (host memory): single calls
// evaluate the tiny network on the host to pick a variant before launching.
// The model trained with the library (costmodel.json, compiled in by the
// build) is installed when the library loads; mela_costmodel_load replaces
// or removes it.
#include "costmodel_weights.inc"
// Installed weights: an immutable snapshot swapped under the mutex and read
// through a shared pointer, so an evaluation neither copies the weights nor
// holds the lock while it runs.
struct CostModelWeights {
    float p[kParams];
};
static std::mutex g_cm_mu;
static std::shared_ptr<const CostModelWeights> g_cm;
static std::atomic<unsigned> g_cm_generation{1};  // bumped on every install or removal

unsigned costmodel_generation() { return g_cm_generation.load(std::memory_order_acquire); }

static std::shared_ptr<const CostModelWeights> current_model()
{
    std::lock_guard<std::mutex> g(g_cm_mu);
    return g_cm;
}

#ifdef MELA_DEFAULT_MODEL
static_assert(sizeof kDefaultModel / sizeof kDefaultModel[0] == kParams, "compiled-in model size");
static const bool g_cm_default = [] {
    auto w = std::make_shared<CostModelWeights>();
    std::memcpy(w->p, kDefaultModel, sizeof w->p);
    g_cm = w;
    return true;
}();
#endif

// The network on the host, layer by layer along contiguous weight rows.
static void host_forward(const float *P, const float *x, float *y)
{
    float h1[kH1], h2[kH2], o[kOut];
    for (int j = 0; j < kH1; ++j) h1[j] = P[ob1 + j];
    for (int i = 0; i < kIn; ++i) {
        const float xi = x[i];
        const float *w = P + oW1 + i * kH1;
        for (int j = 0; j < kH1; ++j) h1[j] += xi * w[j];
    }
    for (int j = 0; j < kH1; ++j) h1[j] = h1[j] > 0.f ? h1[j] : 0.f;
    for (int k = 0; k < kH2; ++k) h2[k] = P[ob2 + k];
    for (int j = 0; j < kH1; ++j) {
        const float hj = h1[j];
        if (hj == 0.f) continue;
        const float *w = P + oW2 + j * kH2;
        for (int k = 0; k < kH2; ++k) h2[k] += hj * w[k];
    }
    for (int k = 0; k < kH2; ++k) h2[k] = h2[k] > 0.f ? h2[k] : 0.f;
    for (int q = 0; q < kOut; ++q) o[q] = P[ob3 + q];
    for (int k = 0; k < kH2; ++k) {
        const float hk = h2[k];
        if (hk == 0.f) continue;
        const float *w = P + oW3 + k * kOut;
        for (int q = 0; q < kOut; ++q) o[q] += hk * w[q];
    }
    for (int q = 0; q < kOut; ++q) y[q] = o[q];
}

void costmodel_features(int op, double m, double n, double p, double density, double batch_count,
                        double batch_log2_cells, float *x)
{
    auto lg = [](double v) { return (float)(std::log2(v > 1 ? v : 1) / 14.0); };
    x[0] = lg(m);
    x[1] = lg(n);
    x[2] = op == MELA_OP_MATMUL ? lg(p) : 0.f;
    const double d = density > 1e-6 ? density : 1e-6;
    x[3] = (float)(std::log10(d) / 3.0 + 1.0);
    x[4] = op == MELA_OP_RANK ? 1.f : 0.f;
    x[5] = op == MELA_OP_NULL ? 1.f : 0.f;
    x[6] = op == MELA_OP_MATMUL ? 1.f : 0.f;
    x[7] = op == MELA_OP_BATCH ? 1.f : 0.f;
    // batch mix: how many matrices share the launch, and how large they are
    x[8] = (float)(std::log2(batch_count > 1 ? batch_count : 1) / 16.0);
    x[9] = (float)(batch_log2_cells / 28.0);
}

bool costmodel_loaded() { return current_model() != nullptr; }

bool costmodel_predict(int op, double m, double n, double p, double density, double batch_count,
                       double batch_log2_cells, float *y_out)
{
    const std::shared_ptr<const CostModelWeights> w = current_model();
    if (!w) return false;
    float x[kIn], y[kOut];
    costmodel_features(op, m, n, p, density, batch_count, batch_log2_cells, x);
    host_forward(w->p, x, y);
    const int nc = config_count(op);
    for (int o = 0; o < nc; ++o) y_out[o] = y[o];
    return true;
}

// Predictions for one request at kProbe densities in one pass: the inputs
// differ only in the density feature, so the first layer is shared and the
// other two run with the probes side by side (the inner loops over the four
// probes vectorise).
bool costmodel_predict_densities(int op, double m, double n, double p, const double *dens, double batch_count,
                                 double batch_log2_cells, float (*y_out)[MELA_MLP_OUT])
{
    constexpr int NP = kCostProbes;
    const std::shared_ptr<const CostModelWeights> w = current_model();
    if (!w) return false;
    const float *P = w->p;
    float x[kIn];
    costmodel_features(op, m, n, p, 0.5, batch_count, batch_log2_cells, x);
    float base[kH1];
    for (int j = 0; j < kH1; ++j) base[j] = P[ob1 + j];
    for (int i = 0; i < kIn; ++i) {
        if (i == 3) continue;  // the density feature, added per probe below
        const float xi = x[i];
        const float *wr = P + oW1 + i * kH1;
        for (int j = 0; j < kH1; ++j) base[j] += xi * wr[j];
    }
    float xd[NP];
    for (int q = 0; q < NP; ++q) {
        const double d = dens[q] > 1e-6 ? dens[q] : 1e-6;
        xd[q] = (float)(std::log10(d) / 3.0 + 1.0);
    }
    float h1[kH1][NP], h2[kH2][NP], o[kOut][NP];
    for (int j = 0; j < kH1; ++j)
        for (int q = 0; q < NP; ++q) {
            const float a = base[j] + xd[q] * P[oW1 + 3 * kH1 + j];
            h1[j][q] = a > 0.f ? a : 0.f;
        }
    for (int k = 0; k < kH2; ++k)
        for (int q = 0; q < NP; ++q) h2[k][q] = P[ob2 + k];
    for (int j = 0; j < kH1; ++j) {
        const float *wr = P + oW2 + j * kH2;
        for (int k = 0; k < kH2; ++k)
            for (int q = 0; q < NP; ++q) h2[k][q] += h1[j][q] * wr[k];
    }
    for (int k = 0; k < kH2; ++k)
        for (int q = 0; q < NP; ++q) h2[k][q] = h2[k][q] > 0.f ? h2[k][q] : 0.f;
    for (int c = 0; c < kOut; ++c)
        for (int q = 0; q < NP; ++q) o[c][q] = P[ob3 + c];
    for (int k = 0; k < kH2; ++k) {
        const float *wr = P + oW3 + k * kOut;
        for (int c = 0; c < kOut; ++c)
            for (int q = 0; q < NP; ++q) o[c][q] += h2[k][q] * wr[c];
    }
    for (int q = 0; q < NP; ++q)
        for (int c = 0; c < kOut; ++c) y_out[q][c] = o[c][q];
    return true;
}

// -1 when no model is loaded (callers use their fixed rule)
int costmodel_choose(int op, double m, double n, double p, double density, double batch_count,
                     double batch_log2_cells)
{
    float y[kOut];
    const int nc = config_count(op);
    if (nc <= 0 || !costmodel_predict(op, m, n, p, density, batch_count, batch_log2_cells, y)) return -1;
    int best = 0;
    for (int o = 1; o < nc; ++o)
        if (y[o] < y[best]) best = o;
    return best;
}

}  // namespace mela

using namespace mela;

extern "C" mela_status mela_mlp_forward(const float *d_params, const float *d_X, int64_t N, float *d_Y,
                                        void *stream)
{
    if (N < 0 || (N > 0 && (!d_params || !d_X || !d_Y))) {
        set_error("mela_mlp_forward: bad arguments");
        return MELA_ERR_INVALID;
    }
    if (N == 0) return MELA_OK;
    mlp_forward_kernel<<<(unsigned)((N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_params, d_X, N, d_Y);
    MELA_LAUNCH_CHECK("mlp_forward_kernel");
    return MELA_OK;
}

extern "C" mela_status mela_mlp_gradient(const float *d_params, const float *d_X, const float *d_T,
                                         const float *d_mask, int64_t N, float inv_count,
                                         float *d_grad, float *d_loss_sum, void *stream)
{
    if (N < 0 || (N > 0 && (!d_params || !d_X || !d_T || !d_mask || !d_grad))) {
        set_error("mela_mlp_gradient: bad arguments");
        return MELA_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    MELA_CUDA_TRY(cudaMemsetAsync(d_grad, 0, sizeof(float) * kParams, s));
    if (d_loss_sum) MELA_CUDA_TRY(cudaMemsetAsync(d_loss_sum, 0, sizeof(float), s));
    if (N == 0) return MELA_OK;
    mlp_backward_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(d_params, d_X, d_T, d_mask, N,
                                                                     inv_count, d_grad, d_loss_sum);
    MELA_LAUNCH_CHECK("mlp_backward_kernel");
    return MELA_OK;
}

extern "C" mela_status mela_mlp_adam_step(float *d_params, const float *d_grad, float *d_m1,
                                          float *d_m2, int64_t step, float lr, void *stream)
{
    if (!d_params || !d_grad || !d_m1 || !d_m2 || step < 1) {
        set_error("mela_mlp_adam_step: bad arguments");
        return MELA_ERR_INVALID;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    adam_kernel<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_grad, d_m1, d_m2,
                                                                          kParams, lr, b1, b2, eps, c1, c2);
    MELA_LAUNCH_CHECK("adam_kernel");
    return MELA_OK;
}

extern "C" mela_status mela_costmodel_load(const float *h_params)
{
    std::shared_ptr<CostModelWeights> w;
    if (h_params) {
        w = std::make_shared<CostModelWeights>();
        std::memcpy(w->p, h_params, sizeof w->p);
    }
    std::lock_guard<std::mutex> g(g_cm_mu);
    g_cm = std::move(w);
    g_cm_generation.fetch_add(1, std::memory_order_acq_rel);
    return MELA_OK;
}

extern "C" int32_t mela_costmodel_choose(int32_t op, int64_t m, int64_t n, int64_t p, double density,
                                         int64_t batch_count, double batch_log2_cells)
{
    return costmodel_choose(op, (double)m, (double)n, (double)p, density, (double)batch_count,
                            batch_log2_cells);
}

extern "C" int32_t mela_costmodel_predict(int32_t op, int64_t m, int64_t n, int64_t p, double density,
                                          int64_t batch_count, double batch_log2_cells, float *y)
{
    const int nc = config_count(op);
    float out[kOut];
    if (nc <= 0 || !y ||
        !costmodel_predict(op, (double)m, (double)n, (double)p, density, (double)batch_count, batch_log2_cells, out))
        return -1;
    for (int i = 0; i < nc; ++i) y[i] = out[i];
    return nc;
}

extern "C" void mela_costmodel_features(int32_t op, int64_t m, int64_t n, int64_t p, double density,
                                        int64_t batch_count, double batch_log2_cells, float *x)
{
    costmodel_features(op, (double)m, (double)n, (double)p, density, (double)batch_count, batch_log2_cells, x);
}
