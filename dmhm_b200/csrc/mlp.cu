// Learned rank predictor: a three-layer perceptron (FP32) that reads the
// features of one randomized H*H compression (hh.cu, rank_features) and
// predicts the fraction of maxRank that the compression keeps, so that the
// compression draws only that many samples (plus the oversampling).
//
// No counterpart in the reference (its randomized product always draws
// SampleRank = maxRank + Oversample() samples, hmat_tools.hpp:1657-1746).
// Training and inference are these kernels: full-batch forward, mean squared
// error on the sigmoid output, backward by the chain rule, Adam.  Every
// reduction runs in a fixed order (no atomics), so training is deterministic.
//
// Parameter layout (one float array of kMlpParams):
//   W1 [kMlpHidden x kMlpFeatures] row-major, b1 [kMlpHidden],
//   W2 [kMlpHidden x kMlpHidden],            b2 [kMlpHidden],
//   W3 [kMlpHidden],                          b3 [1].
#include <cmath>
#include <vector>

#include "engine.h"
#include "mlp.h"

namespace hmb {

namespace {

constexpr int F = kMlpFeatures, Hd = kMlpHidden;
constexpr int OW1 = 0, OB1 = OW1 + Hd * F, OW2 = OB1 + Hd, OB2 = OW2 + Hd * Hd, OW3 = OB2 + Hd,
              OB3 = OW3 + Hd;
static_assert(OB3 + 1 == kMlpParams, "parameter layout");

// Z = X W^T + b (X: n x in, W: out x in), A = relu(Z) (or Z when !relu).
__global__ void dense_fwd_kernel(const float* __restrict__ X, const float* __restrict__ W,
                                 const float* __restrict__ b, float* __restrict__ Z,
                                 float* __restrict__ A, int n, int in, int out, int relu) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * out) return;
    const int i = (int)(e / out), j = (int)(e % out);
    float z = b[j];
    for (int k = 0; k < in; ++k) z = fmaf(X[(long long)i * in + k], W[j * in + k], z);
    Z[e] = z;
    A[e] = relu ? fmaxf(z, 0.0f) : z;
}

// y = sigmoid(z3); loss terms and dZ3 = d(mean (y - t)^2)/dz3.
__global__ void head_kernel(const float* __restrict__ z3, const float* __restrict__ t,
                            float* __restrict__ y, float* __restrict__ dz3,
                            float* __restrict__ sq, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float yi = 1.0f / (1.0f + expf(-z3[i]));
    y[i] = yi;
    if (t) {
        const float d = yi - t[i];
        sq[i] = d * d;
        dz3[i] = 2.0f * d * yi * (1.0f - yi) / (float)n;
    }
}

// dW[j][k] = sum_i dZ[i][j] A[i][k]; db[j] = sum_i dZ[i][j] (fixed order).
__global__ void dense_wgrad_kernel(const float* __restrict__ dZ, const float* __restrict__ Ain,
                                   float* __restrict__ dW, float* __restrict__ db, int n, int in,
                                   int out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= out * (in + 1)) return;
    const int j = e / (in + 1), k = e % (in + 1);
    float s = 0.0f;
    if (k < in)
        for (int i = 0; i < n; ++i) s = fmaf(dZ[(long long)i * out + j], Ain[(long long)i * in + k], s);
    else
        for (int i = 0; i < n; ++i) s += dZ[(long long)i * out + j];
    if (k < in) dW[j * in + k] = s;
    else db[j] = s;
}

// dZin[i][k] = (sum_j dZ[i][j] W[j][k]) * relu'(Zin[i][k]).
__global__ void dense_bgrad_kernel(const float* __restrict__ dZ, const float* __restrict__ W,
                                   const float* __restrict__ Zin, float* __restrict__ dZin, int n,
                                   int in, int out) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * in) return;
    const int i = (int)(e / in), k = (int)(e % in);
    float s = 0.0f;
    for (int j = 0; j < out; ++j) s = fmaf(dZ[(long long)i * out + j], W[j * in + k], s);
    dZin[e] = Zin[e] > 0.0f ? s : 0.0f;
}

// Sum of v[0..n) in a fixed order (one CTA).
__global__ void sum_kernel(const float* __restrict__ v, int n, float* __restrict__ out) {
    __shared__ float red[256];
    float s = 0.0f;
    for (int i = threadIdx.x; i < n; i += 256) s += v[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0] / (float)n;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, int np, float lr,
                            float b1c, float b2c) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= np) return;
    const float gi = g[e];
    const float mi = 0.9f * m[e] + 0.1f * gi;
    const float vi = 0.999f * v[e] + 0.001f * gi * gi;
    m[e] = mi;
    v[e] = vi;
    p[e] -= lr * (mi / b1c) / (sqrtf(vi / b2c) + 1e-8f);
}

unsigned blocks_for(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Activations of one batch.
struct MlpBatch {
    DeviceBuffer<float> x, t, z1, a1, z2, a2, z3, y, dz3, sq, d2, d1, loss;
    int n = 0;
};

void RankModel::init(uint64_t seed) {
    // He-style uniform initialisation from a 64-bit LCG (host), bias 0,
    // output bias log(0.5 / 0.5) = 0.
    std::vector<float> h(kMlpParams, 0.0f);
    uint64_t s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    auto uni = [&]() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return (float)((s >> 11) * (1.0 / 9007199254740992.0)) * 2.0f - 1.0f;
    };
    const float a1 = std::sqrt(6.0f / F), a2 = std::sqrt(6.0f / Hd), a3 = std::sqrt(3.0f / Hd);
    for (int i = 0; i < Hd * F; ++i) h[OW1 + i] = a1 * uni();
    for (int i = 0; i < Hd * Hd; ++i) h[OW2 + i] = a2 * uni();
    for (int i = 0; i < Hd; ++i) h[OW3 + i] = a3 * uni();
    set_params(h.data());
    std::vector<float> z(kMlpParams, 0.0f);
    m.upload(z, ctx->stream);
    v.upload(z, ctx->stream);
    step = 0;
}

void RankModel::set_params(const float* h) {
    std::vector<float> p(h, h + kMlpParams);
    params.upload(p, ctx->stream);
    if (!grad.get()) grad.allocate(kMlpParams, ctx->stream);
}

void RankModel::get_params(float* h) const {
    HMB_CUDA(cudaMemcpyAsync(h, params.get(), kMlpParams * sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream));
    HMB_CUDA(cudaStreamSynchronize(ctx->stream));
}

namespace {

void forward(Context& ctx, const RankModel& M, MlpBatch& B, bool keep_targets) {
    cudaStream_t st = ctx.stream;
    const float* P = M.params.get();
    const int n = B.n;
    LaunchScope ls(ctx, "mlp_forward");
    dense_fwd_kernel<<<blocks_for((long long)n * Hd), 256, 0, st>>>(B.x.get(), P + OW1, P + OB1,
                                                                   B.z1.get(), B.a1.get(), n, F, Hd, 1);
    dense_fwd_kernel<<<blocks_for((long long)n * Hd), 256, 0, st>>>(B.a1.get(), P + OW2, P + OB2,
                                                                   B.z2.get(), B.a2.get(), n, Hd, Hd, 1);
    dense_fwd_kernel<<<blocks_for(n), 256, 0, st>>>(B.a2.get(), P + OW3, P + OB3, B.z3.get(),
                                                    B.z3.get(), n, Hd, 1, 0);
    head_kernel<<<blocks_for(n), 256, 0, st>>>(B.z3.get(), keep_targets ? B.t.get() : nullptr,
                                               B.y.get(), B.dz3.get(), B.sq.get(), n);
    HMB_CHECK_LAUNCH();
}

void backward(Context& ctx, RankModel& M, MlpBatch& B) {
    cudaStream_t st = ctx.stream;
    const float* P = M.params.get();
    float* G = M.grad.get();
    const int n = B.n;
    LaunchScope ls(ctx, "mlp_backward");
    dense_wgrad_kernel<<<blocks_for(1 * (Hd + 1)), 256, 0, st>>>(B.dz3.get(), B.a2.get(), G + OW3,
                                                                 G + OB3, n, Hd, 1);
    dense_bgrad_kernel<<<blocks_for((long long)n * Hd), 256, 0, st>>>(B.dz3.get(), P + OW3,
                                                                     B.z2.get(), B.d2.get(), n, Hd, 1);
    dense_wgrad_kernel<<<blocks_for(Hd * (Hd + 1)), 256, 0, st>>>(B.d2.get(), B.a1.get(), G + OW2,
                                                                  G + OB2, n, Hd, Hd);
    dense_bgrad_kernel<<<blocks_for((long long)n * Hd), 256, 0, st>>>(B.d2.get(), P + OW2,
                                                                     B.z1.get(), B.d1.get(), n, Hd, Hd);
    dense_wgrad_kernel<<<blocks_for(Hd * (F + 1)), 256, 0, st>>>(B.d1.get(), B.x.get(), G + OW1,
                                                                 G + OB1, n, F, Hd);
    HMB_CHECK_LAUNCH();
}

void make_batch(Context& ctx, MlpBatch& B, const float* x, const float* t, int n) {
    cudaStream_t st = ctx.stream;
    B.n = n;
    std::vector<float> hx(x, x + (long long)n * F);
    B.x.upload(hx, st);
    if (t) {
        std::vector<float> ht(t, t + n);
        B.t.upload(ht, st);
    }
    B.z1.allocate((size_t)n * Hd, st);
    B.a1.allocate((size_t)n * Hd, st);
    B.z2.allocate((size_t)n * Hd, st);
    B.a2.allocate((size_t)n * Hd, st);
    B.z3.allocate(n, st);
    B.y.allocate(n, st);
    B.dz3.allocate(n, st);
    B.sq.allocate(n, st);
    B.d2.allocate((size_t)n * Hd, st);
    B.d1.allocate((size_t)n * Hd, st);
    B.loss.allocate(1, st);
}

}  // namespace

float RankModel::loss_and_grad(const float* x, const float* t, int n, float* grad_out) {
    HMB_REQUIRE(n > 0, HM_ERR_ARGUMENT, "empty batch");
    MlpBatch B;
    make_batch(*ctx, B, x, t, n);
    forward(*ctx, *this, B, true);
    backward(*ctx, *this, B);
    sum_kernel<<<1, 256, 0, ctx->stream>>>(B.sq.get(), n, B.loss.get());
    HMB_CHECK_LAUNCH();
    float loss = 0.0f;
    HMB_CUDA(cudaMemcpyAsync(&loss, B.loss.get(), sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (grad_out)
        HMB_CUDA(cudaMemcpyAsync(grad_out, grad.get(), kMlpParams * sizeof(float),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    HMB_CUDA(cudaStreamSynchronize(ctx->stream));
    return loss;
}

float RankModel::train(const float* x, const float* t, int n, int epochs, float lr) {
    HMB_REQUIRE(n > 0 && epochs >= 0 && lr > 0.0f, HM_ERR_ARGUMENT, "bad training arguments");
    MlpBatch B;
    make_batch(*ctx, B, x, t, n);
    cudaStream_t st = ctx->stream;
    for (int e = 0; e < epochs; ++e) {
        forward(*ctx, *this, B, true);
        backward(*ctx, *this, B);
        ++step;
        const float b1c = 1.0f - std::pow(0.9f, (float)step);
        const float b2c = 1.0f - std::pow(0.999f, (float)step);
        LaunchScope ls(*ctx, "mlp_adam");
        adam_kernel<<<blocks_for(kMlpParams), 256, 0, st>>>(params.get(), grad.get(), m.get(), v.get(),
                                                            kMlpParams, lr, b1c, b2c);
        HMB_CHECK_LAUNCH();
    }
    forward(*ctx, *this, B, true);
    sum_kernel<<<1, 256, 0, st>>>(B.sq.get(), n, B.loss.get());
    HMB_CHECK_LAUNCH();
    float loss = 0.0f;
    HMB_CUDA(cudaMemcpyAsync(&loss, B.loss.get(), sizeof(float), cudaMemcpyDeviceToHost, st));
    HMB_CUDA(cudaStreamSynchronize(st));
    return loss;
}

void RankModel::predict(const float* x, int n, float* out) {
    if (n <= 0) return;
    MlpBatch B;
    make_batch(*ctx, B, x, nullptr, n);
    forward(*ctx, *this, B, false);
    HMB_CUDA(cudaMemcpyAsync(out, B.y.get(), n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    HMB_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace hmb
