// Learned rank predictor (see mlp.cu).
#pragma once
#include <cstdint>

#include "engine.h"

namespace hmb {

constexpr int kMlpFeatures = 12;
constexpr int kMlpHidden = 64;
constexpr int kMlpParams =
    kMlpHidden * kMlpFeatures + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpHidden + 1;

struct RankModel {
    Context* ctx = nullptr;
    DeviceBuffer<float> params, grad, m, v;   // parameters, gradient, Adam moments
    int step = 0;

    void init(uint64_t seed);
    void set_params(const float* host);
    void get_params(float* host) const;
    // Mean squared error of sigmoid(f(x)) against t, and its gradient (into
    // `grad`, and into grad_out when given).
    float loss_and_grad(const float* x, const float* t, int n, float* grad_out);
    // `epochs` full-batch Adam steps; returns the final loss.
    float train(const float* x, const float* t, int n, int epochs, float lr);
    // sigmoid(f(x)) for n feature rows (host in, host out).
    void predict(const float* x, int n, float* out);
};

}  // namespace hmb
