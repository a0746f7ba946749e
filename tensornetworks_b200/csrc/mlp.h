// mlp.h -- the learned Davidson correction: a per-element 3-layer MLP
// (4 -> 64 -> 64 -> 1, tanh) with BF16 weights for inference and an FP32
// master copy for training; hand-written forward, backward and Adam kernels.
#pragma once
#include <cuda_bf16.h>

#include "tn_internal.h"

namespace tnb {

constexpr int MLP_IN = 4;
constexpr int MLP_H = 64;
// parameter layout (FP32 master and BF16 copy share it)
constexpr int MLP_W1 = 0;                          // [MLP_IN][MLP_H]
constexpr int MLP_B1 = MLP_W1 + MLP_IN * MLP_H;    // [MLP_H]
constexpr int MLP_W2 = MLP_B1 + MLP_H;             // [MLP_H][MLP_H]
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;     // [MLP_H]
constexpr int MLP_W3 = MLP_B2 + MLP_H;             // [MLP_H]
constexpr int MLP_B3 = MLP_W3 + MLP_H;             // [1]
constexpr int MLP_NP = MLP_B3 + 1;                 // 4545
constexpr float MLP_FEAT_CLIP = 50.f;
constexpr float MLP_TARGET_CLIP = 50.f;

struct MlpModel {
    Ctx* ctx = nullptr;
    DevBuf w32, w16;     // FP32 master parameters, BF16 inference copy
    DevBuf m, v;         // Adam moments
    DevBuf part, loss;   // per-block gradient partials, per-block loss partials
    long long adam_t = 0;
};

// Training pairs: features (MLP_IN floats) and target per element.
struct DvRecorder {
    Ctx* ctx = nullptr;
    DevBuf feats, targets;
    long long size = 0, capacity = 0;
    DevBuf ubuf, scales;  // per-solve scratch: Ritz vector and feature scales of every step
};

// Output of the MLP at one element (weights in FP32 in shared memory).
__device__ __forceinline__ float mlp_eval(const float* __restrict__ w, const float (&f)[MLP_IN]) {
    float h1[MLP_H];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        float a = w[MLP_B1 + j];
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) a = fmaf(f[i], w[MLP_W1 + i * MLP_H + j], a);
        h1[j] = tanhf(a);
    }
    float y = w[MLP_B3];
#pragma unroll 1
    for (int k = 0; k < MLP_H; ++k) {
        float a = w[MLP_B2 + k];
#pragma unroll
        for (int j = 0; j < MLP_H; ++j) a = fmaf(h1[j], w[MLP_W2 + j * MLP_H + k], a);
        y = fmaf(tanhf(a), w[MLP_W3 + k], y);
    }
    return y;
}

__device__ __forceinline__ float mlp_clip(float x, float c) { return fminf(fmaxf(x, -c), c); }

int mlp_init(MlpModel& m, Ctx& c, unsigned long long seed);
int mlp_set_params(MlpModel& m, const float* host);   // FP32 master + BF16 copy, Adam reset
int mlp_get_params(const MlpModel& m, float* host);
// Y = MLP(F) with the BF16 weights (F: n x MLP_IN row-major floats, device).
int mlp_forward(const MlpModel& m, const float* F, long long n, float* Y, cudaStream_t st);
// Gradient of the mean squared error over n pairs with the FP32 weights (host
// output, MLP_NP floats), and the loss.
int mlp_gradient(MlpModel& m, const float* F, const float* T, long long n, float* grad_host, double* loss);
// Adam on minibatches of `batch` consecutive pairs of a seeded permutation.
int mlp_train(MlpModel& m, const float* F, const float* T, long long n, int steps, int batch, double lr,
              unsigned long long seed, double* final_loss);

int recorder_init(DvRecorder& r, Ctx& c, long long capacity);

}  // namespace tnb
