// mlp.h -- the learned Davidson correction: a per-element 3-layer MLP
// (4 -> 64 -> 64 -> 1, tanh) with BF16 weights for inference (the hidden
// layer on the tensor cores) and an FP32 master copy for training;
// hand-written forward, backward and Adam kernels.
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

// ---- inference on the tensor cores ------------------------------------------
//
// A warp evaluates the network on tiles of 16 elements: the 4 -> 64 layer and
// both tanh layers on its lanes (tanh.approx.f32), the 64 x 64 hidden layer
// as 32 BF16 tensor-core products (mma.sync m16n8k16, FP32 accumulation: the
// 16 x 64 activations against W2), and the 64 -> 1 output by a reduction over
// the 4 lanes of each row.  ~1.1 GFLOP for a 131 072-element site vector is a
// few microseconds this way, where the per-element FP32 loop over weights in
// shared memory took ~200 us.  BF16 activations and the approximate tanh move
// the output by ~1e-3 of its scale, far inside what a preconditioner needs.
constexpr int MLP_W2T_LD = 36;  // 32-bit words per row of W2^T in shared memory (rows 4 banks apart)

struct MlpInferSmem {
    uint32_t w2t[MLP_H * MLP_W2T_LD];  // row n, word kk: (W2[2kk][n], W2[2kk + 1][n]) as a BF16 pair
    float w1[MLP_IN * MLP_H], b1[MLP_H], b2[MLP_H], w3[MLP_H], b3;
};

// All threads of the block: the BF16 parameters into shared memory.
__device__ __forceinline__ void mlp_stage(const __nv_bfloat16* __restrict__ w16, MlpInferSmem& s) {
    for (int e = threadIdx.x; e < MLP_H * (MLP_H / 2); e += blockDim.x) {
        const int nn = e / (MLP_H / 2), kk = e % (MLP_H / 2);
        __nv_bfloat162 v;
        v.x = w16[MLP_W2 + (2 * kk) * MLP_H + nn];
        v.y = w16[MLP_W2 + (2 * kk + 1) * MLP_H + nn];
        s.w2t[nn * MLP_W2T_LD + kk] = *reinterpret_cast<const uint32_t*>(&v);
    }
    for (int e = threadIdx.x; e < MLP_IN * MLP_H; e += blockDim.x) s.w1[e] = __bfloat162float(w16[MLP_W1 + e]);
    for (int e = threadIdx.x; e < MLP_H; e += blockDim.x) {
        s.b1[e] = __bfloat162float(w16[MLP_B1 + e]);
        s.b2[e] = __bfloat162float(w16[MLP_B2 + e]);
        s.w3[e] = __bfloat162float(w16[MLP_W3 + e]);
    }
    if (threadIdx.x == 0) s.b3 = __bfloat162float(w16[MLP_B3]);
}

__device__ __forceinline__ float mlp_tanh(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// first layer of one element at hidden unit c
__device__ __forceinline__ float mlp_h1(const MlpInferSmem& s, const float (&f)[MLP_IN], int c) {
    float a = s.b1[c];
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) a = fmaf(f[i], s.w1[i * MLP_H + c], a);
    return mlp_tanh(a);
}

__device__ __forceinline__ uint32_t mlp_pack(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// Every warp of the grid takes tiles of 16 consecutive elements of [0, n);
// feat(e, f) fills the features of element e (e may be >= n: fill anything
// finite), out(e, y) receives the output of element e < n.
template <class Feat, class Out>
__device__ __forceinline__ void mlp_tiles(const MlpInferSmem& s, long long n, Feat feat, Out out) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long ntiles = (n + 15) / 16;
    for (long long tile = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; tile < ntiles; tile += nwarps) {
        const long long e0 = tile * 16 + g, e1 = e0 + 8;  // the fragment rows g and g + 8
        float f0[MLP_IN], f1[MLP_IN];
        feat(e0, f0);
        feat(e1, f1);
        float acc[MLP_H / 8][4];
#pragma unroll
        for (int nt = 0; nt < MLP_H / 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
        for (int ks = 0; ks < MLP_H / 16; ++ks) {
            const int c0 = 16 * ks + 2 * t;  // A fragment: rows g, g + 8; columns c0, c0 + 1, c0 + 8, c0 + 9
            uint32_t a[4];
            a[0] = mlp_pack(mlp_h1(s, f0, c0), mlp_h1(s, f0, c0 + 1));
            a[1] = mlp_pack(mlp_h1(s, f1, c0), mlp_h1(s, f1, c0 + 1));
            a[2] = mlp_pack(mlp_h1(s, f0, c0 + 8), mlp_h1(s, f0, c0 + 9));
            a[3] = mlp_pack(mlp_h1(s, f1, c0 + 8), mlp_h1(s, f1, c0 + 9));
#pragma unroll
            for (int nt = 0; nt < MLP_H / 8; ++nt) {
                const uint32_t* bw = s.w2t + (8 * nt + g) * MLP_W2T_LD + 8 * ks + t;
                const uint32_t b0 = bw[0], b1 = bw[4];  // B fragment: k rows 2t, 2t + 1 and 2t + 8, 2t + 9; column g
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                    "{%8, %9}, {%0, %1, %2, %3};\n"
                    : "+f"(acc[nt][0]), "+f"(acc[nt][1]), "+f"(acc[nt][2]), "+f"(acc[nt][3])
                    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
            }
        }
        // C fragment: rows g (acc[.][0..1]) and g + 8 (acc[.][2..3]), columns 8 nt + 2t + {0, 1}
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < MLP_H / 8; ++nt) {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int col = 8 * nt + 2 * t + i;
                y0 = fmaf(s.w3[col], mlp_tanh(acc[nt][i] + s.b2[col]), y0);
                y1 = fmaf(s.w3[col], mlp_tanh(acc[nt][2 + i] + s.b2[col]), y1);
            }
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (t == 0) {
            if (e0 < n) out(e0, y0 + s.b3);
            if (e1 < n) out(e1, y1 + s.b3);
        }
    }
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
