// mlp.cu -- hand-written inference, gradient and Adam kernels of the learned
// Davidson correction (no reference counterpart).  The network maps the
// features of one element (f0 = (diag - theta)/sigma, f1 = r/rms(r),
// f2 = u sqrt(N), f3 = bond position) to the error of the diagonal correction
// in units of rms(r)/sigma; it is trained by mean squared error on pairs the
// plain FP64 Davidson solver records in its own sweeps (target: the exact
// correction x/(u.x) - u towards the converged eigenvector x, minus the
// diagonal correction r/(theta - diag)).
//
// Inference reads BF16 weights, with the hidden layer on the tensor cores
// (mlp_tiles); training keeps an FP32 master copy: per block, every thread runs forward
// and backward for one pair, the activations go to shared memory, and the
// weight gradients are reduced there (dW2 = H1^T dH2 as a 64 x 64 x chunk
// product), then written as one partial per block and summed in a fixed
// order by the Adam kernel (deterministic).
#include "mlp.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace tnb {

namespace {

constexpr int TR_THREADS = 128;  // pairs per block and chunk

__global__ void mlp_forward_kernel(const __nv_bfloat16* __restrict__ w16, const float* __restrict__ F, long long n,
                                   float* __restrict__ Y) {
    __shared__ MlpInferSmem s;
    mlp_stage(w16, s);
    __syncthreads();
    mlp_tiles(
        s, n,
        [&](long long e, float(&f)[MLP_IN]) {
#pragma unroll
            for (int q = 0; q < MLP_IN; ++q) f[q] = e < n ? F[e * MLP_IN + q] : 0.f;
        },
        [&](long long e, float y) { Y[e] = y; });
}

// Gradient of L = inv_n * sum (y - t)^2 over pairs [first, first + count) of
// the (optionally permuted) set; one partial gradient per block.
__global__ void __launch_bounds__(TR_THREADS) mlp_grad_kernel(const float* __restrict__ w32,
                                                              const float* __restrict__ F,
                                                              const float* __restrict__ T,
                                                              const int* __restrict__ perm, long long first,
                                                              long long count, double inv_n,
                                                              float* __restrict__ part, double* __restrict__ loss_part) {
    extern __shared__ float sm[];
    float* w = sm;                                   // MLP_NP
    float* H1 = w + ((MLP_NP + 3) / 4) * 4;          // [TR_THREADS][MLP_H]
    float* D2 = H1 + TR_THREADS * MLP_H;             // dL/d(pre-activation 2)
    float* D1 = D2 + TR_THREADS * MLP_H;             // dL/d(pre-activation 1)
    float* H2 = D1 + TR_THREADS * MLP_H;             // [TR_THREADS][MLP_H]
    float* FS = H2 + TR_THREADS * MLP_H;             // [TR_THREADS][MLP_IN]
    float* DY = FS + TR_THREADS * MLP_IN;            // [TR_THREADS]
    __shared__ double lsum[TR_THREADS / 32];
    const int tid = threadIdx.x;
    for (int e = tid; e < MLP_NP; e += TR_THREADS) w[e] = w32[e];
    constexpr int NQ = MLP_H * MLP_H / TR_THREADS;
    float gW2[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) gW2[q] = 0.f;
    // thread tid < 64: b1, b2, W3, W1 rows 0-1 of column tid; 64 <= tid < 128: W1 rows 2-3
    float gA = 0, gB = 0, gB1 = 0, gB2 = 0, gW3 = 0, gB3 = 0;
    double lacc = 0;
    __syncthreads();
    const long long per_round = (long long)gridDim.x * TR_THREADS;
    const long long nchunks = (count + per_round - 1) / per_round;
    for (long long ch = 0; ch < nchunks; ++ch) {
        const long long idx = ch * per_round + (long long)blockIdx.x * TR_THREADS + tid;
        const bool valid = idx < count;
        float f[MLP_IN] = {0, 0, 0, 0};
        float tgt = 0;
        if (valid) {
            const long long p = perm ? (long long)perm[first + idx] : first + idx;
#pragma unroll
            for (int q = 0; q < MLP_IN; ++q) f[q] = F[p * MLP_IN + q];
            tgt = T[p];
        }
        // forward
        float* h1 = H1 + tid * MLP_H;
        float* h2 = H2 + tid * MLP_H;
        for (int j = 0; j < MLP_H; ++j) {
            float a = w[MLP_B1 + j];
#pragma unroll
            for (int i = 0; i < MLP_IN; ++i) a = fmaf(f[i], w[MLP_W1 + i * MLP_H + j], a);
            h1[j] = tanhf(a);
        }
        float y = w[MLP_B3];
        for (int k = 0; k < MLP_H; ++k) {
            float a = w[MLP_B2 + k];
            for (int j = 0; j < MLP_H; ++j) a = fmaf(h1[j], w[MLP_W2 + j * MLP_H + k], a);
            const float hk = tanhf(a);
            h2[k] = hk;
            y = fmaf(hk, w[MLP_W3 + k], y);
        }
        // backward of this pair
        const float err = valid ? (y - tgt) : 0.f;
        lacc += (double)err * err;
        const float dy = valid ? (float)(2.0 * inv_n) * err : 0.f;
        DY[tid] = dy;
#pragma unroll
        for (int q = 0; q < MLP_IN; ++q) FS[tid * MLP_IN + q] = f[q];
        float* d2 = D2 + tid * MLP_H;
        for (int k = 0; k < MLP_H; ++k) d2[k] = dy * w[MLP_W3 + k] * (1.f - h2[k] * h2[k]);
        float* d1 = D1 + tid * MLP_H;
        for (int j = 0; j < MLP_H; ++j) {
            float a = 0;
            for (int k = 0; k < MLP_H; ++k) a = fmaf(w[MLP_W2 + j * MLP_H + k], d2[k], a);
            d1[j] = a * (1.f - h1[j] * h1[j]);
        }
        __syncthreads();
        // weight gradients over the chunk's pairs
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int e = tid + q * TR_THREADS;  // dW2[j][k], e = j * MLP_H + k
            const int j = e / MLP_H, k = e % MLP_H;
            float a = 0;
            for (int s = 0; s < TR_THREADS; ++s) a = fmaf(H1[s * MLP_H + j], D2[s * MLP_H + k], a);
            gW2[q] += a;
        }
        if (tid < MLP_H) {
            float b1 = 0, b2 = 0, w3 = 0, w1a = 0, w1b = 0;
            for (int s = 0; s < TR_THREADS; ++s) {
                b1 += D1[s * MLP_H + tid];
                b2 += D2[s * MLP_H + tid];
                w3 = fmaf(H2[s * MLP_H + tid], DY[s], w3);
                w1a = fmaf(FS[s * MLP_IN + 0], D1[s * MLP_H + tid], w1a);
                w1b = fmaf(FS[s * MLP_IN + 1], D1[s * MLP_H + tid], w1b);
            }
            gB1 += b1;
            gB2 += b2;
            gW3 += w3;
            gA += w1a;
            gB += w1b;
        } else if (tid < 2 * MLP_H) {
            const int j = tid - MLP_H;
            float w1c = 0, w1d = 0;
            for (int s = 0; s < TR_THREADS; ++s) {
                w1c = fmaf(FS[s * MLP_IN + 2], D1[s * MLP_H + j], w1c);
                w1d = fmaf(FS[s * MLP_IN + 3], D1[s * MLP_H + j], w1d);
            }
            gA += w1c;
            gB += w1d;
        }
        if (tid == 0) {
            float b3 = 0;
            for (int s = 0; s < TR_THREADS; ++s) b3 += DY[s];
            gB3 += b3;
        }
        __syncthreads();
    }
    float* out = part + (size_t)blockIdx.x * MLP_NP;
#pragma unroll
    for (int q = 0; q < NQ; ++q) out[MLP_W2 + tid + q * TR_THREADS] = gW2[q];
    if (tid < MLP_H) {
        out[MLP_B1 + tid] = gB1;
        out[MLP_B2 + tid] = gB2;
        out[MLP_W3 + tid] = gW3;
        out[MLP_W1 + 0 * MLP_H + tid] = gA;
        out[MLP_W1 + 1 * MLP_H + tid] = gB;
    } else if (tid < 2 * MLP_H) {
        const int j = tid - MLP_H;
        out[MLP_W1 + 2 * MLP_H + j] = gA;
        out[MLP_W1 + 3 * MLP_H + j] = gB;
    }
    if (tid == 0) out[MLP_B3] = gB3;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lacc += __shfl_xor_sync(0xffffffffu, lacc, o);
    if ((tid & 31) == 0) lsum[tid >> 5] = lacc;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int q = 0; q < TR_THREADS / 32; ++q) s += lsum[q];
        loss_part[blockIdx.x] = s * inv_n;
    }
}

// Sum the block partials in order; Adam update of the FP32 master and BF16
// copy when lr > 0; the summed gradient goes to g when given.
__global__ void mlp_adam_kernel(const float* __restrict__ part, int nblocks, float* __restrict__ w32,
                                __nv_bfloat16* __restrict__ w16, float* __restrict__ m, float* __restrict__ v,
                                double lr, double b1t, double b2t, float* __restrict__ g) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_NP) return;
    double gs = 0;
    for (int b = 0; b < nblocks; ++b) gs += part[(size_t)b * MLP_NP + p];
    if (g) g[p] = (float)gs;
    if (lr <= 0) return;
    const double beta1 = 0.9, beta2 = 0.999, eps = 1e-8;
    const double mm = beta1 * m[p] + (1 - beta1) * gs;
    const double vv = beta2 * v[p] + (1 - beta2) * gs * gs;
    m[p] = (float)mm;
    v[p] = (float)vv;
    const double mh = mm / (1 - b1t), vh = vv / (1 - b2t);
    const float nw = (float)(w32[p] - lr * mh / (sqrt(vh) + eps));
    w32[p] = nw;
    w16[p] = __float2bfloat16(nw);
}

__global__ void mlp_to_bf16_kernel(const float* __restrict__ w32, __nv_bfloat16* __restrict__ w16) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < MLP_NP) w16[p] = __float2bfloat16(w32[p]);
}

size_t grad_smem_bytes() {
    return sizeof(float) * (((MLP_NP + 3) / 4) * 4 + 4 * (size_t)TR_THREADS * MLP_H + (size_t)TR_THREADS * MLP_IN +
                            TR_THREADS);
}

int grad_blocks(long long count, int sm) {
    long long b = (count + TR_THREADS - 1) / TR_THREADS;
    return (int)std::max<long long>(1, std::min<long long>(b, (long long)sm));
}

int ensure_grad_attr() {
    static thread_local int dev_set = -1;
    int dev = 0;
    TN_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev_set != dev) {
        TN_CUDA_CHECK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)grad_smem_bytes()));
        dev_set = dev;
    }
    return TN_OK;
}

}  // namespace

int mlp_init(MlpModel& m, Ctx& c, unsigned long long seed) {
    m.ctx = &c;
    TN_CHECK(m.w32.ensure(sizeof(float) * MLP_NP));
    TN_CHECK(m.w16.ensure(sizeof(__nv_bfloat16) * MLP_NP));
    TN_CHECK(m.m.ensure(sizeof(float) * MLP_NP));
    TN_CHECK(m.v.ensure(sizeof(float) * MLP_NP));
    // Glorot-uniform weights from a seeded generator, zero biases
    std::vector<float> h(MLP_NP, 0.f);
    std::mt19937_64 g(seed);
    auto fill = [&](int off, int fan_in, int fan_out, int cnt) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int i = 0; i < cnt; ++i) h[off + i] = (float)(((g() >> 11) * (1.0 / 9007199254740992.0) * 2 - 1) * a);
    };
    fill(MLP_W1, MLP_IN, MLP_H, MLP_IN * MLP_H);
    fill(MLP_W2, MLP_H, MLP_H, MLP_H * MLP_H);
    fill(MLP_W3, MLP_H, 1, MLP_H);
    return mlp_set_params(m, h.data());
}

int mlp_set_params(MlpModel& m, const float* host) {
    cudaStream_t st = m.ctx->stream;
    TN_CUDA_CHECK(cudaMemcpyAsync(m.w32.p, host, sizeof(float) * MLP_NP, cudaMemcpyHostToDevice, st));
    TN_CUDA_CHECK(cudaMemsetAsync(m.m.p, 0, sizeof(float) * MLP_NP, st));
    TN_CUDA_CHECK(cudaMemsetAsync(m.v.p, 0, sizeof(float) * MLP_NP, st));
    mlp_to_bf16_kernel<<<(MLP_NP + 255) / 256, 256, 0, st>>>(m.w32.as<float>(), m.w16.as<__nv_bfloat16>());
    TN_LAUNCH_CHECK();
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    m.adam_t = 0;
    return TN_OK;
}

int mlp_get_params(const MlpModel& m, float* host) {
    cudaStream_t st = m.ctx->stream;
    TN_CUDA_CHECK(cudaMemcpyAsync(host, m.w32.p, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    return TN_OK;
}

int mlp_forward(const MlpModel& m, const float* F, long long n, float* Y, cudaStream_t st) {
    if (n <= 0) return TN_OK;
    const long long b = (n + 127) / 128;  // 8 warps of 16-element tiles per block
    const int grid = (int)std::min<long long>(b, (long long)m.ctx->sm_count * 4);
    mlp_forward_kernel<<<grid, 256, 0, st>>>(m.w16.as<__nv_bfloat16>(), F, n, Y);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int mlp_gradient(MlpModel& m, const float* F, const float* T, long long n, float* grad_host, double* loss) {
    Ctx& c = *m.ctx;
    cudaStream_t st = c.stream;
    if (n <= 0) return TN_BAD_ARG;
    TN_CHECK(ensure_grad_attr());
    const int nb = grad_blocks(n, c.sm_count);
    TN_CHECK(m.part.ensure(sizeof(float) * ((size_t)nb * MLP_NP + MLP_NP)));
    TN_CHECK(m.loss.ensure(sizeof(double) * nb));
    mlp_grad_kernel<<<nb, TR_THREADS, grad_smem_bytes(), st>>>(m.w32.as<float>(), F, T, nullptr, 0, n, 1.0 / n,
                                                              m.part.as<float>(), m.loss.as<double>());
    TN_LAUNCH_CHECK();
    float* g = m.part.as<float>() + (size_t)nb * MLP_NP;
    mlp_adam_kernel<<<(MLP_NP + 255) / 256, 256, 0, st>>>(m.part.as<float>(), nb, m.w32.as<float>(),
                                                          m.w16.as<__nv_bfloat16>(), m.m.as<float>(), m.v.as<float>(),
                                                          0.0, 0.0, 0.0, g);
    TN_LAUNCH_CHECK();
    std::vector<double> lp(nb);
    TN_CUDA_CHECK(cudaMemcpyAsync(grad_host, g, sizeof(float) * MLP_NP, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaMemcpyAsync(lp.data(), m.loss.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    double l = 0;
    for (double x : lp) l += x;
    if (loss) *loss = l;
    return TN_OK;
}

int mlp_train(MlpModel& m, const float* F, const float* T, long long n, int steps, int batch, double lr,
              unsigned long long seed, double* final_loss) {
    Ctx& c = *m.ctx;
    cudaStream_t st = c.stream;
    if (n <= 0 || steps <= 0) return TN_BAD_ARG;
    if (batch <= 0 || batch > n) batch = (int)std::min<long long>(n, 4096);
    TN_CHECK(ensure_grad_attr());
    // seeded permutation of the pairs (host Fisher-Yates, uploaded once)
    std::vector<int> perm(n);
    for (long long i = 0; i < n; ++i) perm[i] = (int)i;
    std::mt19937_64 g(seed);
    for (long long i = n - 1; i > 0; --i) {
        const long long j = (long long)(g() % (unsigned long long)(i + 1));
        std::swap(perm[i], perm[j]);
    }
    DevBuf dperm;
    TN_CHECK(dperm.ensure(sizeof(int) * n));
    TN_CUDA_CHECK(cudaMemcpyAsync(dperm.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    const int nb = grad_blocks(batch, c.sm_count);
    TN_CHECK(m.part.ensure(sizeof(float) * ((size_t)nb * MLP_NP + MLP_NP)));
    TN_CHECK(m.loss.ensure(sizeof(double) * nb));
    const long long nbatches = std::max<long long>(1, n / batch);
    for (int s = 0; s < steps; ++s) {
        const long long first = (s % nbatches) * batch;
        mlp_grad_kernel<<<nb, TR_THREADS, grad_smem_bytes(), st>>>(m.w32.as<float>(), F, T, dperm.as<int>(), first,
                                                                  batch, 1.0 / batch, m.part.as<float>(),
                                                                  m.loss.as<double>());
        TN_LAUNCH_CHECK();
        ++m.adam_t;
        const double b1t = std::pow(0.9, (double)m.adam_t), b2t = std::pow(0.999, (double)m.adam_t);
        mlp_adam_kernel<<<(MLP_NP + 255) / 256, 256, 0, st>>>(m.part.as<float>(), nb, m.w32.as<float>(),
                                                              m.w16.as<__nv_bfloat16>(), m.m.as<float>(),
                                                              m.v.as<float>(), lr, b1t, b2t, nullptr);
        TN_LAUNCH_CHECK();
    }
    std::vector<double> lp(nb);
    TN_CUDA_CHECK(cudaMemcpyAsync(lp.data(), m.loss.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    double l = 0;
    for (double x : lp) l += x;
    if (final_loss) *final_loss = l;
    return TN_OK;
}

int recorder_init(DvRecorder& r, Ctx& c, long long capacity) {
    r.ctx = &c;
    r.capacity = capacity;
    r.size = 0;
    TN_CHECK(r.feats.ensure(sizeof(float) * MLP_IN * (size_t)capacity));
    TN_CHECK(r.targets.ensure(sizeof(float) * (size_t)capacity));
    return TN_OK;
}

}  // namespace tnb
