// mixed.cu -- split-precision effective-Hamiltonian matvec (BF16x3 on tcgen05).
//
//   y = sum_{w1,w2,n} W(w1,w2)(m,n) F_w1 x_n G_w2^T      (MPSSite::GetHeff,
//        MPSSite_Contractions.C:155-193, matrix-free)
//
// Per site (constant over the Krylov loop) the FP64 environments are split
// once into BF16 (hi, lo) pairs in K-major layouts; the channel of F and G that
// carries the completed block energy is shifted by its mean diagonal so that
// the split operand is O(1) instead of O(L) (the matvec then applies
// Heff - sigma I, which has the same eigenvectors; energies are recomputed in
// FP64).  Per matvec: split x (FP64 -> BF16 pairs), stage 1 on the tensor
// cores (P[w1,n] = F_w1 x_n, FP32 out), stage 2 on CUDA cores (the sparse W
// combination, FP32, re-split to BF16 pieces), stage 3 on the tensor cores
// split over w2 for parallelism (Yp[m,w2] = Q[m,w2] G_w2^T, FP32 partials) and a
// deterministic FP64 sum over w2 into y.
#include <cuda_bf16.h>

#include <algorithm>

#include "mixed.h"
#include "pdl.cuh"

namespace tnb {

namespace {

// v = piece0 + piece1 (+ piece2) + O(2^-8 per piece): successive BF16 remainders.
__device__ __forceinline__ void split_bf16(float v, int ns, uint16_t* base, long long pstride, long long e) {
    float r = v;
    for (int q = 0; q < ns; ++q) {
        __nv_bfloat16 h = __float2bfloat16_rn(r);
        base[q * pstride + e] = __bfloat16_as_ushort(h);
        r -= __bfloat162float(h);
    }
}

inline int g1d(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

// mean of the diagonal of block w of a Dw x D x D environment -> out
__global__ void block_trace_kernel(const double* __restrict__ E, int D, int w, double* out) {
    __shared__ double sh[32];
    double s = 0;
    if (w >= 0)
        for (int i = threadIdx.x; i < D; i += blockDim.x) s += E[(long long)w * D * D + (long long)i * D + i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        *out = w >= 0 ? t / D : 0.0;
    }
}

// Environment E (Dw x D x D, column-major blocks: (w,i,j) at w*D*D + j*D + i) ->
// Es[w][i][j] (j contiguous: K-major rows), block wshift shifted by -(*shift) on
// the diagonal.  Used for both F (rows i1, K = j1) and G (rows i2, K = j2).
__global__ void split_env_left_kernel(const double* __restrict__ F, int Dw, int D, int wshift,
                                      const double* __restrict__ shift, uint16_t* __restrict__ out, int ns,
                                      long long pstride) {
    const long long total = (long long)Dw * D * D;
    const double sft = shift ? *shift : 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e % D);
        const int i = (int)((e / D) % D);
        const int w = (int)(e / ((long long)D * D));
        double v = F[(long long)w * D * D + (long long)j * D + i];
        if (w == wshift && i == j) v -= sft;
        split_bf16((float)v, ns, out, pstride, e);
    }
}

__global__ void split_vec_kernel(const double* __restrict__ x, long long n, uint16_t* __restrict__ out, int ns,
                                 long long pstride, const int* skip) {
    pdl_wait();
    if (skip && *skip) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        split_bf16((float)x[e], ns, out, pstride, e);
}

// Q[m][w2][i1][j2] = sum_terms c * P[(w1,n)][i1][j2], split into BF16 pieces.
__global__ void wcombine_split_kernel(const float* __restrict__ P, uint16_t* __restrict__ qout, int ns,
                                      long long pstride, const WTermDev* __restrict__ terms, int nterms,
                                      int D1, int D2, int Dwout, const int* skip) {
    pdl_wait();
    if (skip && *skip) return;
    const long long blk = (long long)D1 * D2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < blk;
         e += (long long)gridDim.x * blockDim.x) {
        int cur = terms[0].out;
        float acc = 0.0f;
        for (int t = 0; t <= nterms; ++t) {
            const bool flush = (t == nterms) || (terms[t].out != cur);
            if (flush) {
                // out slab cur = m*Dwout + w2; Q layout [m][w2][i1][j2]
                const long long o = (long long)cur * blk + e;
                split_bf16(acc, ns, qout, pstride, o);
                if (t == nterms) break;
                acc = 0.0f;
                cur = terms[t].out;
            }
            acc = fmaf((float)terms[t].c, P[(long long)terms[t].in * blk + e], acc);
        }
    }
}

// y[m][e] = sum_w2 Yp[(m*Dw2 + w2)][e]   (FP32 partials -> FP64 site layout)
__global__ void reduce_w2_kernel(const float* __restrict__ Yp, int d, int Dw2, long long blk, double* __restrict__ y,
                                 const int* skip) {
    pdl_wait();
    if (skip && *skip) return;
    const long long total = (long long)d * blk;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long m = e / blk, r = e - m * blk;
        double s = 0.0;
        for (int w = 0; w < Dw2; ++w) s += (double)Yp[((long long)m * Dw2 + w) * blk + r];
        y[e] = s;
    }
}

}  // namespace

static inline size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

int mixed_prepare_site(Ctx& c, MixedSite& ms, const ContractShape& s, const WTermDev* termsLR, int nLR,
                       const double* F, const double* G, int wshiftF, int wshiftG, int nsplit) {
    cudaStream_t st = c.stream;
    const int d = s.d, Dw1 = s.Dw1, Dw2 = s.Dw2, D1 = s.D1, D2 = s.D2;
    if (!mixed_supported(s)) {
        set_error("mixed matvec needs D1, D2 multiples of 16 (got %d, %d)", D1, D2);
        return TN_BAD_SHAPE;
    }
    if (nsplit != 2 && nsplit != 3) return TN_BAD_ARG;
    const int ns = nsplit;
    const long long blk = (long long)D1 * D2;
    const size_t nF = pad8((size_t)Dw1 * D1 * D1), nG = pad8((size_t)Dw2 * D2 * D2), nX = pad8((size_t)d * blk);
    const size_t nP = (size_t)std::max(Dw1, Dw2) * d * blk, nQ = pad8((size_t)d * D1 * Dw2 * D2);
    TN_CHECK(ms.Fs.ensure(2 * ns * nF));
    TN_CHECK(ms.Gs.ensure(2 * ns * nG));
    TN_CHECK(ms.Xs.ensure(2 * ns * nX));
    TN_CHECK(ms.P32.ensure(4 * nP + 64));
    TN_CHECK(ms.Qs.ensure(2 * ns * nQ));
    TN_CHECK(ms.shifts.ensure(4 * sizeof(double)));
    TN_CHECK(ms.err.ensure(sizeof(int)));
    TN_CUDA_CHECK(cudaMemsetAsync(ms.err.p, 0, sizeof(int), st));
    uint16_t* Fp = ms.Fs.as<uint16_t>();
    uint16_t* Gp = ms.Gs.as<uint16_t>();
    double* sh = ms.shifts.as<double>();
    const int wF = (Dw1 > 1) ? wshiftF : -1;
    const int wG = (Dw2 > 1) ? wshiftG : -1;
    block_trace_kernel<<<1, 256, 0, st>>>(F, D1, wF, sh);
    TN_LAUNCH_CHECK();
    block_trace_kernel<<<1, 256, 0, st>>>(G, D2, wG, sh + 1);
    TN_LAUNCH_CHECK();
    split_env_left_kernel<<<g1d(nF), 256, 0, st>>>(F, Dw1, D1, wF, sh, Fp, ns, (long long)nF);
    TN_LAUNCH_CHECK();
    split_env_left_kernel<<<g1d(nG), 256, 0, st>>>(G, Dw2, D2, wG, sh + 1, Gp, ns, (long long)nG);
    TN_LAUNCH_CHECK();
    ms.shape = s;
    ms.termsLR = termsLR;
    ms.nLR = nLR;
    ms.nsplit = ns;
    ms.nX = nX;
    ms.nQ = nQ;
    // stage 1: P[(w1,n)](i1, j2) = sum_j1 Fs[w1](i1, j1) Xs[n](j2, j1)
    TcGemmArgs a1;
    a1.M = D1; a1.N = D2; a1.K = D1; a1.batch = Dw1 * d; a1.nsplit = ns;
    for (int q = 0; q < ns; ++q) {
        a1.a[q] = Fp + q * nF;
        a1.b[q] = ms.Xs.as<uint16_t>() + q * nX;
    }
    a1.lda = D1; a1.a_batch = (long long)D1 * D1; a1.a_nbatch = Dw1; a1.a_bdiv = d; a1.a_bmod = Dw1;
    a1.ldb = D1; a1.b_batch = blk; a1.b_nbatch = d; a1.b_bdiv = 1; a1.b_bmod = d;
    a1.out_mode = TC_OUT_F32_ROWMAJOR; a1.c32 = ms.P32.as<float>(); a1.ldc = D2; a1.c_batch = blk;
    a1.err = ms.err.as<int>();
    TN_CHECK(tc_gemm_plan(a1, &ms.plan1));
    // stage 3, split over w2: Yp[(m,w2)](i1, i2) = sum_j2 Qs[(m,w2)](i1, j2) Gs[w2](i2, j2)
    // (FP32 column-major partials), then y_m = sum_w2 Yp[(m,w2)] in FP64
    TcGemmArgs a3;
    a3.M = D1; a3.N = D2; a3.K = D2; a3.batch = d * Dw2; a3.nsplit = ns;
    for (int q = 0; q < ns; ++q) {
        a3.a[q] = ms.Qs.as<uint16_t>() + q * nQ;
        a3.b[q] = Gp + q * nG;
    }
    a3.lda = D2; a3.a_batch = blk; a3.a_nbatch = d * Dw2; a3.a_bdiv = 1; a3.a_bmod = d * Dw2;
    a3.ldb = D2; a3.b_batch = (long long)D2 * D2; a3.b_nbatch = Dw2; a3.b_bdiv = 1; a3.b_bmod = Dw2;
    a3.out_mode = TC_OUT_F32_COLMAJOR; a3.c32 = ms.P32.as<float>(); a3.ldc = D1; a3.c_batch = blk;
    a3.err = ms.err.as<int>();
    TN_CHECK(tc_gemm_plan(a3, &ms.plan3));
    ms.ready = true;
    return TN_OK;
}

int heff_matvec_mixed(Ctx& c, MixedSite& ms, const double* x, double* y, const int* skip) {
    cudaStream_t st = c.stream;
    const ContractShape& s = ms.shape;
    const long long blk = (long long)s.D1 * s.D2;
    const long long nX = (long long)s.d * blk;
    TN_CHECK(launch_pdl(split_vec_kernel, g1d(nX), 256, 0, st, x, nX, ms.Xs.as<uint16_t>(), ms.nsplit,
                        (long long)ms.nX, skip));
    TcGemmPlan p1 = ms.plan1;
    p1.args.skip = skip;
    TN_CHECK(tc_gemm_run(p1, st));
    TN_CHECK(launch_pdl(wcombine_split_kernel, g1d(blk), 256, 0, st, (const float*)ms.P32.as<float>(),
                        ms.Qs.as<uint16_t>(), ms.nsplit, (long long)ms.nQ, (const WTermDev*)ms.termsLR, ms.nLR, s.D1,
                        s.D2, s.Dw2, skip));
    TcGemmPlan p3 = ms.plan3;
    p3.args.skip = skip;
    TN_CHECK(tc_gemm_run(p3, st));
    if (c.take_tail) {  // the caller forms y with its own next kernel
        MatvecTail& t = *c.take_tail;
        t.deferred = true;
        t.Yp = ms.P32.as<float>();
        t.d = s.d;
        t.Dw2 = s.Dw2;
        t.blk = blk;
        return TN_OK;
    }
    TN_CHECK(launch_pdl(reduce_w2_kernel, g1d(nX), 256, 0, st, (const float*)ms.P32.as<float>(), s.d, s.Dw2, blk, y,
                        skip));
    return TN_OK;
}

int mixed_check_error(MixedSite& ms, cudaStream_t st) {
    int h = 0;
    TN_CUDA_CHECK(cudaMemcpyAsync(&h, ms.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    if (h) {
        set_error("tcgen05 GEMM: a bounded mbarrier wait expired");
        return TN_CUDA_ERROR;
    }
    return TN_OK;
}

double mixed_shift_host(MixedSite& ms, cudaStream_t st) {
    double h[2] = {0, 0};
    cudaMemcpyAsync(h, ms.shifts.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return h[0] + h[1];
}

}  // namespace tnb
