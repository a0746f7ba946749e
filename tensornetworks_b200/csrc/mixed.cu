// mixed.cu -- split-precision effective-Hamiltonian matvec (BF16 pieces on tcgen05).
//
//   y_m = sum_{w1,w2,n} W(w1,w2)(m,n) F_w1 x_n G_w2^T      (MPSSite::GetHeff,
//         MPSSite_Contractions.C:155-193, matrix-free)
//
// Per site (constant over the Krylov loop) the FP64 environments are split
// once into BF16 pieces in K-major layouts: F as [w1][i1][j1], and for every
// distinct (w2, c) pair among the MPO's nonzero entries the scaled copy
// c G_w2 as [u][i2][j2].  The channel of F and G that carries the completed
// block energy is shifted by its mean diagonal so that the split operand is
// O(1) instead of O(L) (the matvec then applies Heff - sigma I, which has the
// same eigenvectors; energies are recomputed in FP64).  Per matvec:
//   split x (FP64 -> BF16 pieces);
//   GEMM 1 (tcgen05): P[(w1,n)](i1, j2) = sum_j1 F_w1(i1, j1) x_n(j1, j2),
//     written by the cluster epilogue straight as BF16 pieces;
//   GEMM 2 (tcgen05): y_m(i1, i2) = sum_{terms (w1,n,u) of m} sum_j2
//     P[(w1,n)](i1, j2) (c_u G_w2u)(i2, j2) -- the MPO combination is the K
//     dimension of one segmented GEMM, so no CUDA-core combination pass, no
//     FP32 partials in HBM and no separate reduction remain; the cluster
//     epilogue writes y in FP64.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <unordered_map>

#include "mixed.h"
#include "pdl.cuh"
#include "split.cuh"

namespace tnb {

namespace {

// v = piece0 + piece1 (+ piece2) + O(2^-8 per piece): successive BF16 remainders.
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

// Environment E (Dw x D x D, (w,i,j) at w*D*D + j*D + i) -> Es[w][i][j]
// (j contiguous: K-major rows), block wshift shifted by -(*shift) on the diagonal.
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

struct ScaleList {
    int n;
    int w[MIXED_MAX_SCALED];
    double c[MIXED_MAX_SCALED];
};

// Gc[u][i][j] = c_u * G_{w_u}(i, j) (block wshift shifted on the diagonal), split.
__global__ void split_env_scaled_kernel(const double* __restrict__ G, int D, int wshift,
                                        const double* __restrict__ shift, const ScaleList sl,
                                        uint16_t* __restrict__ out, int ns, long long pstride) {
    const long long total = (long long)sl.n * D * D;
    const double sft = shift ? *shift : 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e % D);
        const int i = (int)((e / D) % D);
        const int u = (int)(e / ((long long)D * D));
        const int w = sl.w[u];
        double v = G[(long long)w * D * D + (long long)j * D + i];
        if (w == wshift && i == j) v -= sft;
        split_bf16((float)(sl.c[u] * v), ns, out, pstride, e);
    }
}

__global__ void split_vec_kernel(const double* __restrict__ x, long long n, uint16_t* __restrict__ out, int ns,
                                 long long pstride, const int* skip) {
    pdl_launch_dependents();
    pdl_wait();
    if (skip && *skip) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        split_bf16((float)x[e], ns, out, pstride, e);
}

}  // namespace

static inline size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

// Split-K factors of the two GEMMs chosen by measurement, per operator shape
// (d, Dw1, Dw2, D1, D2, pieces, segments per output, SMs): the first time a
// shape is prepared, every candidate pair is timed with CUDA events over a few
// matvecs on the context stream and the fastest kept for the process.
namespace {
std::mutex g_tune_mu;
std::unordered_map<unsigned long long, std::pair<int, int>> g_tune;

int time_matvec_pair(Ctx& c, MixedSite& ms, const TcChainArgs& a1, const TcChainArgs& a2, int sk1, int sk2,
                     double* x, double* y, float* ms_out) {
    TcChainArgs b1 = a1, b2 = a2;
    b1.splitk = sk1;
    b2.splitk = sk2;
    b2.c64 = y;
    TN_CHECK(tc_chain_plan(b1, &ms.plan1));
    TN_CHECK(tc_chain_plan(b2, &ms.plan2));
    for (int w = 0; w < 2; ++w) TN_CHECK(heff_matvec_mixed(c, ms, x, y, nullptr));
    constexpr int REPS = 6;
    // events of its own: the context's timing events may be bracketing a sweep
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TN_CUDA_CHECK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        set_error("mixed autotune: cudaEventCreate failed");
        return TN_CUDA_ERROR;
    }
    int rc = TN_OK;
    cudaError_t er = cudaEventRecord(e0, c.stream);
    for (int r = 0; r < REPS && rc == TN_OK && er == cudaSuccess; ++r) rc = heff_matvec_mixed(c, ms, x, y, nullptr);
    if (er == cudaSuccess) er = cudaEventRecord(e1, c.stream);
    if (er == cudaSuccess) er = cudaEventSynchronize(e1);
    float t = 0;
    if (er == cudaSuccess) er = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    TN_CHECK(rc);
    TN_CUDA_CHECK(er);
    *ms_out = t / REPS;
    return TN_OK;
}
}  // namespace


int mixed_prepare_site(Ctx& c, MixedSite& ms, const ContractShape& s, const double* W_host, const double* F,
                       const double* G, int wshiftF, int wshiftG, int nsplit) {
    cudaStream_t st = c.stream;
    const int d = s.d, Dw1 = s.Dw1, Dw2 = s.Dw2, D1 = s.D1, D2 = s.D2;
    if (!mixed_supported(s)) {
        set_error("mixed matvec needs D1, D2 multiples of 16 (got %d, %d)", D1, D2);
        return TN_BAD_SHAPE;
    }
    if (nsplit != 2 && nsplit != 3) return TN_BAD_ARG;
    const int ns = nsplit;
    const long long blk = (long long)D1 * D2;
    // MPO terms of each output m: (w1 d + n, scaled-copy index u of (w2, c))
    ScaleList sl{};
    const int nb1 = Dw1 * d;
    std::vector<int> tab;
    tab.reserve(4 * nb1 + 4 * d * Dw1 * Dw2 * d + 8);
    for (int b = 0; b <= nb1; ++b) tab.push_back(b);  // GEMM 1: one segment per output batch (w1, n)
    for (int b = 0; b < nb1; ++b) {
        tab.push_back(b / d);  // F block w1
        tab.push_back(b % d);  // x block n
    }
    const int off2 = (int)tab.size();
    std::vector<int> segs2;
    std::vector<int> start2(1, 0);
    int maxseg = 0;
    for (int m = 0; m < d; ++m) {
        int cnt = 0;
        for (int w1 = 0; w1 < Dw1; ++w1)
            for (int w2 = 0; w2 < Dw2; ++w2)
                for (int n = 0; n < d; ++n) {
                    const double cf = W_host[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
                    if (cf == 0.0) continue;
                    int u = 0;
                    while (u < sl.n && !(sl.w[u] == w2 && sl.c[u] == cf)) ++u;
                    if (u == sl.n) {
                        if (sl.n == MIXED_MAX_SCALED) {
                            set_error("mixed matvec: more than %d distinct (w2, coefficient) MPO entries",
                                      MIXED_MAX_SCALED);
                            return TN_BAD_SHAPE;
                        }
                        sl.w[sl.n] = w2;
                        sl.c[sl.n] = cf;
                        ++sl.n;
                    }
                    segs2.push_back(w1 * d + n);
                    segs2.push_back(u);
                    ++cnt;
                }
        start2.push_back(start2.back() + cnt);
        maxseg = std::max(maxseg, cnt);
    }
    tab.insert(tab.end(), start2.begin(), start2.end());
    const int offs2 = (int)tab.size();
    tab.insert(tab.end(), segs2.begin(), segs2.end());
    const int nU = std::max(sl.n, 1);

    const size_t nF = pad8((size_t)Dw1 * D1 * D1), nG = pad8((size_t)nU * D2 * D2);
    const size_t nX = pad8((size_t)d * blk), nP = pad8((size_t)nb1 * blk);
    TN_CHECK(ms.Fs.ensure(2 * ns * nF));
    TN_CHECK(ms.Gc.ensure(2 * ns * nG));
    TN_CHECK(ms.Xs.ensure(2 * ns * nX));
    TN_CHECK(ms.Ps.ensure(2 * ns * nP));
    TN_CHECK(ms.shifts.ensure(4 * sizeof(double)));
    TN_CHECK(ms.err.ensure(sizeof(int)));
    const void* old_segs = ms.segs.p;
    TN_CHECK(ms.segs.ensure(sizeof(int) * tab.size()));
    if (ms.segs.p != old_segs || ms.seg_host != tab) {
        // pageable source: staged before the call returns
        TN_CUDA_CHECK(cudaMemcpyAsync(ms.segs.p, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, st));
        ms.seg_host = tab;
    }
    TN_CUDA_CHECK(cudaMemsetAsync(ms.err.p, 0, sizeof(int), st));
    uint16_t* Fp = ms.Fs.as<uint16_t>();
    uint16_t* Gp = ms.Gc.as<uint16_t>();
    double* sh = ms.shifts.as<double>();
    const int wF = (Dw1 > 1) ? wshiftF : -1;
    const int wG = (Dw2 > 1) ? wshiftG : -1;
    block_trace_kernel<<<1, 256, 0, st>>>(F, D1, wF, sh);
    TN_LAUNCH_CHECK();
    block_trace_kernel<<<1, 256, 0, st>>>(G, D2, wG, sh + 1);
    TN_LAUNCH_CHECK();
    split_env_left_kernel<<<g1d((long long)Dw1 * D1 * D1), 256, 0, st>>>(F, Dw1, D1, wF, sh, Fp, ns, (long long)nF);
    TN_LAUNCH_CHECK();
    if (sl.n > 0) {
        split_env_scaled_kernel<<<g1d((long long)sl.n * D2 * D2), 256, 0, st>>>(G, D2, wG, sh + 1, sl, Gp, ns,
                                                                               (long long)nG);
        TN_LAUNCH_CHECK();
    }
    ms.shape = s;
    ms.nsplit = ns;
    ms.nU = nU;
    ms.nF = nF;
    ms.nG = nG;
    ms.nX = nX;
    ms.nP = nP;
    const int* tabd = ms.segs.as<int>();
    const int mt = (D1 + 127) / 128;
    // GEMM 1: P[(w1,n)](i1, j2) = sum_j1 Fs[w1](i1, j1) Xs[n](j2, j1)  -> BF16 pieces, row-major
    TcChainArgs a1;
    a1.M = D1; a1.N = D2; a1.K = D1; a1.nbatch = nb1; a1.nsplit = ns;
    for (int q = 0; q < ns; ++q) {
        a1.a[q] = Fp + q * nF;
        a1.b[q] = ms.Xs.as<uint16_t>() + q * nX;
    }
    a1.lda = D1; a1.a_batch = (long long)D1 * D1; a1.a_nbatch = Dw1;
    a1.ldb = D1; a1.b_batch = blk; a1.b_nbatch = d;
    a1.seg_start = tabd;
    a1.segs = reinterpret_cast<const TcSeg*>(tabd + nb1 + 1);
    a1.splitk = tc_chain_splitk(((D2 + 63) / 64) * mt * nb1, (D1 + 63) / 64, c.sm_count);
    a1.out_mode = TCC_OUT_BF16_ROWMAJOR;
    a1.c16 = ms.Ps.as<uint16_t>(); a1.c16_piece = (long long)nP; a1.ldc16 = D2; a1.c16_batch = blk;
    a1.err = ms.err.as<int>();
    // GEMM 2: y_m(i1, i2) = sum_{(b, u) in segments(m)} sum_j2 P[b](i1, j2) Gc[u](i2, j2)  -> FP64
    TcChainArgs a2;
    a2.M = D1; a2.N = D2; a2.K = D2; a2.nbatch = d; a2.nsplit = ns;
    for (int q = 0; q < ns; ++q) {
        a2.a[q] = ms.Ps.as<uint16_t>() + q * nP;
        a2.b[q] = Gp + q * nG;
    }
    a2.lda = D2; a2.a_batch = blk; a2.a_nbatch = nb1;
    a2.ldb = D2; a2.b_batch = (long long)D2 * D2; a2.b_nbatch = nU;
    a2.seg_start = tabd + off2;
    a2.segs = reinterpret_cast<const TcSeg*>(tabd + offs2);
    a2.splitk = tc_chain_splitk(((D2 + 63) / 64) * mt * d, maxseg * ((D2 + 63) / 64), c.sm_count);
    a2.out_mode = TCC_OUT_F64_COLMAJOR;
    a2.c64 = nullptr;  // y, set per call
    a2.ldc64 = D1; a2.c64_batch = blk;
    a2.err = ms.err.as<int>();
    // split-K factors: measured once per shape (TN_NO_AUTOTUNE=1: the occupancy heuristic)
    const int chunks1 = (D1 + 63) / 64, chunks2 = maxseg * ((D2 + 63) / 64);
    unsigned long long key = hash_val(HASH_SEED, s);
    key = hash_val(key, ns);
    key = hash_val(key, maxseg);
    key = hash_val(key, c.sm_count);
    bool have = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            a1.splitk = it->second.first;
            a2.splitk = it->second.second;
            have = true;
        }
    }
    const char* nt = std::getenv("TN_NO_AUTOTUNE");
    // TN_CHAIN_SPLITK="s1,s2" forces the pair (tests exercise every variant with it)
    const char* forced = std::getenv("TN_CHAIN_SPLITK");
    int f1 = 0, f2 = 0;
    if (forced && std::sscanf(forced, "%d,%d", &f1, &f2) == 2 && f1 >= 1 && f1 <= 8 && f2 >= 1 && f2 <= 8 &&
        (f1 & (f1 - 1)) == 0 && (f2 & (f2 - 1)) == 0) {
        a1.splitk = f1;
        a2.splitk = f2;
        have = true;
    }
    if (!have && !(nt && nt[0] == '1')) {
        TN_CHECK(ms.tune.ensure(2 * sizeof(double) * (size_t)d * blk));
        double* tx = ms.tune.as<double>();
        double* ty = tx + (size_t)d * blk;
        TN_CUDA_CHECK(cudaMemsetAsync(tx, 0, 2 * sizeof(double) * (size_t)d * blk, st));
        ms.shape = s;
        float best = 1e30f;
        int b1 = a1.splitk, b2 = a2.splitk;
        for (int sk1 = 1; sk1 <= 8 && sk1 <= chunks1; sk1 *= 2)
            for (int sk2 = 1; sk2 <= 8 && sk2 <= chunks2; sk2 *= 2) {
                float t = 0;
                TN_CHECK(time_matvec_pair(c, ms, a1, a2, sk1, sk2, tx, ty, &t));
                if (t < best) {
                    best = t;
                    b1 = sk1;
                    b2 = sk2;
                }
            }
        a1.splitk = b1;
        a2.splitk = b2;
        TN_CHECK(mixed_check_error(ms, st));
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = {b1, b2};
    }
    ms.splitk1 = a1.splitk;
    ms.splitk2 = a2.splitk;
    TN_CHECK(tc_chain_plan(a1, &ms.plan1));
    {
        // plan with a placeholder output; heff_matvec_mixed sets y
        TcChainArgs tmp = a2;
        tmp.c64 = reinterpret_cast<double*>(ms.Xs.p);
        TN_CHECK(tc_chain_plan(tmp, &ms.plan2));
    }
    ms.ready = true;
    return TN_OK;
}

int heff_matvec_mixed(Ctx& c, MixedSite& ms, const double* x, double* y, const int* skip) {
    cudaStream_t st = c.stream;
    const ContractShape& s = ms.shape;
    const long long nX = (long long)s.d * s.D1 * s.D2;
    if (!ms.presplit)
        TN_CHECK(launch_pdl(split_vec_kernel, g1d(nX), 256, 0, st, x, nX, ms.Xs.as<uint16_t>(), ms.nsplit,
                            (long long)ms.nX, skip));
    TcChainPlan p1 = ms.plan1;
    p1.args.skip = skip;
    TN_CHECK(tc_chain_run(p1, st));
    TcChainPlan p2 = ms.plan2;
    p2.args.skip = skip;
    p2.args.c64 = y;
    TN_CHECK(tc_chain_run(p2, st));
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
