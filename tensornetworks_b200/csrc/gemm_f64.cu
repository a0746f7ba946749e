// gemm_f64.cu -- FP64 batched GEMM with split-index addressing (SIMT DFMA).
//
// Used by the plain FP64 sweep for the three contraction stages of the
// effective-Hamiltonian matvec and of the environment updates
// (MPSSite::GetHeff / IterateLeft_F / IterateRightF in the reference,
// MPSSite_Contractions.C:155-400), and for small gauge products.
// Tile 64x64x16, 256 threads, 4x4 outputs per thread, register-staged
// double buffering of the next k-tile.
#include "tn_internal.h"

namespace tnb {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

template <bool A_MCONTIG, bool B_KCONTIG>
__global__ void __launch_bounds__(NT) gemm_f64_kernel(GemmArgs g) {
    if (g.skip && *g.skip) return;
    __shared__ double As[BK][BM + 1];
    __shared__ double Bs[BK][BN + 1];
    const int t = threadIdx.x;
    const int tx = t & 15, ty = t >> 4;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int b = blockIdx.z;
    const int b0 = b / g.nb1, b1 = b - (b / g.nb1) * g.nb1;
    const double* Ab = g.A.ptr + b0 * g.A.sb0 + b1 * g.A.sb1;
    const double* Bb = g.B.ptr + b0 * g.B.sb0 + b1 * g.B.sb1;

    // Per-slot fixed coordinates for the tile loads.
    int am[4], ak[4], bk[4], bn[4];
    long long aoff[4], boff[4];
    bool aok[4], bok[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        int e = t + NT * r;
        if (A_MCONTIG) { am[r] = e % BM; ak[r] = e / BM; }
        else           { ak[r] = e % BK; am[r] = e / BK; }
        if (B_KCONTIG) { bk[r] = e % BK; bn[r] = e / BK; }
        else           { bn[r] = e % BN; bk[r] = e / BN; }
        int gm = m0 + am[r], gn = n0 + bn[r];
        aok[r] = gm < g.M;
        bok[r] = gn < g.N;
        aoff[r] = aok[r] ? g.A.mn.at(gm) : 0;
        boff[r] = bok[r] ? g.B.mn.at(gn) : 0;
    }

    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

    double ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            int gk = k0 + ak[r];
            ra[r] = (aok[r] && gk < g.K) ? __ldg(Ab + aoff[r] + g.A.k.at(gk)) : 0.0;
            int hk = k0 + bk[r];
            rb[r] = (bok[r] && hk < g.K) ? __ldg(Bb + boff[r] + g.B.k.at(hk)) : 0.0;
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            As[ak[r]][am[r]] = ra[r];
            Bs[bk[r]][bn[r]] = rb[r];
        }
    };

    load(0);
    for (int k0 = 0; k0 < g.K; k0 += BK) {
        store();
        __syncthreads();
        if (k0 + BK < g.K) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double a[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }

    double* Cb = g.C.ptr + b0 * g.C.sb0 + b1 * g.C.sb1;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int gm = m0 + ty + 16 * i;
        if (gm >= g.M) continue;
        long long mo = g.C.m.at(gm);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int gn = n0 + tx + 16 * j;
            if (gn >= g.N) continue;
            double* c = Cb + mo + g.C.n.at(gn);
            double v = g.alpha * acc[i][j];
            if (g.beta != 0.0) v += g.beta * *c;
            *c = v;
        }
    }
}

}  // namespace

int gemm_f64(const GemmArgs& g, cudaStream_t st) {
    if (g.M <= 0 || g.N <= 0) return TN_OK;
    if (g.K <= 0) {
        // C = beta*C: express as a K=1 product with a zero operand is wasteful;
        // callers never ask for it.
        set_error("gemm_f64: K must be positive");
        return TN_BAD_ARG;
    }
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, g.nb0 * g.nb1);
    if (grid.y > 65535 || grid.z > 65535) {
        set_error("gemm_f64: grid too large");
        return TN_BAD_SHAPE;
    }
    bool amc = (g.A.mn.s == 1);
    bool bkc = (g.B.k.s == 1);
    if (amc && bkc) gemm_f64_kernel<true, true><<<grid, NT, 0, st>>>(g);
    else if (amc && !bkc) gemm_f64_kernel<true, false><<<grid, NT, 0, st>>>(g);
    else if (!amc && bkc) gemm_f64_kernel<false, true><<<grid, NT, 0, st>>>(g);
    else gemm_f64_kernel<false, false><<<grid, NT, 0, st>>>(g);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

}  // namespace tnb
