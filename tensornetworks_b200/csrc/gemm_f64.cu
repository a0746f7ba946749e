// gemm_f64.cu -- FP64 batched GEMM with split-index addressing (SIMT DFMA).
//
// Used by the plain FP64 sweep for the three contraction stages of the
// effective-Hamiltonian matvec and of the environment updates
// (MPSSite::GetHeff / IterateLeft_F / IterateRightF in the reference,
// MPSSite_Contractions.C:155-400), and for small gauge products.
// Plain strided operands take the FP64 tensor-core (DMMA) kernel below;
// split-index operands the SIMT kernel: tile 64x64x16, 256 threads, 4x4
// outputs per thread, register-staged double buffering of the next k-tile.
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

// ---------------------------------------------------------------------------
// FP64 tensor-core path: mma.sync m8n8k4 (DMMA), for operands whose index maps
// are plain strides over the ranges used (no split indices).  CTA tile 64x64,
// 4 warps each owning a 32x32 quarter (4x4 MMA tiles, 32 accumulators per
// thread), k-tiles of 16 staged in shared memory with the next tile
// prefetched into registers.  The shared row stride 68 (= 4 mod 16 doubles)
// makes the fragment loads of a half-warp hit 16 distinct bank pairs.
constexpr int TBM = 64, TBN = 64, TBK = 16, TNT = 128, TLD = TBM + 4;

struct LinGemm {
    int M, N, K, nb1;
    long long sAm, sAk, sBk, sBn, sCm, sCn;
    long long sA0, sA1, sB0, sB1, sC0, sC1;
    const double *A, *B;
    double* C;
    double alpha, beta;
    const int* skip;
};

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// WM: rows of a warp's tile (32: CTA tile 64 x 64; 16: 32 x 64, twice the
// CTAs for grids that would leave SMs idle or run one latency-bound CTA each).
template <int WM, bool A_MCONTIG, bool B_KCONTIG>
__global__ void __launch_bounds__(TNT) gemm_f64_dmma_kernel(LinGemm g) {
    constexpr int BMT = 2 * WM, LDA = BMT + 4, RA = BMT * TBK / TNT, MI = WM / 8;
    if (g.skip && *g.skip) return;
    __shared__ double As[TBK][LDA];
    __shared__ double Bs[TBK][TLD];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int wm = (warp >> 1) * WM, wn = (warp & 1) * 32;
    const int m0 = blockIdx.y * BMT, n0 = blockIdx.x * TBN;
    const int b = blockIdx.z;
    const int b0 = b / g.nb1, b1 = b - b0 * g.nb1;
    const double* Ab = g.A + b0 * g.sA0 + b1 * g.sA1;
    const double* Bb = g.B + b0 * g.sB0 + b1 * g.sB1;
    // tile slots: RA per thread for A (TBK x BMT), 8 for B (TBK x TBN)
    double ra[RA], rb[8];
    auto load = [&](int k0) {
#pragma unroll
        for (int r = 0; r < RA; ++r) {
            const int e = t + TNT * r;
            int am, ak;
            if (A_MCONTIG) { am = e % BMT; ak = e / BMT; } else { ak = e % TBK; am = e / TBK; }
            const int gm = m0 + am, gk = k0 + ak;
            ra[r] = (gm < g.M && gk < g.K) ? __ldg(Ab + gm * g.sAm + gk * g.sAk) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int e = t + TNT * r;
            int bk, bn;
            if (B_KCONTIG) { bk = e % TBK; bn = e / TBK; } else { bn = e % TBN; bk = e / TBN; }
            const int hk = k0 + bk, gn = n0 + bn;
            rb[r] = (gn < g.N && hk < g.K) ? __ldg(Bb + hk * g.sBk + gn * g.sBn) : 0.0;
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int r = 0; r < RA; ++r) {
            const int e = t + TNT * r;
            int am, ak;
            if (A_MCONTIG) { am = e % BMT; ak = e / BMT; } else { ak = e % TBK; am = e / TBK; }
            As[ak][am] = ra[r];
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int e = t + TNT * r;
            int bk, bn;
            if (B_KCONTIG) { bk = e % TBK; bn = e / TBK; } else { bn = e % TBN; bk = e / TBN; }
            Bs[bk][bn] = rb[r];
        }
    };
    double acc[MI][4][2];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    load(0);
    for (int k0 = 0; k0 < g.K; k0 += TBK) {
        store();
        __syncthreads();
        if (k0 + TBK < g.K) load(k0 + TBK);
#pragma unroll
        for (int ks = 0; ks < TBK; ks += 4) {
            double af[MI], bf[4];
#pragma unroll
            for (int i = 0; i < MI; ++i) af[i] = As[ks + tig][wm + i * 8 + gid];  // A(row gid, col tig)
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = Bs[ks + tig][wn + j * 8 + gid];  // B(row tig, col gid)
#pragma unroll
            for (int i = 0; i < MI; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();
    }
    double* Cb = g.C + b0 * g.sC0 + b1 * g.sC1;
#pragma unroll
    for (int i = 0; i < MI; ++i) {
        const int gm = m0 + wm + i * 8 + gid;
        if (gm >= g.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int gn = n0 + wn + j * 8 + tig * 2 + q;
                if (gn >= g.N) continue;
                double* c = Cb + gm * g.sCm + gn * g.sCn;
                double v = g.alpha * acc[i][j][q];
                if (g.beta != 0.0) v += g.beta * *c;
                *c = v;
            }
    }
}

// An index map that is a plain stride over [0, n).
inline bool plain(const IdxMap& m, int n) { return m.div >= n; }

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
    if (plain(g.A.mn, g.M) && plain(g.A.k, g.K) && plain(g.B.k, g.K) && plain(g.B.mn, g.N) && plain(g.C.m, g.M) &&
        plain(g.C.n, g.N)) {
        LinGemm l;
        l.M = g.M; l.N = g.N; l.K = g.K; l.nb1 = g.nb1;
        l.sAm = g.A.mn.s; l.sAk = g.A.k.s; l.sBk = g.B.k.s; l.sBn = g.B.mn.s; l.sCm = g.C.m.s; l.sCn = g.C.n.s;
        l.sA0 = g.A.sb0; l.sA1 = g.A.sb1; l.sB0 = g.B.sb0; l.sB1 = g.B.sb1; l.sC0 = g.C.sb0; l.sC1 = g.C.sb1;
        l.A = g.A.ptr; l.B = g.B.ptr; l.C = g.C.ptr; l.alpha = g.alpha; l.beta = g.beta; l.skip = g.skip;
        // 64 x 64 CTA tiles, or 32 x 64 when that grid would not fill two CTAs per SM
        static int sms = 0;
        if (sms == 0) {
            int dev = 0;
            cudaGetDevice(&dev);
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
        }
        const long long tiles64 = (long long)((g.N + TBN - 1) / TBN) * ((g.M + TBM - 1) / TBM) * g.nb0 * g.nb1;
        if (tiles64 < 2LL * sms) {
            dim3 tg((g.N + TBN - 1) / TBN, (g.M + 31) / 32, g.nb0 * g.nb1);
            if (amc && bkc) gemm_f64_dmma_kernel<16, true, true><<<tg, TNT, 0, st>>>(l);
            else if (amc && !bkc) gemm_f64_dmma_kernel<16, true, false><<<tg, TNT, 0, st>>>(l);
            else if (!amc && bkc) gemm_f64_dmma_kernel<16, false, true><<<tg, TNT, 0, st>>>(l);
            else gemm_f64_dmma_kernel<16, false, false><<<tg, TNT, 0, st>>>(l);
        } else {
            dim3 tg((g.N + TBN - 1) / TBN, (g.M + TBM - 1) / TBM, g.nb0 * g.nb1);
            if (amc && bkc) gemm_f64_dmma_kernel<32, true, true><<<tg, TNT, 0, st>>>(l);
            else if (amc && !bkc) gemm_f64_dmma_kernel<32, true, false><<<tg, TNT, 0, st>>>(l);
            else if (!amc && bkc) gemm_f64_dmma_kernel<32, false, true><<<tg, TNT, 0, st>>>(l);
            else gemm_f64_dmma_kernel<32, false, false><<<tg, TNT, 0, st>>>(l);
        }
        TN_LAUNCH_CHECK();
        return TN_OK;
    }
    if (amc && bkc) gemm_f64_kernel<true, true><<<grid, NT, 0, st>>>(g);
    else if (amc && !bkc) gemm_f64_kernel<true, false><<<grid, NT, 0, st>>>(g);
    else if (!amc && bkc) gemm_f64_kernel<false, true><<<grid, NT, 0, st>>>(g);
    else gemm_f64_kernel<false, false><<<grid, NT, 0, st>>>(g);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

}  // namespace tnb
