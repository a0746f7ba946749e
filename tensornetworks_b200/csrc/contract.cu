// contract.cu -- FP64 effective-Hamiltonian matvec and environment updates.
//
// Heff x = sum_{w1,w2,n} W(w1,w2)(m,n) F_w1 x_n G_w2^T   (MPSSite::GetHeff,
//   MPSSite_Contractions.C:155-193, applied without forming the dense matrix)
// F'_w2 = sum_{m,n,w1} W(w1,w2)(m,n) A_m^T F_w1 A_n       (IterateLeft_F, :292-345)
// G'_w1 = sum_{m,n,w2} W(w1,w2)(m,n) A_m G_w2 A_n^T       (IterateRightF, :352-400)
// Each is three stages: a batched GEMM, the sparse W combination (memory
// bound, one pass), and a GEMM over the concatenated (w, bond) index.
#include "contract.h"

namespace tnb {

namespace {

__global__ void wcombine_kernel(const double* __restrict__ P, double* __restrict__ Q,
                                const WTermDev* __restrict__ terms, int nterms, long long blk,
                                const int* skip) {
    if (skip && *skip) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < blk;
         e += (long long)gridDim.x * blockDim.x) {
        int cur = terms[0].out;
        double acc = 0.0;
        for (int t = 0; t < nterms; ++t) {
            WTermDev tm = terms[t];
            if (tm.out != cur) {
                Q[(long long)cur * blk + e] = acc;
                acc = 0.0;
                cur = tm.out;
            }
            acc = fma(tm.c, P[(long long)tm.in * blk + e], acc);
        }
        Q[(long long)cur * blk + e] = acc;
    }
}

__global__ void heff_diag_kernel(int d, int Dw1, int Dw2, int D1, int D2, const double* __restrict__ Wd,
                                 const double* __restrict__ F, const double* __restrict__ G,
                                 double* __restrict__ diag) {
    long long N = (long long)d * D1 * D2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N;
         e += (long long)gridDim.x * blockDim.x) {
        int i1 = (int)(e % D1);
        int i2 = (int)((e / D1) % D2);
        int m = (int)(e / ((long long)D1 * D2));
        double v = 0.0;
        for (int w1 = 0; w1 < Dw1; ++w1) {
            double f = F[(long long)w1 * D1 * D1 + (long long)i1 * D1 + i1];
            for (int w2 = 0; w2 < Dw2; ++w2) {
                double w = Wd[(((long long)w1 * Dw2 + w2) * d + m) * d + m];
                if (w != 0.0) v = fma(f * w, G[(long long)w2 * D2 * D2 + (long long)i2 * D2 + i2], v);
            }
        }
        diag[e] = v;
    }
}

__global__ void copy2d_kernel(int rows, int cols, const double* __restrict__ src, IdxMap sr, IdxMap sc,
                              double* __restrict__ dst, IdxMap dr, IdxMap dc, double scale) {
    long long total = (long long)rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int r = (int)(e % rows), c = (int)(e / rows);
        dst[dr.at(r) + dc.at(c)] = scale * src[sr.at(r) + sc.at(c)];
    }
}

// out[e] = sum_s in[s*slab + e]  (deterministic split-K reduction)
__global__ void slab_sum_kernel(const double* __restrict__ in, int nslab, long long slab, double* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < slab;
         e += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nslab; ++q) s += in[(long long)q * slab + e];
        out[e] = s;
    }
}

__global__ void fill_kernel(double* p, long long n, double v) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        p[e] = v;
}

inline int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

// Sort terms by output slab and add zero terms for outputs nothing writes.
std::vector<WTermDev> build_terms(const double* W, int d, int Dw1, int Dw2, bool leftToRight) {
    std::vector<WTermDev> out;
    int Dwin = leftToRight ? Dw1 : Dw2;
    int Dwout = leftToRight ? Dw2 : Dw1;
    for (int m = 0; m < d; ++m)
        for (int wo = 0; wo < Dwout; ++wo) {
            int o = m * Dwout + wo;
            bool any = false;
            for (int wi = 0; wi < Dwin; ++wi)
                for (int n = 0; n < d; ++n) {
                    int w1 = leftToRight ? wi : wo;
                    int w2 = leftToRight ? wo : wi;
                    double c = W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
                    if (c == 0.0) continue;
                    out.push_back({wi * d + n, o, c});
                    any = true;
                }
            if (!any) out.push_back({0, o, 0.0});
        }
    return out;
}

int wcombine(const double* P, double* Q, const WTermDev* terms, int nterms, long long blk,
             const int* skip, cudaStream_t st) {
    if (blk <= 0) return TN_OK;
    wcombine_kernel<<<grid_for(blk), 256, 0, st>>>(P, Q, terms, nterms, blk, skip);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

namespace {

__global__ void gershgorin_kernel(int N, const double* __restrict__ A, int lda, double* sigma) {
    __shared__ double sh[32];
    double mx = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        double r = 0.0;
        for (int j = 0; j < N; ++j) r += fabs(A[(size_t)j * lda + i]);
        mx = fmax(mx, r);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, sh[w]);
        *sigma = 1.001 * t + 1e-300;
    }
}

__global__ void shift_copy_kernel(int N, const double* __restrict__ A, int lda, double* __restrict__ W,
                                  const double* __restrict__ sigma) {
    const double sg = *sigma;
    const long long total = (long long)N * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % N), j = (int)(e / N);
        W[e] = A[(size_t)j * lda + i] + (i == j ? sg : 0.0);
    }
}

}  // namespace

int dense_shift_spd(int N, const double* A, int lda, double* W, double* sigma, cudaStream_t st) {
    gershgorin_kernel<<<1, 256, 0, st>>>(N, A, lda, sigma);
    TN_LAUNCH_CHECK();
    shift_copy_kernel<<<grid_for((long long)N * N), 256, 0, st>>>(N, A, lda, W, sigma);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int copy2d(int rows, int cols, const double* src, IdxMap sr, IdxMap sc, double* dst, IdxMap dr, IdxMap dc,
           double scale, cudaStream_t st) {
    if (rows <= 0 || cols <= 0) return TN_OK;
    copy2d_kernel<<<grid_for((long long)rows * cols), 256, 0, st>>>(rows, cols, src, sr, sc, dst, dr, dc, scale);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

__global__ void slab_sum_skip_kernel(const double* __restrict__ in, int nslab, long long slab, double* __restrict__ out,
                                     const int* skip) {
    if (*skip) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < slab;
         e += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nslab; ++q) s += in[(long long)q * slab + e];
        out[e] = s;
    }
}

int slab_sum_skip(const double* in, int nslab, long long slab, double* out, const int* skip, cudaStream_t st) {
    if (slab <= 0) return TN_OK;
    slab_sum_skip_kernel<<<grid_for(slab), 256, 0, st>>>(in, nslab, slab, out, skip);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int slab_sum(const double* in, int nslab, long long slab, double* out, const int* skip, cudaStream_t st) {
    if (slab <= 0) return TN_OK;
    (void)skip;
    slab_sum_kernel<<<grid_for(slab), 256, 0, st>>>(in, nslab, slab, out);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

__global__ void shift_vector_kernel(double* p, long long n, double v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] += v;
}

int shift_vector(double* p, long long n, double v, cudaStream_t st) {
    if (n <= 0) return TN_OK;
    shift_vector_kernel<<<grid_for(n), 256, 0, st>>>(p, n, v);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int fill(double* p, long long n, double v, cudaStream_t st) {
    if (n <= 0) return TN_OK;
    fill_kernel<<<grid_for(n), 256, 0, st>>>(p, n, v);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int heff_diag(const ContractShape& s, const double* Wdev, const double* F, const double* G, double* diag,
              cudaStream_t st) {
    long long N = (long long)s.d * s.D1 * s.D2;
    heff_diag_kernel<<<grid_for(N), 256, 0, st>>>(s.d, s.Dw1, s.Dw2, s.D1, s.D2, Wdev, F, G, diag);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

// y = Heff x  (FP64).  P, Q: scratch of d*max(Dw1,Dw2)*D1*D2 doubles each.
int heff_matvec_f64(const ContractShape& s, const WTermDev* termsLR, int nLR, const double* F, const double* G,
                    const double* x, double* y, double* P, double* Q, const int* skip, cudaStream_t st) {
    const int d = s.d, Dw1 = s.Dw1, Dw2 = s.Dw2, D1 = s.D1, D2 = s.D2;
    const long long blk = (long long)D1 * D2;
    // Stage 1: P[w1][n] = F_w1 x_n
    GemmArgs g1;
    g1.M = D1; g1.N = D2; g1.K = D1; g1.nb0 = Dw1; g1.nb1 = d;
    g1.A.ptr = F; g1.A.mn = idx(1); g1.A.k = idx(D1); g1.A.sb0 = (long long)D1 * D1; g1.A.sb1 = 0;
    g1.B.ptr = x; g1.B.k = idx(1); g1.B.mn = idx(D1); g1.B.sb0 = 0; g1.B.sb1 = blk;
    g1.C.ptr = P; g1.C.m = idx(1); g1.C.n = idx(D1); g1.C.sb0 = d * blk; g1.C.sb1 = blk;
    g1.skip = skip;
    TN_CHECK(gemm_f64(g1, st));
    // Stage 2: Q[m][w2] = sum W P
    TN_CHECK(wcombine(P, Q, termsLR, nLR, blk, skip, st));
    // Stage 3: y_m = sum_w2 Q[m][w2] G_w2^T, split over w2 for parallelism:
    // partial P[w2][m] = Q[m][w2] G_w2^T (the stage-1 buffer is free again), then a
    // deterministic sum over w2.
    if (Dw2 == 1) {
        GemmArgs g3;
        g3.M = D1; g3.N = D2; g3.K = D2; g3.nb0 = d;
        g3.A.ptr = Q; g3.A.mn = idx(1); g3.A.k = idx(D1); g3.A.sb0 = blk;
        g3.B.ptr = G; g3.B.mn = idx(1); g3.B.k = idx(D2);
        g3.C.ptr = y; g3.C.m = idx(1); g3.C.n = idx(D1); g3.C.sb0 = blk;
        g3.skip = skip;
        return gemm_f64(g3, st);
    }
    GemmArgs g3;
    g3.M = D1; g3.N = D2; g3.K = D2; g3.nb0 = Dw2; g3.nb1 = d;
    g3.A.ptr = Q; g3.A.mn = idx(1); g3.A.k = idx(D1); g3.A.sb0 = blk; g3.A.sb1 = (long long)Dw2 * blk;
    g3.B.ptr = G; g3.B.mn = idx(1); g3.B.k = idx(D2); g3.B.sb0 = (long long)D2 * D2; g3.B.sb1 = 0;
    g3.C.ptr = P; g3.C.m = idx(1); g3.C.n = idx(D1); g3.C.sb0 = (long long)d * blk; g3.C.sb1 = blk;
    g3.skip = skip;
    TN_CHECK(gemm_f64(g3, st));
    if (skip) {
        // the reduction must also honour the skip flag
        return slab_sum_skip(P, Dw2, (long long)d * blk, y, skip, st);
    }
    return slab_sum(P, Dw2, (long long)d * blk, y, nullptr, st);
}

int env_left_f64(const ContractShape& s, const WTermDev* termsLR, int nLR, const double* A, const double* F,
                 double* Fout, double* P, double* Q, cudaStream_t st) {
    const int d = s.d, Dw1 = s.Dw1, Dw2 = s.Dw2, D1 = s.D1, D2 = s.D2;
    const long long blk = (long long)D1 * D2;
    GemmArgs g1;
    g1.M = D1; g1.N = D2; g1.K = D1; g1.nb0 = Dw1; g1.nb1 = d;
    g1.A.ptr = F; g1.A.mn = idx(1); g1.A.k = idx(D1); g1.A.sb0 = (long long)D1 * D1;
    g1.B.ptr = A; g1.B.k = idx(1); g1.B.mn = idx(D1); g1.B.sb1 = blk;
    g1.C.ptr = P; g1.C.m = idx(1); g1.C.n = idx(D1); g1.C.sb0 = d * blk; g1.C.sb1 = blk;
    TN_CHECK(gemm_f64(g1, st));
    TN_CHECK(wcombine(P, Q, termsLR, nLR, blk, nullptr, st));
    // F'_w2(i2,j2) = sum_{m,i1} A_m(i1,i2) Q[m][w2](i1,j2), split over m:
    // partial P[m][w2] = A_m^T Q[m][w2] (D2 x D2), then a sum over m.
    GemmArgs g3;
    g3.M = D2; g3.N = D2; g3.K = D1; g3.nb0 = d; g3.nb1 = Dw2;
    g3.A.ptr = A; g3.A.mn = idx(D1); g3.A.k = idx(1); g3.A.sb0 = blk;
    g3.B.ptr = Q; g3.B.k = idx(1); g3.B.mn = idx(D1); g3.B.sb0 = (long long)Dw2 * blk; g3.B.sb1 = blk;
    const long long out = (long long)Dw2 * D2 * D2;
    if (d == 1) {
        g3.C.ptr = Fout; g3.C.m = idx(1); g3.C.n = idx(D2); g3.C.sb0 = 0; g3.C.sb1 = (long long)D2 * D2;
        return gemm_f64(g3, st);
    }
    g3.C.ptr = P; g3.C.m = idx(1); g3.C.n = idx(D2); g3.C.sb0 = out; g3.C.sb1 = (long long)D2 * D2;
    TN_CHECK(gemm_f64(g3, st));
    return slab_sum(P, d, out, Fout, nullptr, st);
}

int env_right_f64(const ContractShape& s, const WTermDev* termsRL, int nRL, const double* A, const double* G,
                  double* Gout, double* P, double* Q, cudaStream_t st) {
    const int d = s.d, Dw1 = s.Dw1, Dw2 = s.Dw2, D1 = s.D1, D2 = s.D2;
    const long long blk = (long long)D1 * D2;
    // P[w2][n] = G_w2 A_n^T   (D2 x D1, column-major)
    GemmArgs g1;
    g1.M = D2; g1.N = D1; g1.K = D2; g1.nb0 = Dw2; g1.nb1 = d;
    g1.A.ptr = G; g1.A.mn = idx(1); g1.A.k = idx(D2); g1.A.sb0 = (long long)D2 * D2;
    g1.B.ptr = A; g1.B.k = idx(D1); g1.B.mn = idx(1); g1.B.sb1 = blk;
    g1.C.ptr = P; g1.C.m = idx(1); g1.C.n = idx(D2); g1.C.sb0 = d * blk; g1.C.sb1 = blk;
    TN_CHECK(gemm_f64(g1, st));
    TN_CHECK(wcombine(P, Q, termsRL, nRL, blk, nullptr, st));
    // G'_w1(i1,j1) = sum_{m,i2} A_m(i1,i2) Q[m][w1](i2,j1), split over m:
    // partial P[m][w1] = A_m Q[m][w1] (D1 x D1), then a sum over m.
    GemmArgs g3;
    g3.M = D1; g3.N = D1; g3.K = D2; g3.nb0 = d; g3.nb1 = Dw1;
    g3.A.ptr = A; g3.A.mn = idx(1); g3.A.k = idx(D1); g3.A.sb0 = blk;
    g3.B.ptr = Q; g3.B.k = idx(1); g3.B.mn = idx(D2); g3.B.sb0 = (long long)Dw1 * blk; g3.B.sb1 = blk;
    const long long out = (long long)Dw1 * D1 * D1;
    if (d == 1) {
        g3.C.ptr = Gout; g3.C.m = idx(1); g3.C.n = idx(D1); g3.C.sb0 = 0; g3.C.sb1 = (long long)D1 * D1;
        return gemm_f64(g3, st);
    }
    g3.C.ptr = P; g3.C.m = idx(1); g3.C.n = idx(D1); g3.C.sb0 = out; g3.C.sb1 = (long long)D1 * D1;
    TN_CHECK(gemm_f64(g3, st));
    return slab_sum(P, d, out, Gout, nullptr, st);
}

}  // namespace tnb
