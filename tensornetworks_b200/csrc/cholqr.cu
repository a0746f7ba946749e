// cholqr.cu -- Cholesky-QR2 gauge factorisation with a Householder fallback.
//
// The sweep's gauge move needs A = Q R with orthonormal Q for tall site
// matrices (d*D1 x D2, up to 512 x 256 at D = 256).  The Householder QR
// (qr.cu) is bound by its b-column panel steps; Cholesky-QR2 replaces them by
// GEMM-shaped passes:
//     G = A^T A;  R1 = chol(G);  X = A R1^{-1};  G2 = X^T X;  R2 = chol(G2);
//     Q = X R2^{-1};  R = R2 R1
// which is orthonormal to working precision when cond(A) < ~1e7.  The Cholesky
// kernel flags a pivot below 1e-13 * max diag(G) (cond(A) above ~3e6); the
// caller then redoes the factorisation with Householder (rank-deficient
// matrices, such as the zero-padded bonds after a bond-dimension increase,
// always take that path).
#include <algorithm>
#include <cmath>

#include "cholqr.h"
#include "contract.h"
#include "qr.h"

namespace tnb {

namespace {

constexpr int CH_THREADS = 1024;
constexpr int TMAX = 224;   // trailing lower triangle held in shared memory (t(t+1)/2 doubles)
constexpr int PB = 32;      // panel width

__device__ __forceinline__ int poff(int j, int t) { return j * t - (j * (j - 1)) / 2; }  // packed lower, column j

// Single-CTA Cholesky G = L L^T (n x n, column-major, ld n, lower part read).
// Writes R = L^T (upper, ld n, zero below) and the inverses of the 32 x 32
// diagonal blocks of R (Rinv: nb blocks of 32 x 32, column-major).  status = 1
// when a pivot falls below tol * max diag(G).
__global__ void __launch_bounds__(CH_THREADS) chol_kernel(double* __restrict__ G, int n, double tol,
                                                          double* __restrict__ R, double* __restrict__ Rinv,
                                                          int* status) {
    extern __shared__ double sm[];
    __shared__ double s_piv;
    __shared__ int s_fail;
    __shared__ double s_maxd;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    if (tid == 0) {
        s_fail = 0;
        double m = 0;
        for (int i = 0; i < n; ++i) m = fmax(m, G[(size_t)i * n + i]);
        s_maxd = m;
    }
    __syncthreads();
    const double thr = tol * s_maxd;
    int c0 = 0;
    // ---- leading panels from global memory until the trailing triangle fits
    while (n - c0 > TMAX) {
        const int rows = n - c0;
        double* P = sm;  // rows x PB, column-major (ld rows)
        for (int e = tid; e < rows * PB; e += blockDim.x) {
            int i = e % rows, c = e / rows;
            P[e] = G[(size_t)(c0 + c) * n + c0 + i];
        }
        __syncthreads();
        for (int jj = 0; jj < PB; ++jj) {
            if (tid == 0) {
                double dv = P[jj * rows + jj];
                if (!(dv > thr)) s_fail = 1;
                s_piv = sqrt(fmax(dv, thr > 0 ? thr : 1e-300));
            }
            __syncthreads();
            const double r = s_piv;
            for (int i = jj + 1 + tid; i < rows; i += blockDim.x) P[jj * rows + i] /= r;
            if (tid == 0) P[jj * rows + jj] = r;
            __syncthreads();
            for (int k = jj + 1 + wid; k < PB; k += nw) {
                const double lk = P[jj * rows + k];
                for (int i = k + lane; i < rows; i += 32) P[k * rows + i] -= P[jj * rows + i] * lk;
            }
            __syncthreads();
        }
        // L panel -> R^T (row c0+c of R = column of L), trailing update of G in global
        for (int e = tid; e < rows * PB; e += blockDim.x) {
            int i = e % rows, c = e / rows;
            if (i >= c) R[(size_t)(c0 + i) * n + c0 + c] = P[e];
        }
        const int t0 = c0 + PB;
        for (int e = tid; e < (n - t0) * (n - t0); e += blockDim.x) {
            int i = t0 + e % (n - t0), k = t0 + e / (n - t0);
            if (i < k) continue;
            double s = 0;
#pragma unroll 8
            for (int jj = 0; jj < PB; ++jj) s += P[jj * rows + (i - c0)] * P[jj * rows + (k - c0)];
            G[(size_t)k * n + i] -= s;
        }
        __syncthreads();
        c0 += PB;
    }
    // ---- trailing triangle in shared memory, right-looking
    const int t = n - c0;
    double* S = sm;  // packed lower, column-major
    for (int j = 0; j < t; ++j)
        for (int i = j + tid; i < t; i += blockDim.x) S[poff(j, t) + (i - j)] = G[(size_t)(c0 + j) * n + c0 + i];
    __syncthreads();
    for (int j = 0; j < t; ++j) {
        if (tid == 0) {
            double dv = S[poff(j, t)];
            if (!(dv > thr)) s_fail = 1;
            s_piv = sqrt(fmax(dv, thr > 0 ? thr : 1e-300));
        }
        __syncthreads();
        const double r = s_piv;
        const int oj = poff(j, t);
        for (int i = j + 1 + tid; i < t; i += blockDim.x) S[oj + (i - j)] /= r;
        if (tid == 0) S[oj] = r;
        __syncthreads();
        for (int k = j + 1 + wid; k < t; k += nw) {
            const double lk = S[oj + (k - j)];
            const int ok = poff(k, t);
            for (int i = k + lane; i < t; i += 32) S[ok + (i - k)] -= S[oj + (i - j)] * lk;
        }
        __syncthreads();
    }
    for (int j = 0; j < t; ++j)
        for (int i = j + tid; i < t; i += blockDim.x) R[(size_t)(c0 + i) * n + c0 + j] = S[poff(j, t) + (i - j)];
    __syncthreads();
    // zero the strict lower part of R
    for (int e = tid; e < n * n; e += blockDim.x) {
        int i = e % n, j = e / n;
        if (i > j) R[(size_t)j * n + i] = 0.0;
    }
    __syncthreads();
    // inverses of the 32 x 32 diagonal blocks of R (upper): warp per block, lane per column
    const int nb = (n + PB - 1) / PB;
    for (int bk = wid; bk < nb; bk += nw) {
        const int o = bk * PB, bs = min(PB, n - o);
        double* Z = Rinv + (size_t)bk * PB * PB;
        if (lane < PB) {
            // column `lane` of inv(R_bb): solve R_bb z = e_lane by back substitution
            double z[PB];
#pragma unroll
            for (int i = 0; i < PB; ++i) z[i] = 0.0;
            if (lane < bs) {
                for (int i = bs - 1; i >= 0; --i) {
                    double s = (i == lane) ? 1.0 : 0.0;
                    for (int k = i + 1; k < bs; ++k) s -= R[(size_t)(o + k) * n + o + i] * z[k];
                    z[i] = s / R[(size_t)(o + i) * n + o + i];
                }
            }
#pragma unroll
            for (int i = 0; i < PB; ++i) Z[(size_t)lane * PB + i] = (lane < bs && i < bs) ? z[i] : 0.0;
        }
    }
    if (tid == 0 && s_fail) *status = 1;
}

// X = A R^{-1} for tall A (m x n, ld lda), R upper (ld n) with the inverted
// diagonal blocks Rinv.  RB rows per CTA; panel p: X_p = (A_p - X_<p R_<p,p) inv(R_pp).
constexpr int TR_RB = 8;
__global__ void __launch_bounds__(256) trsm_rows_kernel(const double* __restrict__ A, int lda, int m, int n,
                                                        const double* __restrict__ R,
                                                        const double* __restrict__ Rinv, double* __restrict__ X,
                                                        int ldx, const int* status) {
    if (status && *status) return;
    extern __shared__ double xs[];  // TR_RB x n (row-major: xs[r*n + c])
    __shared__ double tmp[TR_RB * PB];
    const int r0 = blockIdx.x * TR_RB;
    const int tid = threadIdx.x;
    const int nb = (n + PB - 1) / PB;
    for (int p = 0; p < nb; ++p) {
        const int o = p * PB, bs = min(PB, n - o);
        // tmp(r, c) = A(r0+r, o+c) - sum_{k<o} X(r, k) R(k, o+c)
        for (int e = tid; e < TR_RB * PB; e += blockDim.x) {
            const int r = e / PB, c = e % PB;
            double s = 0;
            if (r0 + r < m && c < bs) {
                s = A[(size_t)(o + c) * lda + r0 + r];
                const double* Rc = R + (size_t)(o + c) * n;
                for (int k = 0; k < o; ++k) s -= xs[r * n + k] * Rc[k];
            }
            tmp[e] = s;
        }
        __syncthreads();
        // X_p = tmp * inv(R_pp)
        const double* Z = Rinv + (size_t)p * PB * PB;
        for (int e = tid; e < TR_RB * PB; e += blockDim.x) {
            const int r = e / PB, c = e % PB;
            double s = 0;
            if (c < bs)
                for (int k = 0; k <= c; ++k) s += tmp[r * PB + k] * Z[(size_t)c * PB + k];
            if (c < bs) xs[r * n + o + c] = s;
        }
        __syncthreads();
    }
    for (int e = tid; e < TR_RB * n; e += blockDim.x) {
        const int r = e % TR_RB, c = e / TR_RB;
        if (r0 + r < m) X[(size_t)c * ldx + r0 + r] = xs[r * n + c];
    }
}

int gram(Ctx& c, int m, int n, const double* A, double* G, double* part) {
    // G = A^T A, split over row chunks for parallelism, deterministic sum
    int S = 1;
    while (S < 8 && m % (2 * S) == 0 && m / (2 * S) >= 32) S *= 2;
    const int Kc = m / S;
    GemmArgs g;
    g.M = n; g.N = n; g.K = Kc; g.nb0 = S;
    g.A.ptr = A; g.A.mn = idx(m); g.A.k = idx(1); g.A.sb0 = Kc;
    g.B.ptr = A; g.B.k = idx(1); g.B.mn = idx(m); g.B.sb0 = Kc;
    g.C.ptr = S > 1 ? part : G; g.C.m = idx(1); g.C.n = idx(n); g.C.sb0 = (long long)n * n;
    TN_CHECK(gemm_f64(g, c.stream));
    if (S > 1) TN_CHECK(slab_sum(part, S, (long long)n * n, G, nullptr, c.stream));
    return TN_OK;
}

}  // namespace

bool cholqr_supported(int m, int n) { return m >= n && n >= 8 && n <= 512 && m <= 8192; }

int cholqr2_dense(Ctx& c, int m, int n, const double* A, double* Q, int ldq, double* R, int ldr, bool* ok) {
    cudaStream_t st = c.stream;
    *ok = false;
    const int nb = (n + PB - 1) / PB;
    const size_t nn = (size_t)n * n;
    // workspace: G, part(8 nn), R1, R2, Rinv (nb*PB*PB), X (m n), status (2 ints)
    size_t need = sizeof(double) * (nn * 11 + (size_t)nb * PB * PB + (size_t)m * n) + 64;
    TN_CHECK(c.cqr.ensure(need));
    double* G = c.cqr.as<double>();
    double* part = G + nn;
    double* R1 = part + 8 * nn;
    double* R2 = R1 + nn;
    double* Rinv = R2 + nn;
    double* X = Rinv + (size_t)nb * PB * PB;
    int* status = reinterpret_cast<int*>(X + (size_t)m * n);
    TN_CUDA_CHECK(cudaMemsetAsync(status, 0, 2 * sizeof(int), st));
    const int tr = std::min(n, TMAX);
    const size_t chol_smem = sizeof(double) * std::max((size_t)tr * (tr + 1) / 2, (size_t)n * PB);
    TN_CUDA_CHECK(cudaFuncSetAttribute(chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chol_smem));
    const size_t tr_smem = sizeof(double) * (size_t)TR_RB * n;
    TN_CUDA_CHECK(cudaFuncSetAttribute(trsm_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tr_smem));
    const int tgrid = (m + TR_RB - 1) / TR_RB;
    // pass 1
    TN_CHECK(gram(c, m, n, A, G, part));
    chol_kernel<<<1, CH_THREADS, chol_smem, st>>>(G, n, 1e-13, R1, Rinv, status);
    TN_LAUNCH_CHECK();
    trsm_rows_kernel<<<tgrid, 256, tr_smem, st>>>(A, m, m, n, R1, Rinv, X, m, status);
    TN_LAUNCH_CHECK();
    // pass 2
    TN_CHECK(gram(c, m, n, X, G, part));
    chol_kernel<<<1, CH_THREADS, chol_smem, st>>>(G, n, 1e-13, R2, Rinv, status + 1);
    TN_LAUNCH_CHECK();
    trsm_rows_kernel<<<tgrid, 256, tr_smem, st>>>(X, m, m, n, R2, Rinv, Q, ldq, status + 1);
    TN_LAUNCH_CHECK();
    // R = R2 R1
    GemmArgs g;
    g.M = n; g.N = n; g.K = n;
    g.A.ptr = R2; g.A.mn = idx(1); g.A.k = idx(n);
    g.B.ptr = R1; g.B.k = idx(1); g.B.mn = idx(n);
    g.C.ptr = R; g.C.m = idx(1); g.C.n = idx(ldr);
    TN_CHECK(gemm_f64(g, st));
    int hs[2] = {0, 0};
    TN_CUDA_CHECK(cudaMemcpyAsync(hs, status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    *ok = (hs[0] == 0 && hs[1] == 0);
    return TN_OK;
}

}  // namespace tnb
