// qr.cu -- blocked Householder QR (compact WY) in FP64.
//
// Replaces LapackQRSolver::SolveThinQR / SolveThinLQ (dgeqrf + dorgqr,
// LapackQRSolver.C:116-160,277-320) and is the gauge step of the sweep's site
// normalisation.  A panel of b columns is factored by one CTA in shared
// memory (column norms by block reduction, reflector application by one warp
// per column); the trailing matrix and the explicit Q are updated with the
// compact WY form I - V T V^T through the FP64 GEMM.  Reflectors follow the
// dlarfg convention (no reflection when the sub-column is already zero), so a
// zero column gives a zero R row and Q still gets an orthonormal column.
#include <algorithm>

#include "qr.h"

namespace tnb {

namespace {

constexpr int QR_THREADS = 512;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = wsum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0;
    if (wid == 0) {
        s = lane < nw ? sh[lane] : 0.0;
        s = wsum(s);
        if (lane == 0) sh[32] = s;
    }
    __syncthreads();
    return sh[32];
}

// Factor the panel W[j0:m, j0:j0+b]; write reflectors V (explicit, mp x b,
// leading dimension ldv), T (b x b, leading dimension ldt) and R's panel part.
__global__ void __launch_bounds__(QR_THREADS) qr_panel_kernel(double* __restrict__ W, int ldw, int m, int j0, int b,
                                                                double* __restrict__ V, int ldv,
                                                                double* __restrict__ T, int ldt) {
    extern __shared__ double smem[];
    const int mp = m - j0;
    double* P = smem;                  // mp x b
    double* G = P + (size_t)mp * b;    // b x b (V^T V)
    double* tau = G + b * b;           // b
    __shared__ double red[33];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    for (int e = tid; e < mp * b; e += blockDim.x) {
        int i = e % mp, c = e / mp;
        P[e] = W[(size_t)(j0 + c) * ldw + j0 + i];
    }
    __syncthreads();
    for (int jj = 0; jj < b; ++jj) {
        double* pc = P + (size_t)jj * mp;
        double part = 0;
        for (int i = jj + 1 + tid; i < mp; i += blockDim.x) part = fma(pc[i], pc[i], part);
        double xn2 = block_sum(part, red);
        double alpha = pc[jj];
        double t = 0, beta = alpha, scal = 0;
        if (xn2 > 0.0) {
            double nrm = sqrt(alpha * alpha + xn2);
            beta = alpha >= 0 ? -nrm : nrm;
            t = (beta - alpha) / beta;
            scal = 1.0 / (alpha - beta);
        }
        __syncthreads();
        if (tid == 0) { tau[jj] = t; pc[jj] = beta; }
        if (t != 0.0)
            for (int i = jj + 1 + tid; i < mp; i += blockDim.x) pc[i] *= scal;
        __syncthreads();
        if (t != 0.0) {
            for (int c = jj + 1 + wid; c < b; c += nw) {
                double* pq = P + (size_t)c * mp;
                double s = 0;
                for (int i = jj + 1 + lane; i < mp; i += 32) s = fma(pc[i], pq[i], s);
                const double top = pq[jj];
                s = (wsum(s) + top) * t;
                __syncwarp();
                if (lane == 0) pq[jj] = top - s;
                for (int i = jj + 1 + lane; i < mp; i += 32) pq[i] = fma(-s, pc[i], pq[i]);
            }
        }
        __syncthreads();
    }
    // explicit V (unit diagonal, zeros above) and the panel back into W
    for (int e = tid; e < mp * b; e += blockDim.x) {
        int i = e % mp, c = e / mp;
        double p = P[e];
        W[(size_t)(j0 + c) * ldw + j0 + i] = p;
        V[(size_t)c * ldv + i] = (i < c) ? 0.0 : (i == c ? 1.0 : p);
    }
    __syncthreads();
    // G = V^T V (upper triangle), one warp per entry
    for (int e = wid; e < b * b; e += nw) {
        int r = e % b, c = e / b;
        if (r >= c) continue;
        double s = 0;
        for (int i = c + lane; i < mp; i += 32) {
            double vr = (i == r) ? 1.0 : (i < r ? 0.0 : P[(size_t)r * mp + i]);
            double vc = (i == c) ? 1.0 : P[(size_t)c * mp + i];
            s = fma(vr, vc, s);
        }
        s = wsum(s);
        if (lane == 0) G[c * b + r] = s;
    }
    __syncthreads();
    // T (dlarft, forward, columnwise): T(jj,jj)=tau_jj, T(0:jj,jj) = -tau_jj T(0:jj,0:jj) G(0:jj,jj).
    // Row i of T depends only on row i, so thread i builds it in shared memory.
    __shared__ double Ts[32 * 32];
    if (tid < b) {
        const int i = tid;
        for (int jj = 0; jj < b; ++jj) {
            double v;
            if (i < jj) {
                double s = 0;
                for (int l = i; l < jj; ++l) s = fma(Ts[l * 32 + i], G[jj * b + l], s);
                v = -tau[jj] * s;
            } else if (i == jj) v = tau[jj];
            else v = 0.0;
            Ts[jj * 32 + i] = v;
        }
    }
    __syncthreads();
    for (int e = tid; e < b * b; e += blockDim.x) {
        int i = e % b, jj = e / b;
        T[(size_t)jj * ldt + i] = Ts[jj * 32 + i];
    }
}

__global__ void set_identity_kernel(double* Q, int m, int k, int ldq) {
    long long total = (long long)m * k;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % m), j = (int)(e / m);
        Q[(size_t)j * ldq + i] = (i == j) ? 1.0 : 0.0;
    }
}

__global__ void extract_r_kernel(const double* W, int ldw, int k, int n, double* R, int ldr) {
    long long total = (long long)k * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % k), j = (int)(e / k);
        R[(size_t)j * ldr + i] = (i <= j) ? W[(size_t)j * ldw + i] : 0.0;
    }
}

inline int g1d(long long n) {
    long long b = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(b, 148 * 8));
}

int panel_width(int m) {
    // keep the panel (m x b doubles) within ~200 KB of shared memory
    const size_t budget = 200 * 1024;
    int b = 32;
    while (b > 1 && (size_t)m * b * 8 + (size_t)b * b * 8 + b * 8 > budget) b >>= 1;
    return b;
}

}  // namespace

int qr_dense(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr) {
    cudaStream_t st = c.stream;
    if (m <= 0 || n <= 0) return TN_BAD_SHAPE;
    const int k = std::min(m, n);
    const int bmax = panel_width(m);
    if ((size_t)m * bmax * 8 > 200 * 1024 || bmax < 1) {
        set_error("qr: matrix too tall (%d rows)", m);
        return TN_BAD_SHAPE;
    }
    TN_CUDA_CHECK(cudaFuncSetAttribute(qr_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    // workspace: Vall (m x k), Tall (bmax x k), Z, Z2 (bmax x n each)
    size_t need = sizeof(double) * ((size_t)m * k + (size_t)bmax * k + 2 * (size_t)bmax * n + 16);
    TN_CHECK(c.qrw.ensure(need));
    double* Vall = c.qrw.as<double>();
    double* Tall = Vall + (size_t)m * k;
    double* Z = Tall + (size_t)bmax * k;
    double* Z2 = Z + (size_t)bmax * n;

    for (int j0 = 0; j0 < k; j0 += bmax) {
        const int b = std::min(bmax, k - j0);
        const int mp = m - j0;
        double* Vp = Vall + (size_t)j0 * m + j0;  // ld m
        double* Tp = Tall + (size_t)j0 * bmax;     // ld bmax
        size_t smem = sizeof(double) * ((size_t)mp * b + (size_t)b * b + b);
        qr_panel_kernel<<<1, QR_THREADS, smem, st>>>(W, m, m, j0, b, Vp, m, Tp, bmax);
        TN_LAUNCH_CHECK();
        const int nt = n - j0 - b;
        if (nt > 0) {
            double* Wt = W + (size_t)(j0 + b) * m + j0;
            GemmArgs g;
            // Z = V^T Wt   (b x nt)
            g.M = b; g.N = nt; g.K = mp;
            g.A.ptr = Vp; g.A.mn = idx(m); g.A.k = idx(1);
            g.B.ptr = Wt; g.B.k = idx(1); g.B.mn = idx(m);
            g.C.ptr = Z; g.C.m = idx(1); g.C.n = idx(b);
            TN_CHECK(gemm_f64(g, st));
            // Z2 = T^T Z
            GemmArgs h;
            h.M = b; h.N = nt; h.K = b;
            h.A.ptr = Tp; h.A.mn = idx(bmax); h.A.k = idx(1);
            h.B.ptr = Z; h.B.k = idx(1); h.B.mn = idx(b);
            h.C.ptr = Z2; h.C.m = idx(1); h.C.n = idx(b);
            TN_CHECK(gemm_f64(h, st));
            // Wt -= V Z2
            GemmArgs u;
            u.M = mp; u.N = nt; u.K = b; u.alpha = -1.0; u.beta = 1.0;
            u.A.ptr = Vp; u.A.mn = idx(1); u.A.k = idx(m);
            u.B.ptr = Z2; u.B.k = idx(1); u.B.mn = idx(b);
            u.C.ptr = Wt; u.C.m = idx(1); u.C.n = idx(m);
            TN_CHECK(gemm_f64(u, st));
        }
    }
    if (Rout) {
        extract_r_kernel<<<g1d((long long)k * n), 256, 0, st>>>(W, m, k, n, Rout, ldr);
        TN_LAUNCH_CHECK();
    }
    if (Qout) {
        set_identity_kernel<<<g1d((long long)m * k), 256, 0, st>>>(Qout, m, k, ldq);
        TN_LAUNCH_CHECK();
        int last = ((k - 1) / bmax) * bmax;
        for (int j0 = last; j0 >= 0; j0 -= bmax) {
            const int b = std::min(bmax, k - j0);
            const int mp = m - j0;
            const int nq = k - j0;
            double* Vp = Vall + (size_t)j0 * m + j0;
            double* Tp = Tall + (size_t)j0 * bmax;
            double* Qs = Qout + (size_t)j0 * ldq + j0;
            GemmArgs g;
            g.M = b; g.N = nq; g.K = mp;
            g.A.ptr = Vp; g.A.mn = idx(m); g.A.k = idx(1);
            g.B.ptr = Qs; g.B.k = idx(1); g.B.mn = idx(ldq);
            g.C.ptr = Z; g.C.m = idx(1); g.C.n = idx(b);
            TN_CHECK(gemm_f64(g, st));
            GemmArgs h;  // Z2 = T Z
            h.M = b; h.N = nq; h.K = b;
            h.A.ptr = Tp; h.A.mn = idx(1); h.A.k = idx(bmax);
            h.B.ptr = Z; h.B.k = idx(1); h.B.mn = idx(b);
            h.C.ptr = Z2; h.C.m = idx(1); h.C.n = idx(b);
            TN_CHECK(gemm_f64(h, st));
            GemmArgs u;
            u.M = mp; u.N = nq; u.K = b; u.alpha = -1.0; u.beta = 1.0;
            u.A.ptr = Vp; u.A.mn = idx(1); u.A.k = idx(m);
            u.B.ptr = Z2; u.B.k = idx(1); u.B.mn = idx(b);
            u.C.ptr = Qs; u.C.m = idx(1); u.C.n = idx(ldq);
            TN_CHECK(gemm_f64(u, st));
        }
    }
    return TN_OK;
}

}  // namespace tnb
