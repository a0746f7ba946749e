// qr.cu -- blocked Householder QR (compact WY) in FP64.
//
// Replaces LapackQRSolver::SolveThinQR / SolveThinLQ (dgeqrf + dorgqr,
// LapackQRSolver.C:116-160,277-320) and is the gauge step of the sweep's site
// normalisation.  One path per row range: m <= 512, 32-column panels by the
// warp-column panel (panel_wc) inside the persistent cooperative kernel (or,
// when that cannot launch, the two-stream look-ahead); 512 < m <= 1536,
// 16-column panels (qr_panel_tall_kernel) with block-reflector updates on the
// FP64 tensor cores (wy_cols_kernel); m > 1536, a shared-memory panel
// (qr_panel_kernel) with FP64-GEMM updates.  The trailing matrix and the
// explicit Q are updated with the compact WY form I - V T V^T.  Reflectors
// follow the dlarfg convention (no reflection when the sub-column is already
// zero), so a zero column gives a zero R row and Q still gets an orthonormal
// column.
#include <algorithm>

#include "qr.h"

#include <cooperative_groups.h>

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

// Asynchronous 8-byte global -> shared copies (all in flight until the wait).
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Warp-column panel (B = 32 columns, mp <= 32 RPL rows, 512 threads).
// Warp w owns panel columns 2w, 2w+1 whole: lane l holds rows l + 32 q
// (q < RPL) of its two columns in registers, so every column sum is a warp
// reduction (shuffles, no shared memory) and the only block barrier of a step
// hands the next reflector to the other warps.  Step j: the warp owning column
// j has published its rows below j (u_j, the unscaled reflector; zero at rows
// <= j) and its row j (alpha) in shared memory; every warp reads u_j, forms
// S_c = u_j . p_c for its two columns and |u_j|^2 (the same butterfly in every
// warp, so every lane of every warp holds the same sums and the same dlarfg
// values), then for c > j applies the reflector,
//     v_j^T p_c = p_c[j] + scal_j S_c,   p_c -= tau_j (v_j^T p_c) v_j,
// and for c < j (a finished column, which still holds u_c below its
// diagonal) records the Gram entry v_c^T v_j = scal_c (u_c[j] + scal_j S_c) of
// the T build.  The column-ownership test is warp-uniform, so finished
// columns cost no update.  The warp owning column j+1 then publishes it (it
// has just applied reflector j to it) into the other parity's buffer, and one
// barrier ends the step.  Reflectors follow dlarfg (no reflection when the
// sub-column is zero).  The panel comes from global memory by L2 loads
// (ld.global.cg): in the persistent QR other CTAs write these columns during
// the same launch.
constexpr int PWC_MAXR = 512;   // rows of the warp-column panel
constexpr int PWC_WARPS = 16;   // two columns per warp: four warps per scheduler hide the step's latencies
constexpr int PWC_THREADS = 32 * PWC_WARPS;
struct PanelWcSmem {
    double ub[2][PWC_MAXR];  // u_j by step parity
    double alph[2];          // row j of column j
    double Gs[32][33];       // Gs[l][jj] = v_l^T v_jj, l < jj
    double taus[32], scals[32], betas[32];
    double Tsm[32][33];      // T(i, jj)
    double Xs[32][33];       // products of the blocked T build
};

// T of the compact WY form from the reflectors' taus and Gram entries, by the
// whole block (at least 128 threads).
__device__ void build_t(const double (&Gs)[32][33], const double* taus, double (&Tsm)[32][33], double (&Xs)[32][33],
                        int b, double* __restrict__ T, int ldt) {
    constexpr int B = 32;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // T (dlarft, forward, columnwise) blockwise.  For reflectors split into two
    // groups, I - V T V^T = (I - V1 T11 V1^T)(I - V2 T22 V2^T) gives
    // T = [T11, -T11 (V1^T V2) T22; 0, T22]: the four 8 x 8 diagonal blocks by
    // the recurrence T(i, jj) = -tau_jj sum_{l=i}^{jj-1} T(i, l) G(l, jj) (one
    // warp each, lane i builds row i), then the off-diagonal blocks at widths 8
    // and 16 as small products over the whole block.  Columns past b have
    // tau = 0 and zero Gram entries, so they come out zero.
    for (int e = tid; e < B * (B + 1); e += (int)blockDim.x) (&Tsm[0][0])[e] = 0.0;
    __syncthreads();
    if (w < 4 && lane < 8) {
        const int q0 = 8 * w, i = lane;
        double trow[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            double a = 0;
#pragma unroll
            for (int l = 0; l < jj; ++l)
                if (l >= i) a = fma(trow[l], Gs[q0 + l][q0 + jj], a);
            const double tj = q0 + jj < b ? taus[q0 + jj] : 0.0;
            trow[jj] = (jj < i) ? 0.0 : (jj == i ? tj : -tj * a);
        }
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) Tsm[q0 + i][q0 + jj] = trow[jj];
    }
    __syncthreads();
#pragma unroll
    for (int h = 8; h < B; h *= 2) {
        // pairs of h x h blocks at r0 = 0, 2h, ...: X = G12 T22, then T12 = -T11 X
        const int npair = B / (2 * h);
        for (int e = tid; e < npair * h * h; e += (int)blockDim.x) {
            const int pr = e / (h * h), a = (e / h) % h, c = e % h, r0 = 2 * h * pr;
            double xx = 0;
            for (int k = 0; k <= c; ++k) xx = fma(Gs[r0 + a][r0 + h + k], Tsm[r0 + h + k][r0 + h + c], xx);
            Xs[r0 + a][r0 + h + c] = xx;
        }
        __syncthreads();
        for (int e = tid; e < npair * h * h; e += (int)blockDim.x) {
            const int pr = e / (h * h), a = (e / h) % h, c = e % h, r0 = 2 * h * pr;
            double t = 0;
            for (int k = a; k < h; ++k) t = fma(Tsm[r0 + a][r0 + k], Xs[r0 + k][r0 + h + c], t);
            Tsm[r0 + a][r0 + h + c] = -t;
        }
        __syncthreads();
    }
    for (int e = tid; e < b * b; e += (int)blockDim.x) {
        const int i = e % b, jj = e / b;
        T[(size_t)jj * ldt + i] = Tsm[i][jj];
    }
}

template <int RPL>
__device__ __forceinline__ void panel_wc(double* __restrict__ W, int ldw, int m, int j0, int b,
                                         double* __restrict__ V, int ldv, double* __restrict__ T, int ldt,
                                         PanelWcSmem& sm) {
    constexpr int B = 32, CPW = 32 / PWC_WARPS;  // columns per warp
    static_assert(32 * RPL <= PWC_MAXR && CPW * PWC_WARPS == B, "panel shape");
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int mp = m - j0;
    for (int e = tid; e < B * (B + 1); e += PWC_THREADS) (&sm.Gs[0][0])[e] = 0.0;  // entries past b stay zero
    double p[CPW][RPL];
#pragma unroll
    for (int ci = 0; ci < CPW; ++ci) {
        const int c = CPW * w + ci;
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int ri = lane + 32 * q;
            p[ci][q] = (c < b && ri < mp) ? __ldcg(W + (size_t)(j0 + c) * ldw + j0 + ri) : 0.0;
        }
    }
    // column c (slot c % CPW of warp c / CPW) into the step buffer `par`
    auto publish = [&](int c, int par) {
        const int ci = c % CPW;
#pragma unroll
        for (int cc = 0; cc < CPW; ++cc) {
            if (cc != ci) continue;
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                const int ri = lane + 32 * q;
                sm.ub[par][ri] = ri > c ? p[cc][q] : 0.0;
            }
            if (lane == c) sm.alph[par] = p[cc][0];
        }
    };
    if (w == 0) publish(0, 0);
    __syncthreads();
#pragma unroll 1
    for (int j = 0; j < b; ++j) {
        const int par = j & 1;
        double u[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) u[q] = sm.ub[par][lane + 32 * q];
        const double alpha = sm.alph[par];
        double x[CPW + 1];
#pragma unroll
        for (int ci = 0; ci < CPW; ++ci) {
            double a0 = 0, a1 = 0;
#pragma unroll
            for (int q = 0; q < RPL; q += 2) {
                a0 = fma(u[q], p[ci][q], a0);
                if (q + 1 < RPL) a1 = fma(u[q + 1], p[ci][q + 1], a1);
            }
            x[ci] = a0 + a1;
        }
        {
            double a0 = 0, a1 = 0;
#pragma unroll
            for (int q = 0; q < RPL; q += 2) {
                a0 = fma(u[q], u[q], a0);
                if (q + 1 < RPL) a1 = fma(u[q + 1], u[q + 1], a1);
            }
            x[CPW] = a0 + a1;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int v = 0; v <= CPW; ++v) x[v] += __shfl_xor_sync(0xffffffffu, x[v], o);
        }
        const double xn2 = x[CPW];
        double tau = 0, beta = alpha, scal = 1;
        if (xn2 > 0.0) {
            const double nrm = sqrt(alpha * alpha + xn2);
            beta = alpha >= 0 ? -nrm : nrm;
            const double amb = alpha - beta;
            const double rinv = 1.0 / (beta * amb);  // tau = -amb / beta, scal = 1 / amb
            tau = -amb * amb * rinv;
            scal = beta * rinv;
        }
#pragma unroll
        for (int ci = 0; ci < CPW; ++ci) {
            const int c = CPW * w + ci;
            const double pj = __shfl_sync(0xffffffffu, p[ci][0], j);  // row j of column c
            const double g = fma(scal, x[ci], pj);                   // v_j^T p_c
            if (c > j && c < b) {
                if (tau != 0.0) {
                    const double t = tau * g, cu = t * scal;
#pragma unroll
                    for (int q = 0; q < RPL; ++q) p[ci][q] = fma(-cu, u[q], p[ci][q]);
                    if (lane == j) p[ci][0] -= t;
                }
            } else if (c < j && lane == 0) {
                sm.Gs[c][j] = sm.scals[c] * g;
            }
        }
        if (w == j / CPW && lane == 0) {
            sm.taus[j] = tau;
            sm.scals[j] = scal;
            sm.betas[j] = beta;
        }
        if (j + 1 < b && w == (j + 1) / CPW) publish(j + 1, par ^ 1);
        __syncthreads();
    }
    // the factored panel: R above and on the diagonal, v below it
#pragma unroll
    for (int ci = 0; ci < CPW; ++ci) {
        const int c = CPW * w + ci;
        if (c < b) {
            const double sc = sm.scals[c], be = sm.betas[c];
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
                const int ri = lane + 32 * q;
                if (ri < mp) {
                    const double val = ri < c ? p[ci][q] : (ri == c ? be : sc * p[ci][q]);
                    W[(size_t)(j0 + c) * ldw + j0 + ri] = val;
                    if (V) V[(size_t)c * ldv + ri] = ri < c ? 0.0 : (ri == c ? 1.0 : val);
                }
            }
        }
    }
    build_t(sm.Gs, sm.taus, sm.Tsm, sm.Xs, b, T, ldt);
}

// the panel by rows per lane
__device__ __forceinline__ void panel_wc_any(double* W, int ldw, int m, int j0, int b, double* V, int ldv, double* T,
                                             int ldt, PanelWcSmem& sm) {
    const int mp = m - j0;
    if (mp <= 64) panel_wc<2>(W, ldw, m, j0, b, V, ldv, T, ldt, sm);
    else if (mp <= 128) panel_wc<4>(W, ldw, m, j0, b, V, ldv, T, ldt, sm);
    else if (mp <= 256) panel_wc<8>(W, ldw, m, j0, b, V, ldv, T, ldt, sm);
    else panel_wc<16>(W, ldw, m, j0, b, V, ldv, T, ldt, sm);
}

__global__ void __launch_bounds__(PWC_THREADS) qr_panel_wc_kernel(double* __restrict__ W, int ldw, int m, int j0, int b,
                                                         double* __restrict__ V, int ldv, double* __restrict__ T,
                                                         int ldt) {
    __shared__ PanelWcSmem sm;
    panel_wc_any(W, ldw, m, j0, b, V, ldv, T, ldt, sm);
}

// Panel launch of the look-ahead and single-stream paths (m <= 512, 32-wide
// panels): the warp-column kernel.
template <int NT, int R, int B, int U>
void launch_panel(cudaStream_t st, double* W, int ldw, int m, int j0, int b, double* V, int ldv, double* T, int ldt) {
    static_assert(B == 32, "the warp-column panel is 32 columns wide");
    qr_panel_wc_kernel<<<1, PWC_THREADS, 0, st>>>(W, ldw, m, j0, b, V, ldv, T, ldt);
}

// C (mp x nc, ld ldc) <- (I - V T' V^T) C with T' = T^T (TRANS: applying Q^T,
// the trailing update) or T (forming Q).  V is mp x b (ld ldv, unit lower
// trapezoidal; only the entries below the diagonal are read, so V may be the
// factored panel itself), T is b x b upper triangular (ld ldt), b <= B.
// One CTA per 8 columns of C.  The whole of V and the CTA's columns of C are
// staged in shared memory by asynchronous copies (all in flight at once; the
// kernel is latency bound otherwise), then Z = V^T C, Z2 = T' Z, C -= V Z2.
// Shared layout: column-major with the odd stride mp + 1, so that both the
// lane-per-column reads of the Z reduction and the lane-per-row reads of the
// update are free of bank conflicts.
constexpr int WY_COLS = 8;
constexpr int WY_THREADS = 256;

inline size_t wy_smem_bytes(int mp, int B) { return sizeof(double) * (size_t)(mp + 1) * (B + WY_COLS); }


template <int B, bool TRANS>
__global__ void __launch_bounds__(WY_THREADS) wy_apply_kernel(const double* __restrict__ V, int ldv,
                                                              const double* __restrict__ T, int ldt, int b,
                                                              double* __restrict__ C, int ldc, int mp, int nc,
                                                              double* __restrict__ C2 = nullptr, int ldc2 = 0,
                                                              int nc2 = 0) {
    constexpr int NPART = WY_THREADS / (B * WY_COLS);  // row partitions of the Z reduction
    extern __shared__ double wsm[];
    const int ld = mp + 1;
    double* Vs = wsm;                  // B columns of length ld
    double* Cs = Vs + (size_t)ld * B;  // WY_COLS columns of length ld
    __shared__ double Zp[NPART][B][WY_COLS];
    __shared__ double Z2[B][WY_COLS];
    __shared__ double Ts[B][B + 1];  // Ts[c][r] = T(r, c)
    const int tid = threadIdx.x;
    // blocks past the first target's columns work on the second target (same V, T)
    int blk = blockIdx.x;
    const int nblk1 = (nc + WY_COLS - 1) / WY_COLS;
    if (blk >= nblk1) {
        blk -= nblk1;
        C = C2;
        ldc = ldc2;
        nc = nc2;
    }
    const int c0 = blk * WY_COLS;
    const int ncol = min(WY_COLS, nc - c0);
    for (int e = tid; e < mp * B; e += WY_THREADS) {
        const int r = e % mp, col = e / mp;
        if (col < b && r > col) cp_async8(Vs + (size_t)col * ld + r, V + (size_t)col * ldv + r);
        else Vs[(size_t)col * ld + r] = (col < b && r == col) ? 1.0 : 0.0;
    }
    for (int e = tid; e < mp * WY_COLS; e += WY_THREADS) {
        const int r = e % mp, col = e / mp;
        if (col < ncol) cp_async8(Cs + (size_t)col * ld + r, C + (size_t)(c0 + col) * ldc + r);
        else Cs[(size_t)col * ld + r] = 0.0;
    }
    for (int e = tid; e < B * B; e += WY_THREADS) {
        const int r = e % B, col = e / B;
        if (r < b && col < b) cp_async8(&Ts[col][r], T + (size_t)col * ldt + r);
        else Ts[col][r] = 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    {
        const int bb = tid % B, cc = (tid / B) % WY_COLS, part = tid / (B * WY_COLS);
        const double* vcol = Vs + (size_t)bb * ld;
        const double* ccol = Cs + (size_t)cc * ld;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        int r = part;
        for (; r + 3 * NPART < mp; r += 4 * NPART) {
            a0 = fma(vcol[r], ccol[r], a0);
            a1 = fma(vcol[r + NPART], ccol[r + NPART], a1);
            a2 = fma(vcol[r + 2 * NPART], ccol[r + 2 * NPART], a2);
            a3 = fma(vcol[r + 3 * NPART], ccol[r + 3 * NPART], a3);
        }
        for (; r < mp; r += NPART) a0 = fma(vcol[r], ccol[r], a0);
        Zp[part][bb][cc] = (a0 + a1) + (a2 + a3);
    }
    __syncthreads();
    if (tid < B * WY_COLS) {
        const int bb = tid % B, cc = tid / B;
        double s = 0;
        if (bb < b) {
            if (TRANS) {
                for (int l = 0; l <= bb; ++l) {
                    double z = 0;
#pragma unroll
                    for (int pp = 0; pp < NPART; ++pp) z += Zp[pp][l][cc];
                    s = fma(Ts[bb][l], z, s);
                }
            } else {
                for (int l = bb; l < b; ++l) {
                    double z = 0;
#pragma unroll
                    for (int pp = 0; pp < NPART; ++pp) z += Zp[pp][l][cc];
                    s = fma(Ts[l][bb], z, s);
                }
            }
        }
        Z2[bb][cc] = s;
    }
    __syncthreads();
    for (int r = tid; r < mp; r += WY_THREADS) {
        double acc[WY_COLS];
#pragma unroll
        for (int q = 0; q < WY_COLS; ++q) acc[q] = Cs[(size_t)q * ld + r];
#pragma unroll 4
        for (int l = 0; l < B; ++l) {
            const double vl = Vs[(size_t)l * ld + r];
#pragma unroll
            for (int q = 0; q < WY_COLS; ++q) acc[q] = fma(-vl, Z2[l][q], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < WY_COLS; ++q)
            if (q < ncol) C[(size_t)(c0 + q) * ldc + r] = acc[q];
    }
}

// Narrow trailing update, C (mp x nc) <- (I - V T^T V^T) C, for a few columns
// on the critical path.  The rows are split over a cluster of four CTAs (each
// stages only its quarter of V and C); each CTA forms its partial Z = V^T C
// (B x 8), the cluster adds the four partials through distributed shared
// memory, and each CTA applies Z2 = T^T Z to its own rows.
constexpr int WYN_RANKS = 4;
template <int B>
__global__ void __cluster_dims__(1, WYN_RANKS, 1) __launch_bounds__(256)
    wy_narrow_kernel(const double* __restrict__ V, int ldv, const double* __restrict__ T, int ldt, int b,
                     double* __restrict__ C, int ldc, int mp, int nc) {
    constexpr int NC = WY_COLS;
    static_assert(B * NC == 256, "one thread per entry of Z");
    extern __shared__ double wsm[];
    __shared__ double Zp[B][NC];  // this CTA's partial V^T C
    __shared__ double Zs[B][NC];
    __shared__ double Z2[B][NC];
    __shared__ double Ts[B][B + 1];  // Ts[c][r] = T(r, c)
    namespace cgx = cooperative_groups;
    cgx::cluster_group cluster = cgx::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int tid = threadIdx.x;
    const int rb = (mp + WYN_RANKS - 1) / WYN_RANKS;
    const int r0 = rank * rb, nr = max(0, min(rb, mp - r0));
    const int ld = rb + 1;
    double* Vs = wsm;
    double* Cs = Vs + (size_t)ld * B;
    const int c0 = blockIdx.x * NC, ncol = min(NC, nc - c0);
    for (int e = tid; e < nr * B; e += 256) {
        const int r = e % nr, col = e / nr;
        if (col < b && r0 + r > col) cp_async8(Vs + (size_t)col * ld + r, V + (size_t)col * ldv + r0 + r);
        else Vs[(size_t)col * ld + r] = (col < b && r0 + r == col) ? 1.0 : 0.0;
    }
    for (int e = tid; e < nr * NC; e += 256) {
        const int r = e % nr, col = e / nr;
        if (col < ncol) cp_async8(Cs + (size_t)col * ld + r, C + (size_t)(c0 + col) * ldc + r0 + r);
        else Cs[(size_t)col * ld + r] = 0.0;
    }
    for (int e = tid; e < B * B; e += 256) {
        const int r = e % B, col = e / B;
        if (r < b && col < b) cp_async8(&Ts[col][r], T + (size_t)col * ldt + r);
        else Ts[col][r] = 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    {
        const int l = tid % B, q = tid / B;
        const double* vcol = Vs + (size_t)l * ld;
        const double* ccol = Cs + (size_t)q * ld;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        int r = 0;
        for (; r + 3 < nr; r += 4) {
            a0 = fma(vcol[r], ccol[r], a0);
            a1 = fma(vcol[r + 1], ccol[r + 1], a1);
            a2 = fma(vcol[r + 2], ccol[r + 2], a2);
            a3 = fma(vcol[r + 3], ccol[r + 3], a3);
        }
        for (; r < nr; ++r) a0 = fma(vcol[r], ccol[r], a0);
        Zp[l][q] = (a0 + a1) + (a2 + a3);
    }
    cluster.sync();
    {
        const int l = tid % B, q = tid / B;
        double z = 0;
#pragma unroll
        for (int k = 0; k < WYN_RANKS; ++k) z += cluster.map_shared_rank(&Zp[0][0], k)[l * NC + q];
        Zs[l][q] = z;
    }
    cluster.sync();  // every rank has read the partials; they may go away now
    {
        const int bb = tid % B, q = tid / B;
        double s = 0;
        if (bb < b)
            for (int l = 0; l <= bb; ++l) s = fma(Ts[bb][l], Zs[l][q], s);
        Z2[bb][q] = s;
    }
    __syncthreads();
    for (int r = tid; r < nr; r += 256) {
        double acc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) acc[q] = Cs[(size_t)q * ld + r];
#pragma unroll 4
        for (int l = 0; l < B; ++l) {
            const double vl = Vs[(size_t)l * ld + r];
#pragma unroll
            for (int q = 0; q < NC; ++q) acc[q] = fma(-vl, Z2[l][q], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (q < ncol) C[(size_t)(c0 + q) * ldc + r0 + r] = acc[q];
    }
}

inline size_t wyn_smem_bytes(int mp, int B) {
    const int rb = (mp + WYN_RANKS - 1) / WYN_RANKS;
    return sizeof(double) * (size_t)(rb + 1) * (B + WY_COLS);
}

// ---------------------------------------------------------------------------
// Persistent blocked QR (m <= 512, 32-wide panels): one cooperative launch.
// CTA 0 factors the panels in order; every other CTA takes trailing-update
// tasks -- one 2-column block of W or 8-column block of Qt (= Q^T,
// accumulated as in the look-ahead path) under one block reflector -- from a
// global counter, in the
// order reflector by reflector and, within a reflector, W's blocks from the left
// (so the next panel's columns come first), then Qt's.  Progress is tracked in
// global memory: refready = panels factored, applied[block] = reflectors
// applied to that block.  A task for reflector kk waits for refready > kk and
// applied == kk; panel kk waits for applied >= kk on its own blocks.  The
// other tasks of reflector kk also wait until its tasks on panel kk+1's
// columns (the critical ones) have finished, so that those stage their data
// without competition (word [3] counts finished critical tasks).  Tasks
// only wait on earlier tasks and on panels, and every CTA is resident
// (cooperative launch), so the waits end; each is bounded all the same
// (spin_limit polls): on expiry it raises the error word, and every wait gives
// up once the error word is set.  Data written by other CTAs within the launch
// is read with L2 loads (ld.global.cg), never through L1.

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// true once *flag >= target; false if the error word is set or the poll limit runs out
__device__ bool wait_geq(const int* flag, int target, const int* err, long long limit) {
    for (long long it = 0; it < limit; ++it) {
        if (ld_acquire(flag) >= target) return true;
        if (ld_acquire(err)) return false;
        if (it > 32) __nanosleep(128);
    }
    return false;
}

struct WySmem {
    double Zp[512];     // partial V^T C, [part][l][q] (one per thread)
    double Z2[32][8];
    double Ts[32][33];  // Ts[c][r] = T(r, c)
};

// C (mp x ncol, ncol <= NC, ld ldc) <- (I - V T^T V^T) C for one 32-wide block
// reflector (V unit lower trapezoidal, read below the diagonal only; T upper),
// staged in shared memory.  V is a factored panel, final before any task reads
// it, so it comes by asynchronous copies through L1 (all in flight at once);
// C and T, rewritten by other CTAs during the launch, come by L2 loads
// (ld.global.cg), which never allocate in L1.  The 32 x NC dots of Z = V^T C
// are split over 256 / (32 NC) row partitions.  All 256 threads call it.
template <int NC>
__device__ void wy_task(const double* __restrict__ V, int ldv, const double* __restrict__ T, int ldt, int b,
                        double* __restrict__ C, int ldc, int mp, int ncol, double* dyn, WySmem& ws) {
    constexpr int TH = PWC_THREADS, B = 32, RT = (512 + TH - 1) / TH, NPART = TH / (B * NC);  // mp <= 512 rows
    static_assert(NPART * B * NC == TH, "one thread per (partition, l, q)");
    const int ld = mp + 1, tid = threadIdx.x;
    double* Vs = dyn;
    double* Cs = Vs + (size_t)ld * B;
#pragma unroll 8
    for (int col = 0; col < B; ++col) {
#pragma unroll
        for (int h = 0; h < RT; ++h) {
            const int r = tid + TH * h;
            if (r < mp) {
                if (col < b && r > col) cp_async8(Vs + (size_t)col * ld + r, V + (size_t)col * ldv + r);
                else Vs[(size_t)col * ld + r] = (col < b && r == col) ? 1.0 : 0.0;
            }
        }
    }
#pragma unroll
    for (int col = 0; col < NC; ++col) {
#pragma unroll
        for (int h = 0; h < RT; ++h) {
            const int r = tid + TH * h;
            if (r < mp) Cs[(size_t)col * ld + r] = col < ncol ? __ldcg(C + (size_t)col * ldc + r) : 0.0;
        }
    }
    for (int e = tid; e < B * B; e += TH) {
        const int r = e & (B - 1), col = e / B;
        ws.Ts[col][r] = (r < b && col < b) ? __ldcg(T + (size_t)col * ldt + r) : 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    {
        const int l = tid % B, q = (tid / B) % NC, part = tid / (B * NC);
        const double* vcol = Vs + (size_t)l * ld;
        const double* ccol = Cs + (size_t)q * ld;
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        int r = part;
        for (; r + 3 * NPART < mp; r += 4 * NPART) {
            a0 = fma(vcol[r], ccol[r], a0);
            a1 = fma(vcol[r + NPART], ccol[r + NPART], a1);
            a2 = fma(vcol[r + 2 * NPART], ccol[r + 2 * NPART], a2);
            a3 = fma(vcol[r + 3 * NPART], ccol[r + 3 * NPART], a3);
        }
        for (; r < mp; r += NPART) a0 = fma(vcol[r], ccol[r], a0);
        ws.Zp[(part * B + l) * NC + q] = (a0 + a1) + (a2 + a3);
    }
    __syncthreads();
    if (tid < B * NC) {
        const int bb = tid % B, q = tid / B;
        double s = 0;
        if (bb < b)
            for (int l = 0; l <= bb; ++l) {
                double z = 0;
#pragma unroll
                for (int pp = 0; pp < NPART; ++pp) z += ws.Zp[(pp * B + l) * NC + q];
                s = fma(ws.Ts[bb][l], z, s);
            }
        ws.Z2[bb][q] = s;
    }
    __syncthreads();
    for (int r = tid; r < mp; r += TH) {
        double acc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) acc[q] = Cs[(size_t)q * ld + r];
#pragma unroll 4
        for (int l = 0; l < B; ++l) {
            const double vl = Vs[(size_t)l * ld + r];
#pragma unroll
            for (int q = 0; q < NC; ++q) acc[q] = fma(-vl, ws.Z2[l][q], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (q < ncol) C[(size_t)q * ldc + r] = acc[q];
    }
    __syncthreads();
}

inline size_t qrp_smem_bytes(int m) { return sizeof(double) * (size_t)(m + 1) * 40 + sizeof(WySmem); }

// sync words: [0] refready, [1] task counter, [2] error, [3] finished tasks on
// the column blocks of the panel after their reflector's, [4 ..] applied counts of
// W's 2-column blocks, then of Qt's 8-column blocks (zeroed before the launch);
// *derr is a sticky error word of the context.
constexpr int QRP_MAXM = 512;
constexpr int QRP_WB = 2;  // columns of W per task (the next panel's 32 columns make 16 tasks)
constexpr int QRP_QB = 8;  // columns of Qt per task
constexpr int QRP_UNAVAILABLE = -1;  // the persistent QR cannot be launched: take the look-ahead path
__global__ void __launch_bounds__(PWC_THREADS, 1)
    qr_persistent_kernel(double* __restrict__ W, int m, int n, int k, double* __restrict__ Tall,
                         double* __restrict__ Qt, int* __restrict__ sync, int* __restrict__ derr,
                         long long spin_limit) {
    extern __shared__ double dyn[];  // the workers' V and C blocks, then their WySmem
    __shared__ PanelWcSmem ps;
    __shared__ int task_sh, ok_sh;
    WySmem& ws = *reinterpret_cast<WySmem*>(dyn + (size_t)(m + 1) * 40);
    const int K = (k + 31) / 32;
    int* refready = sync;
    int* next_task = sync + 1;
    int* err = sync + 2;
    int* crit_done = sync + 3;
    int* applied_w = sync + 4;
    int* applied_q = applied_w + (n + QRP_WB - 1) / QRP_WB;
    // tasks of reflector kk on panel kk+1's column blocks (before kk: crit_before)
    auto crit_tasks = [&](int kk) {
        const int start = 32 * (kk + 1);
        if (start >= k) return 0;
        const int end = min(start + 32, k);  // panel kk+1's columns
        return (end - 1) / QRP_WB - start / QRP_WB + 1;
    };
    if (blockIdx.x == 0) {
        for (int kk = 0; kk < K; ++kk) {
            const int j0 = 32 * kk, b = min(32, k - j0);
            if (kk > 0) {
                if (threadIdx.x == 0) ok_sh = 1;
                __syncthreads();
                if (threadIdx.x < 32 / QRP_WB) {
                    const int cb = j0 / QRP_WB + (int)threadIdx.x;
                    if (QRP_WB * cb < j0 + b && !wait_geq(applied_w + cb, kk, err, spin_limit)) {
                        atomicExch(err, 1);
                        atomicExch(derr, 1);
                        ok_sh = 0;
                    }
                }
                __syncthreads();
                if (!ok_sh) return;  // the same decision in every thread
                __threadfence();
            }
            double* Tk = Tall + (size_t)j0 * 32;
            panel_wc_any(W, m, m, j0, b, nullptr, 0, Tk, 32, ps);
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                st_release(refready, kk + 1);
            }
        }
        return;
    }
    const int nqb = Qt ? (m + QRP_QB - 1) / QRP_QB : 0;
    for (;;) {
        if (threadIdx.x == 0) task_sh = atomicAdd(next_task, 1);
        __syncthreads();
        int t = task_sh;
        int kk = 0, kind = -1, blk = 0;
        for (; kk < K; ++kk) {
            const int start = min(32 * (kk + 1), k);  // first column after panel kk
            const int nwb = n > start ? (n - 1) / QRP_WB - start / QRP_WB + 1 : 0;
            if (t < nwb) { kind = 0; blk = start / QRP_WB + t; break; }
            t -= nwb;
            if (t < nqb) { kind = 1; blk = t; break; }
            t -= nqb;
        }
        if (kind < 0) return;
        const int j0 = 32 * kk, b = min(32, k - j0), mp = m - j0;
        int* flag = kind == 0 ? applied_w + blk : applied_q + blk;
        const int ncrit = crit_tasks(kk);
        const bool critical = kind == 0 && QRP_WB * blk < min(j0 + b + 32, k);
        int crit_target = 0;  // critical tasks of reflectors 0 .. kk
        if (!critical && ncrit > 0)
            for (int q = 0; q <= kk; ++q) crit_target += crit_tasks(q);
        if (threadIdx.x == 0) {
            bool ok = wait_geq(refready, kk + 1, err, spin_limit) && wait_geq(flag, kk, err, spin_limit);
            if (ok && crit_target > 0) ok = wait_geq(crit_done, crit_target, err, spin_limit);
            if (!ok) {
                atomicExch(err, 1);
                atomicExch(derr, 1);
            }
            ok_sh = ok;
        }
        __syncthreads();
        if (!ok_sh) return;
        __threadfence();
        const double* V = W + (size_t)j0 * m + j0;
        const double* Tk = Tall + (size_t)j0 * 32;
        if (kind == 0) {
            const int cs = max(QRP_WB * blk, j0 + b), ce = min(QRP_WB * blk + QRP_WB, n);
            wy_task<QRP_WB>(V, m, Tk, 32, b, W + (size_t)cs * m + j0, m, mp, ce - cs, dyn, ws);
        } else {
            const int cs = QRP_QB * blk, ce = min(cs + QRP_QB, m);
            wy_task<QRP_QB>(V, m, Tk, 32, b, Qt + (size_t)cs * m + j0, m, mp, ce - cs, dyn, ws);
        }
        if (threadIdx.x == 0) {
            __threadfence();
            st_release(flag, kk + 1);
            if (critical) atomicAdd(crit_done, 1);
        }
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

// dst (cols x rows, ld ldd) = src (rows x cols, ld lds)^T, through 32 x 32 shared tiles
__global__ void transpose_kernel(const double* __restrict__ src, int lds, double* __restrict__ dst, int ldd, int rows,
                                 int cols) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = r0 + threadIdx.x, c = c0 + y;
        if (r < rows && c < cols) tile[y][threadIdx.x] = src[(size_t)c * lds + r];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int c = c0 + threadIdx.x, r = r0 + y;
        if (r < rows && c < cols) dst[(size_t)r * ldd + c] = tile[threadIdx.x][y];
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

namespace {

// Several panels: look-ahead on two streams.  The main stream runs panel k,
// then applies its block reflector to panel k+1's columns only ("narrow"),
// then panel k+1; the side stream, meanwhile, applies it to the columns
// beyond ("wide") and accumulates Q forward, Q <- Q (I - V_k T_k V_k^T), kept
// transposed (Qt = Q^T, m x m) so that the same kernel serves both targets in
// one launch: Qt[j0:, :] <- (I - V T^T V^T) Qt[j0:, :].  The narrow update of
// panel k+1 waits for the wide update of panel k, which brought panel k+2's
// columns up to date.  R and Q's first k columns (Qt's first k rows,
// transposed) are read out once the side stream has finished.
template <int NT, int R, int B, int U>
int qr_lookahead(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr, double* Vall,
                 double* Tall) {
    cudaStream_t s0 = c.stream, s1 = c.aux;
    cudaEvent_t ev_p = c.ev_x[0], ev_w = c.ev_x[1], ev_q = c.ev_x[2];
    const int k = std::min(m, n);
    double* Qt = nullptr;
    if (Qout) {
        TN_CHECK(c.qaccum.ensure(sizeof(double) * (size_t)m * m));
        Qt = c.qaccum.as<double>();
    }
    // the side stream starts after everything already queued on the main stream
    TN_CUDA_CHECK(cudaEventRecord(ev_p, s0));
    TN_CUDA_CHECK(cudaStreamWaitEvent(s1, ev_p, 0));
    if (Qout) {
        set_identity_kernel<<<g1d((long long)m * m), 256, 0, s1>>>(Qt, m, m, m);
        TN_LAUNCH_CHECK();
    }
    bool have_wide = false;
    for (int j0 = 0; j0 < k; j0 += B) {
        const int b = std::min(B, k - j0);
        const int mp = m - j0;
        // the 32-wide panel kernel leaves the reflectors only in W (below the diagonal)
        double* Vp = B == 32 ? W + (size_t)j0 * m + j0 : Vall + (size_t)j0 * m + j0;  // ld m
        double* Tp = Tall + (size_t)j0 * B;                                           // ld B
        launch_panel<NT, R, B, U>(s0, W, m, m, j0, b, B == 32 ? nullptr : Vp, m, Tp, B);
        TN_LAUNCH_CHECK();
        TN_CUDA_CHECK(cudaEventRecord(ev_p, s0));
        // narrow: the next panel's columns (after the previous wide update reached them)
        const int c1 = j0 + b;
        const int nb_next = std::max(0, std::min(B, k - c1));
        if (nb_next > 0) {
            if (have_wide) TN_CUDA_CHECK(cudaStreamWaitEvent(s0, ev_w, 0));
            if (B == 32) {
                dim3 grid((nb_next + WY_COLS - 1) / WY_COLS, WYN_RANKS);
                wy_narrow_kernel<32><<<grid, 256, wyn_smem_bytes(mp, 32), s0>>>(Vp, m, Tp, B, b,
                                                                                W + (size_t)c1 * m + j0, m, mp, nb_next);
            } else {
                wy_apply_kernel<B, true><<<(nb_next + WY_COLS - 1) / WY_COLS, WY_THREADS, wy_smem_bytes(mp, B), s0>>>(
                    Vp, m, Tp, B, b, W + (size_t)c1 * m + j0, m, mp, nb_next);
            }
            TN_LAUNCH_CHECK();
        }
        // wide: every column beyond the next panel, and Qt's rows j0.., on the side stream
        TN_CUDA_CHECK(cudaStreamWaitEvent(s1, ev_p, 0));
        const int c2 = c1 + nb_next;
        const int nw = std::max(0, n - c2), nq = Qout ? m : 0;
        const int blocks = (nw + WY_COLS - 1) / WY_COLS + (nq + WY_COLS - 1) / WY_COLS;
        if (blocks > 0) {
            wy_apply_kernel<B, true><<<blocks, WY_THREADS, wy_smem_bytes(mp, B), s1>>>(
                Vp, m, Tp, B, b, W + (size_t)c2 * m + j0, m, mp, nw, Qt ? Qt + j0 : nullptr, m, nq);
            TN_LAUNCH_CHECK();
        }
        TN_CUDA_CHECK(cudaEventRecord(ev_w, s1));
        have_wide = true;
    }
    TN_CUDA_CHECK(cudaEventRecord(ev_q, s1));
    TN_CUDA_CHECK(cudaStreamWaitEvent(s0, ev_q, 0));
    if (Rout) {
        extract_r_kernel<<<g1d((long long)k * n), 256, 0, s0>>>(W, m, k, n, Rout, ldr);
        TN_LAUNCH_CHECK();
    }
    if (Qout) {
        dim3 grid((m + 31) / 32, (k + 31) / 32);
        transpose_kernel<<<grid, dim3(32, 8), 0, s0>>>(Qt, m, Qout, ldq, k, m);
        TN_LAUNCH_CHECK();
    }
    return TN_OK;
}

// Host side of the persistent QR (32-wide panels, m <= 512, k > 32).  Returns
// QRP_UNAVAILABLE (nothing enqueued) when the cooperative launch is impossible.
int qr_persistent(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr, double* Tall) {
    cudaStream_t st = c.stream;
    const int k = std::min(m, n);
    static thread_local int attr_dev = -1, max_per_sm = 0;
    int dev = 0;
    TN_CUDA_CHECK(cudaGetDevice(&dev));
    const size_t smem = qrp_smem_bytes(QRP_MAXM);
    if (attr_dev != dev) {
        TN_CUDA_CHECK(cudaFuncSetAttribute(qr_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        TN_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_per_sm, qr_persistent_kernel, PWC_THREADS, smem));
        attr_dev = dev;
    }
    // Q forward inside the launch (Q^T accumulated m x m by the workers, beside
    // the panels; the default, measured faster at 512 x 256) or backward after
    // it (the dorgqr order on the thin m x k Q, one launch per reflector).
    const bool fwdq = Qout && c.qr_forward_q;
    const int nwb = (n + QRP_WB - 1) / QRP_WB, nqb = fwdq ? (m + QRP_QB - 1) / QRP_QB : 0;
    const int tasks = std::max(1, (n - 32 + QRP_WB - 1) / QRP_WB) + nqb;  // most tasks of one reflector
    // at most 64 workers: they keep ahead of the panel chain and leave SMs to
    // other contexts sharing the device
    const int G = std::min(std::min(max_per_sm * c.sm_count, 1 + tasks), 65);
    if (G < 2) return QRP_UNAVAILABLE;
    const size_t words = 4 + (size_t)nwb + (size_t)nqb;
    TN_CHECK(c.qrsync.ensure(sizeof(int) * words));
    if (!c.derr.p) {
        TN_CHECK(c.derr.ensure(sizeof(int)));
        TN_CUDA_CHECK(cudaMemset(c.derr.p, 0, sizeof(int)));
    }
    double* Qt = nullptr;
    if (fwdq) {
        TN_CHECK(c.qaccum.ensure(sizeof(double) * (size_t)m * m));
        Qt = c.qaccum.as<double>();
        set_identity_kernel<<<g1d((long long)m * m), 256, 0, st>>>(Qt, m, m, m);
        TN_LAUNCH_CHECK();
    }
    TN_CUDA_CHECK(cudaMemsetAsync(c.qrsync.p, 0, sizeof(int) * words, st));
    int* sync = c.qrsync.as<int>();
    int* derr = c.derr.as<int>();
    long long spin_limit = c.qr_spin_limit;
    cudaError_t e;
    {
        void* args[] = {&W, &m, &n, (void*)&k, &Tall, &Qt, &sync, &derr, &spin_limit};
        e = cudaLaunchCooperativeKernel((const void*)qr_persistent_kernel, dim3(G), dim3(PWC_THREADS), args, smem, st);
        if (e == cudaErrorCooperativeLaunchTooLarge) {
            cudaGetLastError();
            return QRP_UNAVAILABLE;
        }
    }
    TN_CUDA_CHECK(e);
    count_launch();
    if (Rout) {
        extract_r_kernel<<<g1d((long long)k * n), 256, 0, st>>>(W, m, k, n, Rout, ldr);
        TN_LAUNCH_CHECK();
    }
    if (fwdq) {
        dim3 grid((m + 31) / 32, (k + 31) / 32);
        transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(Qt, m, Qout, ldq, k, m);
        TN_LAUNCH_CHECK();
    } else if (Qout) {
        // Q = H_0 ... H_{K-1} [I; 0]: the last reflector first, each on the
        // columns j0 .. k-1 and rows j0 .. m-1 it reaches (V read below the
        // diagonal of the factored W)
        set_identity_kernel<<<g1d((long long)m * k), 256, 0, st>>>(Qout, m, k, ldq);
        TN_LAUNCH_CHECK();
        for (int j0 = ((k - 1) / 32) * 32; j0 >= 0; j0 -= 32) {
            const int b = std::min(32, k - j0), nq = k - j0;
            wy_apply_kernel<32, false><<<(nq + WY_COLS - 1) / WY_COLS, WY_THREADS, wy_smem_bytes(m - j0, 32), st>>>(
                W + (size_t)j0 * m + j0, m, Tall + (size_t)j0 * 32, 32, b, Qout + (size_t)j0 * ldq + j0, ldq, m - j0,
                nq);
            TN_LAUNCH_CHECK();
        }
    }
    return TN_OK;
}

template <int NT, int R, int B, int U>
int qr_dense_reg(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr) {
    cudaStream_t st = c.stream;
    const int k = std::min(m, n);
    static thread_local int attr_set[2] = {-1, -1};  // device whose attributes are set
    int dev = 0;
    TN_CUDA_CHECK(cudaGetDevice(&dev));
    if (attr_set[B == 32] != dev) {
        const int bytes = (int)wy_smem_bytes(B == 32 ? 512 : 1024, B);
        TN_CUDA_CHECK(cudaFuncSetAttribute(wy_apply_kernel<B, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        TN_CUDA_CHECK(cudaFuncSetAttribute(wy_apply_kernel<B, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        if (B == 32)
            TN_CUDA_CHECK(cudaFuncSetAttribute(wy_narrow_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)wyn_smem_bytes(512, 32)));
        attr_set[B == 32] = dev;
    }
    size_t need = sizeof(double) * ((size_t)m * k + (size_t)B * k + 16);
    TN_CHECK(c.qrw.ensure(need));
    double* Vall = c.qrw.as<double>();
    double* Tall = Vall + (size_t)m * k;
    if (B == 32 && k > B && m <= QRP_MAXM && c.use_persistent_qr) {
        const int rc = qr_persistent(c, m, n, W, Qout, ldq, Rout, ldr, Tall);
        if (rc != QRP_UNAVAILABLE) return rc;
    }
    if (k > B && c.aux) return qr_lookahead<NT, R, B, U>(c, m, n, W, Qout, ldq, Rout, ldr, Vall, Tall);
    for (int j0 = 0; j0 < k; j0 += B) {
        const int b = std::min(B, k - j0);
        const int mp = m - j0;
        double* Vp = Vall + (size_t)j0 * m + j0;  // ld m
        double* Tp = Tall + (size_t)j0 * B;        // ld B
        launch_panel<NT, R, B, U>(st, W, m, m, j0, b, Vp, m, Tp, B);
        TN_LAUNCH_CHECK();
        const int nt = n - j0 - b;
        if (nt > 0) {
            wy_apply_kernel<B, true><<<(nt + WY_COLS - 1) / WY_COLS, WY_THREADS, wy_smem_bytes(mp, B), st>>>(
                Vp, m, Tp, B, b, W + (size_t)(j0 + b) * m + j0, m, mp, nt);
            TN_LAUNCH_CHECK();
        }
    }
    if (Rout) {
        extract_r_kernel<<<g1d((long long)k * n), 256, 0, st>>>(W, m, k, n, Rout, ldr);
        TN_LAUNCH_CHECK();
    }
    if (Qout) {
        set_identity_kernel<<<g1d((long long)m * k), 256, 0, st>>>(Qout, m, k, ldq);
        TN_LAUNCH_CHECK();
        const int last = ((k - 1) / B) * B;
        for (int j0 = last; j0 >= 0; j0 -= B) {
            const int b = std::min(B, k - j0);
            const int nq = k - j0;
            wy_apply_kernel<B, false><<<(nq + WY_COLS - 1) / WY_COLS, WY_THREADS, wy_smem_bytes(m - j0, B), st>>>(
                Vall + (size_t)j0 * m + j0, m, Tall + (size_t)j0 * B, B, b, Qout + (size_t)j0 * ldq + j0, ldq,
                m - j0, nq);
            TN_LAUNCH_CHECK();
        }
    }
    return TN_OK;
}

// ---- tall matrices (512 < m <= 1536) -----------------------------------------
//
// 16-column panels factored by qr_panel_tall_kernel -- one CTA, warp w owns
// column w with RPL rows per lane in registers, the reflector u_j read from
// shared memory in the dot pass and again in the update pass (holding it in
// registers as panel_wc does would need 4 RPL registers a thread) -- then the
// panel's block reflector applied to the trailing columns, and after the last
// panel to Q (formed backwards, the dorgqr order), by wy_cols_kernel: one CTA
// per eight columns of C, Z = V^T C and C -= V (T' Z) on the FP64 tensor
// cores, with V (from below the diagonal of the factored W) staged in shared
// memory.
__device__ __forceinline__ void cq_dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

constexpr int TALL_B = 16;        // columns per panel (one per warp)
constexpr int TALL_MAXR = 1536;   // rows

struct PanelTallSmem {
    double ub[2][TALL_MAXR];  // u_j by step parity
    double alph[2];
    double Gs[32][33];        // Gs[l][jj] = v_l^T v_jj, l < jj (b <= 16 of 32 used)
    double taus[32], scals[32], betas[32];
    double Tsm[32][33];
    double Xs[32][33];
};

template <int RPL>
__global__ void __launch_bounds__(PWC_THREADS, 1) qr_panel_tall_kernel(double* __restrict__ W, int ldw, int m, int j0,
                                                                        int b, double* __restrict__ T, int ldt) {
    static_assert(32 * RPL <= TALL_MAXR, "panel rows");
    extern __shared__ double tall_dyn[];
    PanelTallSmem& sm = *reinterpret_cast<PanelTallSmem*>(tall_dyn);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;  // warp w: column w of the panel (w < b)
    const int mp = m - j0;
    for (int e = tid; e < 32 * 33; e += PWC_THREADS) (&sm.Gs[0][0])[e] = 0.0;
    double p[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
        const int ri = lane + 32 * q;
        p[q] = (w < b && ri < mp) ? __ldcg(W + (size_t)(j0 + w) * ldw + j0 + ri) : 0.0;
    }
    auto publish = [&](int c, int par) {  // by the warp that owns column c
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int ri = lane + 32 * q;
            sm.ub[par][ri] = ri > c ? p[q] : 0.0;
        }
        if (lane == c) sm.alph[par] = p[0];
    };
    if (w == 0) publish(0, 0);
    __syncthreads();
#pragma unroll 1
    for (int j = 0; j < b; ++j) {
        const int par = j & 1;
        const double* u = sm.ub[par];
        const double alpha = sm.alph[par];
        double x0 = 0, x1 = 0, n0 = 0, n1 = 0;
#pragma unroll
        for (int q = 0; q < RPL; q += 2) {
            const double ua = u[lane + 32 * q];
            x0 = fma(ua, p[q], x0);
            n0 = fma(ua, ua, n0);
            if (q + 1 < RPL) {
                const double ub = u[lane + 32 * (q + 1)];
                x1 = fma(ub, p[q + 1], x1);
                n1 = fma(ub, ub, n1);
            }
        }
        double x = x0 + x1, xn2 = n0 + n1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_xor_sync(0xffffffffu, x, o);
            xn2 += __shfl_xor_sync(0xffffffffu, xn2, o);
        }
        double tau = 0, beta = alpha, scal = 1;
        if (xn2 > 0.0) {
            const double nrm = sqrt(alpha * alpha + xn2);
            beta = alpha >= 0 ? -nrm : nrm;
            const double amb = alpha - beta;
            const double rinv = 1.0 / (beta * amb);  // tau = -amb / beta, scal = 1 / amb
            tau = -amb * amb * rinv;
            scal = beta * rinv;
        }
        const double pj = __shfl_sync(0xffffffffu, p[0], j);  // row j of this warp's column
        const double g = fma(scal, x, pj);                   // v_j^T p
        if (w > j && w < b) {
            if (tau != 0.0) {
                const double tt = tau * g, cu = tt * scal;
#pragma unroll
                for (int q = 0; q < RPL; ++q) p[q] = fma(-cu, u[lane + 32 * q], p[q]);
                if (lane == j) p[0] -= tt;
            }
        } else if (w < j && lane == 0) {
            sm.Gs[w][j] = sm.scals[w] * g;
        }
        if (w == j && lane == 0) {
            sm.taus[j] = tau;
            sm.scals[j] = scal;
            sm.betas[j] = beta;
        }
        if (j + 1 < b && w == j + 1) publish(j + 1, par ^ 1);
        __syncthreads();
    }
    // the factored panel: R above and on the diagonal, v below it
    if (w < b) {
        const double sc = sm.scals[w], be = sm.betas[w];
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
            const int ri = lane + 32 * q;
            if (ri < mp) W[(size_t)(j0 + w) * ldw + j0 + ri] = ri < w ? p[q] : (ri == w ? be : sc * p[q]);
        }
    }
    build_t(sm.Gs, sm.taus, sm.Tsm, sm.Xs, b, T, ldt);
}

// C (mp x nc, ld ldc) <- (I - V T' V^T) C, V mp x b (b <= 16) unit lower
// trapezoidal read below its diagonal (ld ldv), T' = T^T (TRANS: applying
// Q^T, the trailing update) or T (forming Q); T b x b upper, ld ldt.  One CTA
// per WYC_COLS = 8 columns of C, both products on the FP64 tensor cores (mma
// m8n8k4): V is staged in shared memory once (unit diagonal, zeros above it
// and past b written out; leading dimension 4 mod 16 doubles, so the
// fragment loads of both products are conflict-free), Z = V^T C is summed
// over the warps' row ranges in a fixed order, Z2 = T' Z is formed once, and
// each warp takes row tiles of C -= V Z2.
constexpr int WYC_COLS = 8;
constexpr int WYC_THREADS = 256;

inline int wyc_ldv(int mp) {
    const int m4 = (mp + 7) & ~7;
    return m4 + ((m4 & 15) == 0 ? 4 : 12);  // 4 mod 16
}
inline size_t wyc_smem_bytes(int mp) { return sizeof(double) * (size_t)TALL_B * (size_t)wyc_ldv(mp); }

template <bool TRANS>
__global__ void __launch_bounds__(WYC_THREADS) wy_cols_kernel(const double* __restrict__ V, int ldv,
                                                              const double* __restrict__ T, int ldt, int b,
                                                              double* __restrict__ C, int ldc, int mp, int nc) {
    constexpr int NW = WYC_THREADS / 32;
    extern __shared__ double Vs[];                   // [TALL_B][lds]
    __shared__ double zp[NW][2][64];                 // per-warp partial Z tiles (two 8 x 8 M-tiles)
    __shared__ double Zs[TALL_B][WYC_COLS + 1];      // Z, then Z2 = T' Z
    __shared__ double Tp[TALL_B][TALL_B + 1];        // T'
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, t4 = lane & 3;
    const int c0 = WYC_COLS * blockIdx.x;
    const int mp8 = (mp + 7) & ~7;
    const int lds = mp8 + ((mp8 & 15) == 0 ? 4 : 12);
    // V by asynchronous copies, all in flight at once; the unit diagonal, the
    // zeros above it and past b, and the padding rows by plain stores
    for (int l = 0; l < TALL_B; ++l) {
        for (int r = tid; r < mp8; r += WYC_THREADS) {
            double* dst = Vs + l * lds + r;
            if (l < b && r > l && r < mp) cp_async8(dst, V + (size_t)l * ldv + r);
            else *dst = (l < b && r == l) ? 1.0 : 0.0;
        }
    }
    cp_async_wait_all();
    {
        const int l = tid / TALL_B, k = tid % TALL_B;  // 256 threads: the 16 x 16 T'
        double v = 0.0;
        if (l < b && k < b && (TRANS ? k <= l : k >= l)) v = TRANS ? T[(size_t)l * ldt + k] : T[(size_t)k * ldt + l];
        Tp[l][k] = v;
    }
    __syncthreads();
    // Z = V^T C over this warp's groups of 4 rows; the warp's C entries are
    // loaded up front (independent loads in flight together)
    {
        constexpr int MAXKS = (TALL_MAXR / 4 + NW - 1) / NW;
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        const int col = c0 + g;
        const double* Cg = C + (size_t)min(col, nc - 1) * ldc;
        double cv[MAXKS];
#pragma unroll
        for (int i = 0; i < MAXKS; ++i) {
            const int r = 4 * (w + NW * i) + t4;
            cv[i] = (col < nc && r < mp) ? Cg[r] : 0.0;  // B[t][g] = C[4ks + t][c0 + g]
        }
#pragma unroll
        for (int i = 0; i < MAXKS; ++i) {
            const int ks = w + NW * i;
            if (4 * ks < mp8) {
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
                    cq_dmma(acc[mi], Vs[(8 * mi + g) * lds + 4 * ks + t4], cv[i]);  // A[g][t] = V[4ks + t][8mi + g]
            }
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
            zp[w][mi][2 * lane] = acc[mi][0];
            zp[w][mi][2 * lane + 1] = acc[mi][1];
        }
    }
    __syncthreads();
    if (tid < 128) {  // Z[l][n]: tile mi = l / 8, fragment row l % 8, column n
        const int mi = tid >> 6, e = tid & 63, ln = e >> 1;
        const int l = 8 * mi + (ln >> 2), n = 2 * (ln & 3) + (e & 1);
        double s = 0.0;
#pragma unroll
        for (int p = 0; p < NW; ++p) s += zp[p][mi][e];
        Zs[l][n] = s;
    }
    __syncthreads();
    double z2 = 0.0;
    if (tid < 128) {
        const int l = tid >> 3, n = tid & 7;
#pragma unroll
        for (int k = 0; k < TALL_B; ++k) z2 = fma(Tp[l][k], Zs[k][n], z2);
    }
    __syncthreads();
    if (tid < 128) Zs[tid >> 3][tid & 7] = z2;
    __syncthreads();
    // C -= V Z2, 8-row tiles
    double bz[4];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) bz[ks] = Zs[4 * ks + t4][g];  // B[t][g] = Z2[4ks + t][g]
    constexpr int MAXRT = (TALL_MAXR / 8 + NW - 1) / NW;
    double dd[MAXRT][2];
#pragma unroll
    for (int i = 0; i < MAXRT; ++i) {
        const int r0 = 8 * (w + NW * i);
        dd[i][0] = dd[i][1] = 0.0;
        if (r0 < mp8) {
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) cq_dmma(dd[i], Vs[(4 * ks + t4) * lds + r0 + g], bz[ks]);  // A[g][t] = V[r0 + g][4ks + t]
        }
    }
    // the read-modify-writes of C after all the products, so their loads overlap
#pragma unroll
    for (int i = 0; i < MAXRT; ++i) {
        const int r = 8 * (w + NW * i) + g;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int col = c0 + 2 * t4 + h;
            if (r < mp && col < nc) C[(size_t)col * ldc + r] -= dd[i][h];
        }
    }
}

template <int RPL>
int launch_panel_tall(cudaStream_t st, double* W, int ldw, int m, int j0, int b, double* T, int ldt) {
    static thread_local int attr_dev = -1;
    int dev = 0;
    TN_CUDA_CHECK(cudaGetDevice(&dev));
    if (attr_dev != dev) {
        TN_CUDA_CHECK(cudaFuncSetAttribute(qr_panel_tall_kernel<RPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sizeof(PanelTallSmem)));
        attr_dev = dev;
    }
    qr_panel_tall_kernel<RPL><<<1, PWC_THREADS, sizeof(PanelTallSmem), st>>>(W, ldw, m, j0, b, T, ldt);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

// Householder QR of an m x n matrix W (ld m), 512 < m <= 1536, in 16-column
// panels; R to Rout (k x n), Q (m x k) to Qout, when given.
int qr_tall(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr) {
    cudaStream_t st = c.stream;
    const int k = std::min(m, n), B = TALL_B;
    if (m > TALL_MAXR) return TN_BAD_SHAPE;
    TN_CHECK(c.qrw.ensure(sizeof(double) * ((size_t)B * k + 16)));
    double* Tall = c.qrw.as<double>();
    static thread_local int attr_dev = -1;
    int dev = 0;
    TN_CUDA_CHECK(cudaGetDevice(&dev));
    if (attr_dev != dev) {
        const int bytes = (int)wyc_smem_bytes(TALL_MAXR);
        TN_CUDA_CHECK(cudaFuncSetAttribute(wy_cols_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        TN_CUDA_CHECK(cudaFuncSetAttribute(wy_cols_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        attr_dev = dev;
    }
    auto update = [&](cudaStream_t us, bool trans, int j0, int b, double* Cp, int ldc, int mp, int nc) -> int {
        const int blocks = (nc + WYC_COLS - 1) / WYC_COLS;
        const double* Vp = W + (size_t)j0 * m + j0;
        const double* Tp = Tall + (size_t)j0 * B;
        const size_t smem = wyc_smem_bytes(mp);
        if (trans) wy_cols_kernel<true><<<blocks, WYC_THREADS, smem, us>>>(Vp, m, Tp, B, b, Cp, ldc, mp, nc);
        else wy_cols_kernel<false><<<blocks, WYC_THREADS, smem, us>>>(Vp, m, Tp, B, b, Cp, ldc, mp, nc);
        TN_LAUNCH_CHECK();
        return TN_OK;
    };
    // Look-ahead on two streams (as qr_lookahead): the main stream factors
    // panel k, applies its reflector to panel k+1's columns only ("narrow") and
    // factors panel k+1; the side stream applies it to every column beyond
    // ("wide") meanwhile.  A narrow update waits for the previous wide update,
    // which brought the same columns up to date with the reflector before.
    cudaStream_t s1 = c.aux;
    cudaEvent_t ev_p = c.ev_x[0], ev_w = c.ev_x[1], ev_q = c.ev_x[2];
    if (s1) {
        TN_CUDA_CHECK(cudaEventRecord(ev_p, st));  // the side stream starts after what is queued already
        TN_CUDA_CHECK(cudaStreamWaitEvent(s1, ev_p, 0));
    }
    bool have_wide = false;
    for (int j0 = 0; j0 < k; j0 += B) {
        const int b = std::min(B, k - j0), mp = m - j0;
        double* Tp = Tall + (size_t)j0 * B;
        if (mp <= 512) TN_CHECK(launch_panel_tall<16>(st, W, m, m, j0, b, Tp, B));
        else if (mp <= 768) TN_CHECK(launch_panel_tall<24>(st, W, m, m, j0, b, Tp, B));
        else if (mp <= 1024) TN_CHECK(launch_panel_tall<32>(st, W, m, m, j0, b, Tp, B));
        else if (mp <= 1280) TN_CHECK(launch_panel_tall<40>(st, W, m, m, j0, b, Tp, B));
        else TN_CHECK(launch_panel_tall<48>(st, W, m, m, j0, b, Tp, B));
        const int c1 = j0 + b, nt = n - c1;
        if (nt <= 0) continue;
        if (!s1) {
            TN_CHECK(update(st, true, j0, b, W + (size_t)c1 * m + j0, m, mp, nt));
            continue;
        }
        TN_CUDA_CHECK(cudaEventRecord(ev_p, st));
        const int nb_next = std::max(0, std::min(B, k - c1));
        if (nb_next > 0) {
            if (have_wide) TN_CUDA_CHECK(cudaStreamWaitEvent(st, ev_w, 0));
            TN_CHECK(update(st, true, j0, b, W + (size_t)c1 * m + j0, m, mp, nb_next));
        }
        const int c2 = c1 + nb_next, nw = n - c2;
        TN_CUDA_CHECK(cudaStreamWaitEvent(s1, ev_p, 0));
        if (nw > 0) TN_CHECK(update(s1, true, j0, b, W + (size_t)c2 * m + j0, m, mp, nw));
        TN_CUDA_CHECK(cudaEventRecord(ev_w, s1));
        have_wide = true;
    }
    if (s1) {
        TN_CUDA_CHECK(cudaEventRecord(ev_q, s1));
        TN_CUDA_CHECK(cudaStreamWaitEvent(st, ev_q, 0));
    }
    if (Rout) {
        extract_r_kernel<<<g1d((long long)k * n), 256, 0, st>>>(W, m, k, n, Rout, ldr);
        TN_LAUNCH_CHECK();
    }
    if (Qout) {
        set_identity_kernel<<<g1d((long long)m * k), 256, 0, st>>>(Qout, m, k, ldq);
        TN_LAUNCH_CHECK();
        for (int j0 = ((k - 1) / B) * B; j0 >= 0; j0 -= B) {
            const int b = std::min(B, k - j0);
            TN_CHECK(update(st, false, j0, b, Qout + (size_t)j0 * ldq + j0, ldq, m - j0, k - j0));
        }
    }
    return TN_OK;
}

}  // namespace

int check_device_error(Ctx& c) {
    if (!c.derr.p) return TN_OK;
    int h = 0;
    TN_CUDA_CHECK(cudaMemcpy(&h, c.derr.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (!h) return TN_OK;
    TN_CUDA_CHECK(cudaMemset(c.derr.p, 0, sizeof(int)));
    set_error("a bounded wait between the CTAs of the persistent QR expired");
    return TN_CUDA_ERROR;
}

int qr_dense(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr) {
    cudaStream_t st = c.stream;
    if (m <= 0 || n <= 0) return TN_BAD_SHAPE;
    if (m <= 512) return qr_dense_reg<256, 2, 32, 2>(c, m, n, W, Qout, ldq, Rout, ldr);
    if (m <= TALL_MAXR) return qr_tall(c, m, n, W, Qout, ldq, Rout, ldr);
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
