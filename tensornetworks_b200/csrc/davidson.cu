// davidson.cu -- device Davidson for the lowest eigenpair of Heff, with the
// diagonal correction t = r / (theta - diag), optionally plus a learned
// per-element MLP estimate of its error.  No reference counterpart (the
// reference diagonalises the dense Heff with zheevx,
// MPSSite_Variational.C:18-33); it is the "Davidson
// correction equation" solver of the learned preconditioner, and plain
// diagonal Davidson is its fallback whenever the learned correction stalls.
//
// One step (all on the device, deterministic last-block reductions):
//   orthogonalise the correction t against V twice (CGS2), normalise -> v_k
//   w_k = H v_k;  S(:, k) = V^T w_k;  lowest pair (theta, s) of S
//   u = V s,  r = W s - theta u,  |r|;  converged / restart / stall flags
//   t = correction(r, theta, diag, u)
// The projected problem (k <= 32) is tridiagonalised by one warp
// (Householder, lanes = rows), its lowest eigenvalue found by Sturm
// multisection over the block and its eigenvector by inverse iteration.
#include "davidson.h"

#include <algorithm>
#include <cmath>

#include "mlp.h"
#include "tridiag.cuh"

namespace tnb {

namespace {

constexpr int DV_THREADS = 256;
constexpr int KCH = 8;

__device__ __forceinline__ double dwsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Reduce KCH per-thread values over the block into out[] (valid after return).
__device__ void dv_block_sum(double (&v)[KCH], double* out, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < KCH; ++q) v[q] = dwsum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < KCH; ++q) sh[q * 32 + wid] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < KCH; ++q) {
            double s = lane < nw ? sh[q * 32 + lane] : 0.0;
            s = dwsum(s);
            if (lane == 0) out[q] = s;
        }
    }
    __syncthreads();
}

// Ticket of the last block to finish (after every block has written its partials).
__device__ bool dv_last_block(DvState* st) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int prev = atomicAdd(&st->counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

__global__ void dv_reset_kernel(DvState* st, double tol, double tol_rel, int kmax, int max_iters, int learned,
                                double pos) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        st->done = 0;
        st->k = 0;
        st->matvecs = 0;
        st->converged = 0;
        st->counter = 0;
        st->restart = 0;
        st->stalled = 0;
        st->iters = 0;
        st->kmax = kmax;
        st->max_iters = max_iters;
        st->learned = learned;
        st->learned_steps = 0;
        st->recorded = 0;
        st->tol = tol;
        st->tol_rel = tol_rel;
        st->theta = 0;
        st->resid = 1e300;
        st->rms_r = 0;
        st->sigma = 1;
        st->tnorm = 0;
        st->pos = pos;
    }
}

__global__ void dv_copy_kernel(const double* __restrict__ x, double* __restrict__ t, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        t[i] = x[i];
}

// h = V^T t over the k basis vectors.
__global__ void dv_dots_kernel(const double* __restrict__ V, const double* __restrict__ t, long long N,
                               double* partial, DvState* st) {
    if (st->done) return;
    const int k = st->k;
    if (k == 0) return;
    __shared__ double sh[KCH * 32];
    __shared__ double res[KCH];
    for (int k0 = 0; k0 < k; k0 += KCH) {
        double v[KCH] = {0};
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
             i += (long long)gridDim.x * blockDim.x) {
            const double ti = t[i];
#pragma unroll
            for (int q = 0; q < KCH; ++q)
                if (k0 + q < k) v[q] = fma(V[(long long)(k0 + q) * N + i], ti, v[q]);
        }
        dv_block_sum(v, res, sh);
        if (threadIdx.x < KCH && k0 + (int)threadIdx.x < k)
            partial[(long long)blockIdx.x * DV_MAXK + k0 + threadIdx.x] = res[threadIdx.x];
    }
    if (!dv_last_block(st)) return;
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        double s = 0;
        for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(partial + (long long)b * DV_MAXK + j);
        st->h[j] = s;
    }
    if (threadIdx.x == 0) st->counter = 0;
}

// t' = t - V h;  h2 = V^T t';  |t'|^2 and |t|^2.  Last block: h2 and the norm
// of t'' = t' - V h2 (second Gram-Schmidt pass), relative to |t|.
__global__ void dv_orth_kernel(const double* __restrict__ V, double* __restrict__ t, long long N, double* partial,
                               DvState* st) {
    if (st->done) return;
    const int k = st->k;
    __shared__ double sh[KCH * 32];
    __shared__ double res[KCH];
    __shared__ double hs[DV_MAXK];
    for (int j = threadIdx.x; j < k; j += blockDim.x) hs[j] = st->h[j];
    __syncthreads();
    double t0 = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double ti = t[i];
        t0 = fma(ti, ti, t0);
        for (int j = 0; j < k; ++j) ti = fma(-hs[j], V[(long long)j * N + i], ti);
        t[i] = ti;
    }
    // slots: h2[0..k-1], |t'|^2 at k, |t|^2 at k+1
    for (int k0 = 0; k0 < k + 2; k0 += KCH) {
        double v[KCH] = {0};
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
             i += (long long)gridDim.x * blockDim.x) {
            const double ti = t[i];
#pragma unroll
            for (int q = 0; q < KCH; ++q) {
                const int j = k0 + q;
                if (j < k) v[q] = fma(V[(long long)j * N + i], ti, v[q]);
                else if (j == k) v[q] = fma(ti, ti, v[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < KCH; ++q)
            if (k0 + q == k + 1) v[q] = t0;  // |t|^2 (this thread's grid-stride partial)
        dv_block_sum(v, res, sh);
        if (threadIdx.x < KCH && k0 + (int)threadIdx.x < k + 2)
            partial[(long long)blockIdx.x * (DV_MAXK + 2) + k0 + threadIdx.x] = res[threadIdx.x];
    }
    if (!dv_last_block(st)) return;
    __shared__ double h2s[DV_MAXK + 2];
    for (int j = threadIdx.x; j < k + 2; j += blockDim.x) {
        double s = 0;
        for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(partial + (long long)b * (DV_MAXK + 2) + j);
        h2s[j] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ss = 0;
        for (int j = 0; j < k; ++j) {
            st->h2[j] = h2s[j];
            ss += h2s[j] * h2s[j];
        }
        const double tn = sqrt(fmax(h2s[k] - ss, 0.0));
        const double t0n = sqrt(h2s[k + 1]);
        st->tnorm = tn;
        // the correction lies in the span of V: the subspace cannot grow
        if (!(tn > 1e-10 * t0n) || !(t0n > 0)) st->done = 1;
        st->counter = 0;
    }
}

// v_k = (t' - V h2) / tnorm into V[k] and xcur; the last block advances k.
__global__ void dv_newvec_kernel(double* __restrict__ V, const double* __restrict__ t, long long N,
                                 double* __restrict__ xcur, DvState* st) {
    if (st->done) return;
    const int k = st->k;
    __shared__ double hs[DV_MAXK];
    for (int j = threadIdx.x; j < k; j += blockDim.x) hs[j] = st->h2[j];
    __syncthreads();
    const double inv = 1.0 / st->tnorm;
    double* vk = V + (long long)k * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double ti = t[i];
        for (int j = 0; j < k; ++j) ti = fma(-hs[j], V[(long long)j * N + i], ti);
        ti *= inv;
        vk[i] = ti;
        xcur[i] = ti;
    }
    if (!dv_last_block(st)) return;
    if (threadIdx.x == 0) {
        st->k = k + 1;
        st->counter = 0;
    }
}

// Lowest eigenpair of the n x n symmetric A (shared, ld DV_MAXK + 1), n <= 32:
// warp 0 tridiagonalises (reflectors kept below the subdiagonal), the block
// bisects, thread 0 runs inverse iteration, warp 0 back-transforms.
__device__ void small_lowest_pair(int n, double (*A)[DV_MAXK + 1], double* theta_out, double* s_out) {
    __shared__ double dd[DV_MAXK], ee[DV_MAXK], tauv[DV_MAXK], y[DV_MAXK];
    __shared__ double dl[DV_MAXK], d2[DV_MAXK], du[DV_MAXK], du2[DV_MAXK];
    __shared__ int piv[DV_MAXK];
    const int tid = threadIdx.x, lane = tid & 31;
    const unsigned full = 0xffffffffu;
    if (tid < 32) {
        for (int j = 0; j + 2 < n; ++j) {
            const double xi = (lane > j && lane < n) ? A[lane][j] : 0.0;
            const double alpha = __shfl_sync(full, xi, j + 1);
            const double ss = dwsum(lane > j + 1 ? xi * xi : 0.0);
            double tau = 0, beta = alpha, vi = (lane == j + 1) ? 1.0 : 0.0;
            if (ss > 0) {
                const double nrm = sqrt(alpha * alpha + ss);
                beta = alpha >= 0 ? -nrm : nrm;
                tau = (beta - alpha) / beta;
                const double sc = 1.0 / (alpha - beta);
                if (lane > j + 1 && lane < n) vi = xi * sc;
            }
            if (tau != 0.0) {
                double p = 0;
                for (int l = j + 1; l < n; ++l) {
                    const double vl = __shfl_sync(full, vi, l);
                    if (lane > j && lane < n) p = fma(A[lane][l], vl, p);
                }
                p *= tau;
                const double K = 0.5 * tau * dwsum((lane > j && lane < n) ? p * vi : 0.0);
                const double wi = p - K * vi;
                __syncwarp();
                for (int l = j + 1; l < n; ++l) {
                    const double vl = __shfl_sync(full, vi, l), wl = __shfl_sync(full, wi, l);
                    if (lane > j && lane < n) A[lane][l] -= vi * wl + wi * vl;
                }
            }
            __syncwarp();
            if (lane == 0) {
                dd[j] = A[j][j];
                ee[j] = beta;
                tauv[j] = tau;
            }
            if (lane > j + 1 && lane < n) A[lane][j] = vi;
            __syncwarp();
        }
        if (lane == 0) {
            if (n >= 2) {
                dd[n - 2] = A[n - 2][n - 2];
                ee[n - 2] = A[n - 1][n - 2];
            }
            dd[n - 1] = A[n - 1][n - 1];
        }
    }
    __syncthreads();
    const double th = block_eig_k(n, dd, ee, 0);
    if (tid == 0) {
        double scale = 0;
        for (int i = 0; i < n; ++i) scale = fmax(scale, fabs(dd[i]) + (i < n - 1 ? fabs(ee[i]) : 0.0));
        scale = fmax(scale, 1e-300);
        for (int i = 0; i < n; ++i) y[i] = 1.0 + 0.1 * ((i * 7919) % 97) / 97.0;
        if (n > 1) {
            for (int it = 0; it < 3; ++it) {
                tri_solve(n, dd, ee, th + 4e-15 * scale, 2.2e-16 * scale, y, dl, d2, du, du2, piv);
                double mx = 0;
                for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(y[i]));
                if (mx > 0)
                    for (int i = 0; i < n; ++i) y[i] /= mx;
            }
        } else {
            y[0] = 1.0;
        }
    }
    __syncthreads();
    if (tid < 32) {
        double si = lane < n ? y[lane] : 0.0;
        for (int j = n - 3; j >= 0; --j) {
            const double vi = (lane == j + 1) ? 1.0 : ((lane > j + 1 && lane < n) ? A[lane][j] : 0.0);
            const double dot = dwsum(vi * si);
            si -= tauv[j] * vi * dot;
        }
        const double nr = sqrt(dwsum(si * si));
        // sign fixed by the largest component (deterministic)
        double mx = fabs(si);
        int im = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double omx = __shfl_xor_sync(full, mx, o);
            const int oim = __shfl_xor_sync(full, im, o);
            if (omx > mx || (omx == mx && oim < im)) {
                mx = omx;
                im = oim;
            }
        }
        const double sg = __shfl_sync(full, si, im) < 0 ? -1.0 : 1.0;
        if (lane < n) s_out[lane] = sg * si / nr;
        if (lane == 0) *theta_out = th;
    }
}

// W[k-1] = wcur;  S(:, k-1) = V^T wcur;  lowest pair of S.
__global__ void dv_proj_kernel(const double* __restrict__ V, double* __restrict__ W, const double* __restrict__ wcur,
                               long long N, double* partial, DvState* st) {
    if (st->done) return;
    const int k = st->k;
    double* wk = W + (long long)(k - 1) * N;
    __shared__ double sh[KCH * 32];
    __shared__ double res[KCH];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        wk[i] = wcur[i];
    for (int k0 = 0; k0 < k; k0 += KCH) {
        double v[KCH] = {0};
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
             i += (long long)gridDim.x * blockDim.x) {
            const double wi = wcur[i];
#pragma unroll
            for (int q = 0; q < KCH; ++q)
                if (k0 + q < k) v[q] = fma(V[(long long)(k0 + q) * N + i], wi, v[q]);
        }
        dv_block_sum(v, res, sh);
        if (threadIdx.x < KCH && k0 + (int)threadIdx.x < k)
            partial[(long long)blockIdx.x * DV_MAXK + k0 + threadIdx.x] = res[threadIdx.x];
    }
    if (!dv_last_block(st)) return;
    __shared__ double A[DV_MAXK][DV_MAXK + 1];
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        double s = 0;
        for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(partial + (long long)b * DV_MAXK + j);
        st->S[(k - 1) * DV_MAXK + j] = s;
        st->S[j * DV_MAXK + (k - 1)] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
        const int i = e % k, j = e / k;
        // symmetrise with the mean of the two computed triangles
        A[i][j] = 0.5 * (st->S[j * DV_MAXK + i] + st->S[i * DV_MAXK + j]);
    }
    __syncthreads();
    small_lowest_pair(k, A, &st->theta, st->s);
    if (threadIdx.x == 0) {
        st->matvecs += 1;
        st->counter = 0;
    }
}

// u = V s, wu = W s, r = wu - theta u; |r|^2 and sum (diag - theta)^2.
// Inside a graph loop (cond != 0) it also decides whether the loop runs
// another step; it ends the loop at the latest at the iteration cap.
__global__ void dv_resid_kernel(const double* __restrict__ V, const double* __restrict__ W,
                                const double* __restrict__ diag, long long N, double* __restrict__ r,
                                double* __restrict__ u, double* __restrict__ wu, double* partial, DvState* st,
                                cudaGraphConditionalHandle cond) {
    if (st->done) {
        if (cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0u);
        return;
    }
    const int k = st->k;
    const double th = st->theta;
    __shared__ double ss[DV_MAXK];
    __shared__ double sh[KCH * 32];
    __shared__ double res[KCH];
    for (int j = threadIdx.x; j < k; j += blockDim.x) ss[j] = st->s[j];
    __syncthreads();
    double v[KCH] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double ui = 0, wi = 0;
        for (int j = 0; j < k; ++j) {
            ui = fma(ss[j], V[(long long)j * N + i], ui);
            wi = fma(ss[j], W[(long long)j * N + i], wi);
        }
        const double ri = fma(-th, ui, wi);
        u[i] = ui;
        wu[i] = wi;
        r[i] = ri;
        v[0] = fma(ri, ri, v[0]);
        const double dg = diag[i] - th;
        v[1] = fma(dg, dg, v[1]);
    }
    dv_block_sum(v, res, sh);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = res[0];
        partial[2 * blockIdx.x + 1] = res[1];
    }
    if (!dv_last_block(st)) return;
    if (threadIdx.x == 0) {
        double rr = 0, dg2 = 0;
        for (int b = 0; b < (int)gridDim.x; ++b) {
            rr += __ldcg(partial + 2 * b);
            dg2 += __ldcg(partial + 2 * b + 1);
        }
        const double resid = sqrt(rr);
        st->resid = resid;
        st->rms_r = resid / sqrt((double)N);
        st->sigma = fmax(sqrt(dg2 / (double)N), 1e-300);
        const int it = st->iters;
        if (it < 256) st->rhist[it] = resid;
        st->iters = it + 1;
        const double tolEff =
            fmax(fmax(st->tol, 1e-13 * fmax(1.0, fabs(th))), st->tol_rel * fmax(fabs(th), st->sigma));
        if (resid <= tolEff) {
            st->done = 1;
            st->converged = 1;
        }
        // split-precision operator: a residual that no longer halves over two
        // steps has reached the operator's noise floor
        if (st->tol_rel > 0 && it >= 2 && resid > 0.5 * st->rhist[it - 2]) st->done = 1;
        if (st->iters >= st->max_iters) st->done = 1;
        // learned correction: fall back to the diagonal one when the residual stalls
        if (st->learned && !st->stalled && it >= 3 && resid > 0.7 * st->rhist[it - 3]) st->stalled = 1;
        st->restart = (k >= st->kmax) ? 1 : 0;
        st->counter = 0;
        if (cond) cudaGraphSetConditional(cond, st->done ? 0u : 1u);
    }
}

// Restart from the Ritz vector: V[0] = u, W[0] = W s, S = [theta], k = 1.
__global__ void dv_restart_kernel(double* __restrict__ V, double* __restrict__ W, const double* __restrict__ u,
                                  const double* __restrict__ wu, long long N, DvState* st) {
    if (st->done || !st->restart) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        V[i] = u[i];
        W[i] = wu[i];
    }
    if (!dv_last_block(st)) return;
    if (threadIdx.x == 0) {
        st->S[0] = st->theta;
        st->s[0] = 1.0;
        st->k = 1;
        st->restart = 0;
        st->counter = 0;
    }
}

// Diagonal correction r / (theta - diag), the denominator kept away from zero.
__device__ __forceinline__ double diag_correction(double ri, double di, double th, double eps) {
    double den = th - di;
    if (fabs(den) < eps) den = den < 0 ? -eps : eps;
    return ri / den;
}

// Correction t from the residual: the diagonal one, plus (learned) the MLP's
// estimate of its error, in units of rms(r) / sigma.
__global__ void dv_correct_kernel(const double* __restrict__ r, const double* __restrict__ diag,
                                  const double* __restrict__ u, double* __restrict__ t, long long N,
                                  const __nv_bfloat16* __restrict__ w16, DvState* st) {
    if (st->done) return;
    const double th = st->theta;
    const double eps = 1e-8 * fmax(1.0, fabs(th));
    const bool use_mlp = (w16 != nullptr) && st->learned && !st->stalled;
    if (use_mlp) {
        __shared__ MlpInferSmem s;
        mlp_stage(w16, s);
        __syncthreads();
        const double rs = st->rms_r, sg = st->sigma;
        const float sqn = (float)sqrt((double)N);
        const float rinv = rs > 0 ? (float)(1.0 / rs) : 0.f, sinv = (float)(1.0 / sg);
        const float pos = (float)st->pos;
        const double back = rs / sg;
        mlp_tiles(
            s, N,
            [&](long long i, float(&f)[MLP_IN]) {
                const bool in = i < N;
                f[0] = in ? mlp_clip((float)(diag[i] - th) * sinv, MLP_FEAT_CLIP) : 0.f;
                f[1] = in ? mlp_clip((float)r[i] * rinv, MLP_FEAT_CLIP) : 0.f;
                f[2] = in ? mlp_clip((float)u[i] * sqn, MLP_FEAT_CLIP) : 0.f;
                f[3] = pos;
            },
            [&](long long i, float y) { t[i] = diag_correction(r[i], diag[i], th, eps) + (double)y * back; });
        if (blockIdx.x == 0 && threadIdx.x == 0) st->learned_steps += 1;
        return;
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        t[i] = diag_correction(r[i], diag[i], th, eps);
}

// Training record of this step: features of every element, the Ritz vector,
// and (in the target slot) the normalised diagonal correction; the targets
// are completed once the eigenvector is known.
__global__ void dv_record_kernel(const double* __restrict__ r, const double* __restrict__ diag,
                                 const double* __restrict__ u, long long N, DvState* st, float* feats, float* targets,
                                 long long base, long long capacity, double* ubuf, double* scales, int max_steps) {
    if (st->done) return;
    const int step = st->iters - 1;  // the step whose residual was just formed
    if (step < 0 || step >= max_steps) return;
    const long long off = base + (long long)step * N;
    if (off + N > capacity) return;
    const double th = st->theta, rs = st->rms_r, sg = st->sigma;
    const float sqn = (float)sqrt((double)N);
    const float rinv = rs > 0 ? (float)(1.0 / rs) : 0.f, sinv = (float)(1.0 / sg);
    const double eps = 1e-8 * fmax(1.0, fabs(th));
    const double norm = rs > 0 ? sg / rs : 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        targets[off + i] = mlp_clip((float)(diag_correction(r[i], diag[i], th, eps) * norm), 1e30f);
        float* f = feats + (off + i) * MLP_IN;
        f[0] = mlp_clip((float)(diag[i] - th) * sinv, MLP_FEAT_CLIP);
        f[1] = mlp_clip((float)r[i] * rinv, MLP_FEAT_CLIP);
        f[2] = mlp_clip((float)u[i] * sqn, MLP_FEAT_CLIP);
        f[3] = (float)st->pos;
        ubuf[(long long)step * N + i] = u[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scales[2 * step] = rs;
        scales[2 * step + 1] = sg;
        st->recorded = step + 1;
    }
}

// out = a . b (deterministic last-block reduction)
__global__ void dv_dot_kernel(const double* __restrict__ a, const double* __restrict__ b, long long N,
                              double* partial, double* out, unsigned int* counter) {
    __shared__ double sh[KCH * 32];
    __shared__ double res[KCH];
    __shared__ bool last;
    double v[KCH] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        v[0] = fma(a[i], b[i], v[0]);
    dv_block_sum(v, res, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = res[0];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        double s = 0;
        for (int b2 = 0; b2 < (int)gridDim.x; ++b2) s += __ldcg(partial + b2);
        *out = s;
        *counter = 0;
    }
}

// Targets of one recorded step: the error of the diagonal correction against
// the exact one t* = x / (u.x) - u, both scaled by sigma / rms_r (the slot
// holds the scaled diagonal correction on entry).
__global__ void dv_target_kernel(const double* __restrict__ x, const double* __restrict__ ub, long long N,
                                 const double* __restrict__ ux, const double* __restrict__ scales, float* targets) {
    const double dot = *ux;
    const double inv = fabs(dot) > 1e-300 ? 1.0 / dot : 0.0;
    const double sc = scales[0] > 0 ? scales[1] / scales[0] : 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double ts = x[i] * inv - ub[i];
        targets[i] = mlp_clip((float)(ts * sc - (double)targets[i]), MLP_TARGET_CLIP);
    }
}

__global__ void dv_final_kernel(const double* __restrict__ u, double* __restrict__ x, long long N,
                                const DvState* st) {
    if (st->iters == 0) return;  // never reached a Ritz vector: keep x
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        x[i] = u[i];
}

inline int dv_grid(long long N, int sm) {
    long long b = (N + DV_THREADS - 1) / DV_THREADS;
    long long cap = (long long)sm * 2;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

int davidson_solve(Ctx& c, long long N, double* x, int kmax, int max_iters, double tol, const MatvecFn& mv,
                   const double* diag, const MlpModel* mlp, double pos, DvResult* out, DvRecorder* rec,
                   unsigned long long graph_key, double tol_rel) {
    cudaStream_t st = c.stream;
    if (N <= 0) return TN_BAD_SHAPE;
    if (!diag) {
        set_error("davidson: the operator diagonal is required");
        return TN_BAD_ARG;
    }
    int km = std::max(2, std::min(kmax > 0 ? kmax : 16, DV_MAXK));
    if ((long long)km > N) km = (int)std::max<long long>(1, N);
    if (max_iters <= 0) max_iters = 200;
    if (max_iters > 255) max_iters = 255;
    const int grid = dv_grid(N, c.sm_count);
    // workspace: V, W (km each), wcur, xcur, t, r, u, wu, partials
    const size_t need = sizeof(double) * ((size_t)(2 * km + 6) * N + (size_t)grid * (DV_MAXK + 2) + 64);
    TN_CHECK(c.dv.ensure(need));
    TN_CHECK(c.dvstate.ensure(sizeof(DvState)));
    TN_CHECK(c.pinned.ensure(std::max(sizeof(DvState), sizeof(LzState))));
    double* V = c.dv.as<double>();
    double* W = V + (size_t)km * N;
    double* wcur = W + (size_t)km * N;
    double* xcur = wcur + N;
    double* t = xcur + N;
    double* r = t + N;
    double* u = r + N;
    double* wu = u + N;
    double* partial = wu + N;
    DvState* s = c.dvstate.as<DvState>();
    DvState* hs = reinterpret_cast<DvState*>(c.pinned.p);
    const __nv_bfloat16* w16 = mlp ? mlp->w16.as<__nv_bfloat16>() : nullptr;
    const bool learned = mlp != nullptr;
    const bool recording = rec && rec->size < rec->capacity && !learned;
    if (recording) {
        TN_CHECK(rec->ubuf.ensure(sizeof(double) * (size_t)max_iters * N));
        TN_CHECK(rec->scales.ensure(sizeof(double) * (2 * (size_t)max_iters + 8)));
    }

    dv_reset_kernel<<<1, 32, 0, st>>>(s, tol, tol_rel, km, max_iters, learned ? 1 : 0, pos);
    TN_LAUNCH_CHECK();
    dv_copy_kernel<<<grid, DV_THREADS, 0, st>>>(x, t, N);
    TN_LAUNCH_CHECK();

    auto enqueue_step = [&](cudaGraphConditionalHandle cond) -> int {
        dv_dots_kernel<<<grid, DV_THREADS, 0, st>>>(V, t, N, partial, s);
        TN_LAUNCH_CHECK();
        dv_orth_kernel<<<grid, DV_THREADS, 0, st>>>(V, t, N, partial, s);
        TN_LAUNCH_CHECK();
        dv_newvec_kernel<<<grid, DV_THREADS, 0, st>>>(V, t, N, xcur, s);
        TN_LAUNCH_CHECK();
        TN_CHECK(mv(xcur, wcur, &s->done));
        dv_proj_kernel<<<grid, DV_THREADS, 0, st>>>(V, W, wcur, N, partial, s);
        TN_LAUNCH_CHECK();
        dv_resid_kernel<<<grid, DV_THREADS, 0, st>>>(V, W, diag, N, r, u, wu, partial, s, cond);
        TN_LAUNCH_CHECK();
        if (recording) {
            dv_record_kernel<<<grid, DV_THREADS, 0, st>>>(r, diag, u, N, s, rec->feats.as<float>(),
                                                          rec->targets.as<float>(), rec->size,
                                                          rec->capacity, rec->ubuf.as<double>(),
                                                          rec->scales.as<double>(), max_iters);
            TN_LAUNCH_CHECK();
        }
        dv_restart_kernel<<<grid, DV_THREADS, 0, st>>>(V, W, u, wu, N, s);
        TN_LAUNCH_CHECK();
        dv_correct_kernel<<<grid, DV_THREADS, 0, st>>>(r, diag, u, t, N, w16, s);
        TN_LAUNCH_CHECK();
        return TN_OK;
    };

    LzGraph* gr = nullptr;
    if (graph_key && c.use_graphs && st != nullptr && !recording) {
        unsigned long long key = hash_val(graph_key, 0x6461766964ULL);
        key = hash_val(key, N);
        key = hash_val(key, km);
        key = hash_val(key, grid);
        key = hash_val(key, (const void*)V);
        key = hash_val(key, (const void*)s);
        key = hash_val(key, (const void*)diag);
        key = hash_val(key, (const void*)w16);
        key = hash_val(key, st);
        key = hash_val(key, alloc_generation());
        auto it = c.lzgraphs.find(key);
        if (it == c.lzgraphs.end()) {
            if (c.lzgraphs.size() >= 256) c.clear_graphs();
            LzGraph g;
            TN_CUDA_CHECK(cudaGraphCreate(&g.graph, 0));
            cudaGraphConditionalHandle h;
            TN_CUDA_CHECK(cudaGraphConditionalHandleCreate(&h, g.graph, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            TN_CUDA_CHECK(cudaGraphAddNode(&node, g.graph, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            const unsigned long long n0 = launch_count();
            TN_CUDA_CHECK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            int rc = enqueue_step(h);
            cudaGraph_t captured = nullptr;
            cudaError_t ec = cudaStreamEndCapture(st, &captured);
            g.kernels_per_iter = launch_count() - n0;
            if (rc != TN_OK || ec != cudaSuccess) {
                cudaGraphDestroy(g.graph);
                if (rc != TN_OK) return rc;
                TN_CUDA_CHECK(ec);
            }
            cudaError_t ei = cudaGraphInstantiate(&g.exec, g.graph, 0);
            if (ei != cudaSuccess) {
                cudaGraphDestroy(g.graph);
                TN_CUDA_CHECK(ei);
            }
            it = c.lzgraphs.emplace(key, g).first;
        }
        gr = &it->second;
    }

    if (gr) {
        TN_CUDA_CHECK(cudaGraphLaunch(gr->exec, st));
    } else {
        // host loop in chunks; the device flags make the surplus launches no-ops
        for (int done_steps = 0; done_steps < max_iters;) {
            const int chunk = std::min(8, max_iters - done_steps);
            for (int j = 0; j < chunk; ++j) TN_CHECK(enqueue_step(0));
            done_steps += chunk;
            TN_CUDA_CHECK(cudaMemcpyAsync(hs, s, sizeof(DvState), cudaMemcpyDeviceToHost, st));
            TN_CUDA_CHECK(cudaStreamSynchronize(st));
            if (hs->done) break;
        }
    }
    dv_final_kernel<<<grid, DV_THREADS, 0, st>>>(u, x, N, s);
    TN_LAUNCH_CHECK();
    TN_CUDA_CHECK(cudaMemcpyAsync(hs, s, sizeof(DvState), cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    if (gr)  // kernels the graph ran: one body per step taken
        for (int k = 0; k < hs->iters; ++k)
            for (unsigned long long q = 0; q < gr->kernels_per_iter; ++q) count_launch();
    if (recording && hs->recorded > 0) {
        // targets of every recorded step from the converged vector x
        const int steps = std::min(hs->recorded, max_iters);
        long long kept = 0;
        double* ux = rec->scales.as<double>() + 2 * max_iters;
        for (int j = 0; j < steps; ++j) {
            const long long off = rec->size + (long long)j * N;
            if (off + N > rec->capacity) break;
            const double* ub = rec->ubuf.as<double>() + (size_t)j * N;
            dv_dot_kernel<<<grid, DV_THREADS, 0, st>>>(ub, x, N, partial, ux, &s->counter);
            TN_LAUNCH_CHECK();
            dv_target_kernel<<<grid, DV_THREADS, 0, st>>>(x, ub, N, ux, rec->scales.as<double>() + 2 * j,
                                                          rec->targets.as<float>() + off);
            TN_LAUNCH_CHECK();
            kept += N;
        }
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        rec->size += kept;
    }
    if (out) {
        out->theta = hs->theta;
        out->resid = hs->resid;
        out->matvecs = hs->matvecs;
        out->iters = hs->iters;
        out->converged = hs->converged;
        out->learned_steps = hs->learned_steps;
        out->stalled = hs->stalled;
    }
    if (!std::isfinite(hs->theta)) {
        set_error("davidson: non-finite Ritz value");
        return TN_NAN_DETECTED;
    }
    return TN_OK;
}

}  // namespace tnb
