// lanczos.cu -- device-resident restarted Lanczos for the lowest eigenpair of Heff.
//
// Replaces the dense zheevx call of MPSSite::Refine (MPSSite_Variational.C:18-33,
// LapackEigenSolver.C:62-109).  Everything except the decision to restart stays
// on the device: the dots, the full reorthogonalisation (classical Gram-Schmidt
// applied twice, FP64 coefficients), the norm, the tridiagonal eigenproblem
// (multisection on Sturm counts over a whole thread block) and the convergence
// flag.  Kernels launched after convergence see the flag and return at once.
// Vector passes are grid-stride, coalesced, FP64, with warp-shuffle block
// reductions and a deterministic last-block final reduction.
#include "lanczos.h"
#include "qr.h"
#include "tridiag.cuh"
#include "pdl.cuh"

#include <cmath>
#include <cstddef>
#include <vector>

namespace tnb {

namespace {

constexpr int LZ_THREADS = 512;  // with one block per SM (vec_grid): few partials for the last-block sums
constexpr int KCHUNK = 8;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Reduce KCHUNK per-thread values over the block; result valid in thread 0's out[].
__device__ void block_sum_chunk(double (&v)[KCHUNK], double* out, double* sh /* [KCHUNK][32] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < KCHUNK; ++q) v[q] = warp_sum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < KCHUNK; ++q) sh[q * 32 + wid] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < KCHUNK; ++q) {
            double s = lane < nw ? sh[q * 32 + lane] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[q] = s;
        }
    }
    __syncthreads();
}

// out[k] = sum over the nb blocks' partials partial[b * stride + k], k < nk, by
// the whole block (every thread must call it): each thread adds its share of
// the blocks in a fixed order, then a block reduction, so the result does not
// depend on timing.  out is shared memory with room for nk rounded up to KCHUNK.
__device__ void reduce_partials(const double* partial, int nb, int stride, int nk, double* out, double* sh) {
    for (int k0 = 0; k0 < nk; k0 += KCHUNK) {
        double v[KCHUNK] = {0};
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
            for (int q = 0; q < KCHUNK; ++q)
                if (k0 + q < nk) v[q] += __ldcg(partial + (long long)b * stride + k0 + q);
        }
        block_sum_chunk(v, out + k0, sh);
    }
}

// acc + sgn * sum_{k < nk} c[k] V[k N + i] with the basis loads issued eight at
// a time (independent, all in flight before their FMAs): a thread touches only a
// few elements, so without this the loop is one load latency per basis vector.
__device__ __forceinline__ double basis_combine(const double* __restrict__ V, long long N, long long i,
                                                const double* c, int nk, double sgn, double acc) {
    int k = 0;
    for (; k + 8 <= nk; k += 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = __ldg(V + (long long)(k + q) * N + i);
#pragma unroll
        for (int q = 0; q < 8; ++q) acc = fma(sgn * c[k + q], v[q], acc);
    }
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (k + q < nk) v[q] = __ldg(V + (long long)(k + q) * N + i);
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (k + q < nk) acc = fma(sgn * c[k + q], v[q], acc);
    return acc;
}

// Step j's tridiagonal problem (alpha, beta of steps 0..j in the state), by the
// whole calling block: the lowest Ritz value, its residual estimate, and the
// decision to stop the restart -- converged, the split-precision operator's
// noise floor (a residual that no longer halves over two steps), or the basis
// limit -- which, inside a graph loop (cond != 0), also ends the loop.  Every
// step reaches it, so the loop ends at the latest at the basis limit.
__device__ void lz_decide_step(LzState* st, int j, cudaGraphConditionalHandle cond) {
    const int nk = j + 1;
    __shared__ double a[LZ_MAXK], b[LZ_MAXK];
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
        a[i] = st->alpha[i];
        b[i] = st->beta[i];
    }
    __syncthreads();
    if (threadIdx.x >= 32) return;  // warp 0 decides (the callers' next barrier waits for it)
    const double th = warp_eig_k(nk, a, b, 0);
    if (threadIdx.x == 0) {
        const double yl = last_component(nk, a, b, th);
        const double bj = b[j];
        const double resid = bj * yl;
        double tolEff = fmax(st->tol, 1e-13 * fmax(1.0, fabs(th)));
        if (st->tol_rel > 0) {
            double tn = 0;
            for (int i = 0; i < nk; ++i) tn = fmax(tn, fabs(a[i]) + fabs(b[i]) + (i > 0 ? fabs(b[i - 1]) : 0.0));
            tolEff = fmax(tolEff, st->tol_rel * tn);
        }
        st->theta = th;
        st->resid = resid;
        st->nb = nk;
        st->rhist[j] = resid;
        int done = 0;
        const bool conv = (resid <= tolEff) || (bj <= 1e-14 * fmax(1.0, fabs(th)));
        if (conv) { done = 1; st->converged = 1; }
        if (st->tol_rel > 0 && j >= 2 && resid > 0.5 * st->rhist[j - 2]) done = 1;
        if (nk >= st->mmax || nk >= LZ_MAXK - 1) done = 1;  // basis exhausted for this restart
        if (done) st->done = 1;
        if (cond) cudaGraphSetConditional(cond, done ? 0u : 1u);
    }
}

// ---- kernels ---------------------------------------------------------------

// A restart's reset (first: the whole solve's); with a step-loop handle it
// also re-arms that WHILE loop, whose value persists between restarts.
__global__ void lz_reset_kernel(LzState* st, double tol, double tol_rel, int first, int mmax,
                                cudaGraphConditionalHandle steps_loop = 0) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        st->done = 0;
        st->nb = 0;
        st->counter = 0;
        st->j = 0;
        st->jn = 0;
        st->mmax = mmax;
        if (first) {
            st->matvecs = 0;
            st->converged = 0;
            st->tol = tol;
            st->tol_rel = tol_rel;
            st->theta = 0;
            st->theta2 = 0;
            st->resid = 1e300;
            st->restarts = 0;
            st->steps = 0;
            st->prev_resid = 1e300;
        }
        if (steps_loop) cudaGraphSetConditional(steps_loop, 1u);
    }
}

// After a restart's Ritz vector: whether another restart runs (the host
// loop's rule: stop when converged, when the basis spans the whole space,
// after maxRestarts, or -- split-precision operators -- when the residual no
// longer halves between restarts).
__global__ void lz_decide_kernel(LzState* st, cudaGraphConditionalHandle restarts_loop, int maxRestarts,
                                 long long N, int mm) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int r = st->restarts;  // index of the restart just finished
    st->restarts = r + 1;
    st->steps += st->nb;
    bool stop = false;
    if (st->converged) stop = true;
    else if ((long long)mm >= N) { st->converged = 1; stop = true; }
    else if (st->tol_rel > 0) {
        if (r > 0 && st->resid > 0.5 * st->prev_resid) stop = true;
        else st->prev_resid = st->resid;
    }
    if (r + 1 >= maxRestarts) stop = true;
    cudaGraphSetConditional(restarts_loop, stop ? 0u : 1u);
}

__global__ void lz_summary_kernel(const LzState* st, LzSummary* out, int kernels_per_step) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    out->theta = st->theta;
    out->theta2 = st->theta2;
    out->resid = st->resid;
    out->matvecs = st->matvecs;
    out->restarts = st->restarts;
    out->converged = st->converged;
    out->steps = st->steps;
    // first reset, per restart (reset, norm, scale, Ritz coefficients and vector,
    // decision), this kernel
    out->launches = 1 + 6LL * st->restarts + (long long)kernels_per_step * st->steps + 1;
}

// ||x||^2 -> st->xnorm (last block).
__global__ void lz_norm_kernel(const double* __restrict__ x, long long N, double* partial, LzState* st) {
    __shared__ double sh[KCHUNK * 32];
    __shared__ double res[KCHUNK];
    __shared__ bool last;
    double v[KCHUNK] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double t = x[i];
        v[0] = fma(t, t, v[0]);
    }
    block_sum_chunk(v, res, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = res[0];
        __threadfence();
        unsigned int prev = atomicAdd(&st->counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        reduce_partials(partial, gridDim.x, 1, 1, res, sh);
        if (threadIdx.x == 0) {
            st->xnorm = sqrt(res[0]);
            st->counter = 0;
        }
    }
}

// v0 = x / |x| (and the matvec input copy xcur when given).
__global__ void lz_scale_kernel(const double* x, double* v0, long long N, const LzState* st, int fill_if_zero,
                                double* xcur, VecSplit sp = VecSplit{}) {
    double nr = st->xnorm;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double v;
        if (nr > 0) v = x[i] / nr;
        else if (fill_if_zero) {
            // deterministic start vector when x = 0
            unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ULL;
            h ^= h >> 29;
            v = ((double)((h >> 11) & 0xFFFFF) / 1048576.0 - 0.5) / sqrt((double)N / 12.0);
        } else v = 0.0;
        v0[i] = v;
        if (xcur) xcur[i] = v;
        if (sp.out) split_bf16((float)v, sp.ns, sp.out, sp.stride, i);
    }
}

// The three kernels of a step hand their sums on as per-block partials: the
// next kernel's every block adds the previous kernel's partials itself, in
// the same fixed order (so every block holds bitwise the same sums), instead
// of a last block reducing them at the end of the previous kernel while the
// other SMs idle.

// Partials of h_k = V_k . w, k = 0..j, into partA.
__global__ void lz_dots_kernel(const double* __restrict__ V, const double* __restrict__ w, long long N,
                               double* partA, LzState* st) {
    pdl_wait();
    if (st->done) return;
    __shared__ double sh[KCHUNK * 32];
    __shared__ double res[KCHUNK];
    const int j = st->j;
    const int nk = j + 1;
    for (int k0 = 0; k0 < nk; k0 += KCHUNK) {
        double v[KCHUNK] = {0};
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
             i += (long long)gridDim.x * blockDim.x) {
            double wi = w[i];
#pragma unroll
            for (int q = 0; q < KCHUNK; ++q)
                if (k0 + q < nk) v[q] = fma(V[(long long)(k0 + q) * N + i], wi, v[q]);
        }
        block_sum_chunk(v, res, sh);
        if (threadIdx.x < KCHUNK && k0 + threadIdx.x < nk)
            partA[(long long)blockIdx.x * LZ_MAXK + k0 + threadIdx.x] = res[threadIdx.x];
    }
}

// h from partA; w' = w - V h; partials of h2 = V^T w' and |w'|^2 into partB.
// Block 0 keeps h in the state (alpha_j = h_j + h2_j is formed next).
__global__ void lz_update_kernel(const double* __restrict__ V, double* __restrict__ w, long long N,
                                 const double* partA, double* partB, LzState* st) {
    pdl_wait();
    if (st->done) return;
    __shared__ double sh[KCHUNK * 32];
    __shared__ double res[KCHUNK];
    __shared__ double hs[LZ_MAXK + KCHUNK];
    const int j = st->j;
    const int nk = j + 1;
    reduce_partials(partA, gridDim.x, LZ_MAXK, nk, hs, sh);
    if (blockIdx.x == 0)
        for (int k = threadIdx.x; k < nk; k += blockDim.x) st->h[k] = hs[k];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double wi = w[i];
        wi = basis_combine(V, N, i, hs, nk, -1.0, wi);
        w[i] = wi;
    }
    for (int k0 = 0; k0 < nk + 1; k0 += KCHUNK) {
        double v[KCHUNK] = {0};
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
             i += (long long)gridDim.x * blockDim.x) {
            double wi = w[i];
#pragma unroll
            for (int q = 0; q < KCHUNK; ++q) {
                int k = k0 + q;
                if (k < nk) v[q] = fma(V[(long long)k * N + i], wi, v[q]);
                else if (k == nk) v[q] = fma(wi, wi, v[q]);
            }
        }
        block_sum_chunk(v, res, sh);
        if (threadIdx.x < KCHUNK && k0 + (int)threadIdx.x <= nk)
            partB[(long long)blockIdx.x * LZ_MAXK + k0 + threadIdx.x] = res[threadIdx.x];
    }
}

// h2 and |w'|^2 from partB, beta_j; V_{j+1} = (w' - V h2) / beta_j, also into
// the matvec input xcur.  Block 0 records alpha_j and beta_j, then solves the
// tridiagonal problem of step j and decides whether the restart ends (and,
// inside a graph loop, whether the loop runs another step), after its share
// of the vector.  The last block to finish advances the step index.  Blocks
// that start after block 0 has ended the restart return at once; the step's
// vector is then unused (and the half-counted ticket is cleared by the next
// reset).
__global__ void lz_next_kernel(double* __restrict__ V, const double* __restrict__ w, long long N,
                               const double* partB, LzState* st, double* __restrict__ xcur, VecSplit sp,
                               cudaGraphConditionalHandle cond = 0) {
    pdl_wait();
    if (st->done) {
        if (cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0u);
        return;
    }
    __shared__ double sh[KCHUNK * 32];
    __shared__ double h2s[LZ_MAXK + KCHUNK];
    __shared__ bool last;
    const int j = st->j;
    const int nk = j + 1;
    reduce_partials(partB, gridDim.x, LZ_MAXK, nk + 1, h2s, sh);
    double ss = 0;
    for (int k = 0; k < nk; ++k) ss = fma(h2s[k], h2s[k], ss);
    const double beta = sqrt(fmax(h2s[nk] - ss, 0.0));
    const double inv = beta > 0 ? 1.0 / beta : 0.0;
    double* vn = V + (long long)(j + 1) * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double wi = w[i];
        wi = basis_combine(V, N, i, h2s, nk, -1.0, wi);
        wi *= inv;
        vn[i] = wi;
        xcur[i] = wi;
        if (sp.out) split_bf16((float)wi, sp.ns, sp.out, sp.stride, i);
    }
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            for (int k = 0; k < nk; ++k) st->h2[k] = h2s[k];
            st->alpha[j] = st->h[j] + h2s[j];
            st->beta[j] = beta;
            st->matvecs += 1;
            st->jn = j + 1;
        }
        __syncthreads();
        lz_decide_step(st, j, cond);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int prev = atomicAdd(&st->counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        st->j = j + 1;
        st->counter = 0;
    }
}

// Ritz coefficients y of the lowest eigenpair of T_nb (inverse iteration), and theta2.
__global__ void lz_ritz_coeffs_kernel(LzState* st) {
    const int n = st->nb;
    if (n <= 0) return;
    __shared__ double a[LZ_MAXK], b[LZ_MAXK];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a[i] = st->alpha[i];
        b[i] = st->beta[i];
    }
    __syncthreads();
    // warp 0 the lowest eigenvalue, warp 1 the next (the gap, for the statistics)
    __shared__ double ths[2];
    const int wv = threadIdx.x >> 5;
    if (wv < 2) {
        const double e = (wv == 0 || n > 1) ? warp_eig_k(n, a, b, wv) : 0.0;
        if ((threadIdx.x & 31) == 0) ths[wv] = e;
    }
    __syncthreads();
    const double th = ths[0], th2 = n > 1 ? ths[1] : th;
    if (threadIdx.x != 0) return;
    st->theta = th;
    st->theta2 = th2;
    __shared__ double y[LZ_MAXK], dl[LZ_MAXK], dd[LZ_MAXK], du[LZ_MAXK], du2[LZ_MAXK];
    __shared__ int piv[LZ_MAXK];
    double scale = 0;
    for (int i = 0; i < n; ++i) scale = fmax(scale, fabs(a[i]) + (i < n - 1 ? fabs(b[i]) : 0.0));
    scale = fmax(scale, 1e-300);
    for (int i = 0; i < n; ++i) y[i] = 1.0 + 0.1 * ((i * 7919) % 97) / 97.0;
    for (int it = 0; it < 3; ++it) {
        tri_solve(n, a, b, th + 4e-15 * scale, 2.2e-16 * scale, y, dl, dd, du, du2, piv);
        double mx = 0;
        for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(y[i]));
        if (mx > 0) for (int i = 0; i < n; ++i) y[i] /= mx;
    }
    double nr = 0;
    for (int i = 0; i < n; ++i) nr += y[i] * y[i];
    nr = sqrt(nr);
    int im = 0;
    for (int i = 1; i < n; ++i) if (fabs(y[i]) > fabs(y[im])) im = i;
    double sg = (y[im] < 0) ? -1.0 : 1.0;
    for (int i = 0; i < n; ++i) st->y[i] = sg * y[i] / nr;
}

// x = V y
__global__ void lz_ritz_vector_kernel(const double* __restrict__ V, double* __restrict__ x, long long N,
                                      const LzState* st) {
    __shared__ double ys[LZ_MAXK];
    const int n = st->nb;
    for (int k = threadIdx.x; k < n; k += blockDim.x) ys[k] = st->y[k];
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double s = 0;
        s = basis_combine(V, N, i, ys, n, 1.0, s);
        x[i] = s;
    }
}

// Rayleigh quotient theta = x.y / x.x and residual |y - theta x| / |x|.
__global__ void rq_dots_kernel(const double* __restrict__ x, const double* __restrict__ y, long long N,
                               double* partial, LzState* st) {
    __shared__ double sh[KCHUNK * 32];
    __shared__ double res[KCHUNK];
    __shared__ bool last;
    double v[KCHUNK] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double a = x[i];
        v[0] = fma(a, y[i], v[0]);
        v[1] = fma(a, a, v[1]);
    }
    block_sum_chunk(v, res, sh);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = res[0];
        partial[2 * blockIdx.x + 1] = res[1];
        __threadfence();
        unsigned int prev = atomicAdd(&st->counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        reduce_partials(partial, gridDim.x, 2, 2, res, sh);
        if (threadIdx.x == 0) {
            const double xy = res[0], xx = res[1];
            st->theta = xx > 0 ? xy / xx : 0.0;
            st->xnorm = sqrt(xx);
            st->counter = 0;
        }
    }
}

__global__ void rq_resid_kernel(const double* __restrict__ x, const double* __restrict__ y, long long N,
                                double* partial, LzState* st) {
    __shared__ double sh[KCHUNK * 32];
    __shared__ double res[KCHUNK];
    __shared__ bool last;
    const double th = st->theta;
    double v[KCHUNK] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double r = y[i] - th * x[i];
        v[0] = fma(r, r, v[0]);
    }
    block_sum_chunk(v, res, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = res[0];
        __threadfence();
        unsigned int prev = atomicAdd(&st->counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        reduce_partials(partial, gridDim.x, 1, 1, res, sh);
        if (threadIdx.x == 0) {
            st->resid = st->xnorm > 0 ? sqrt(res[0]) / st->xnorm : 0.0;
            st->counter = 0;
        }
    }
}

inline int vec_grid(long long N, int sm) {
    long long b = (N + LZ_THREADS - 1) / LZ_THREADS;
    long long cap = (long long)sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Per-block partial sums a step needs: the dots', then the update's.
inline size_t partial_doubles(long long N, int sm) { return 2 * (size_t)vec_grid(N, sm) * LZ_MAXK; }

}  // namespace

// w = Heff xcur and h = V^T w: the matvec, then the dots.
int step_matvec_dots(Ctx& c, const MatvecFn& mv, int grid, const double* V, double* w, const double* xcur,
                     long long N, double* partial, LzState* s) {
    TN_CHECK(mv(xcur, w, &s->done));
    return launch_pdl(lz_dots_kernel, grid, LZ_THREADS, 0, c.stream, V, (const double*)w, N, partial, s);
}

// One Lanczos step: the matvec, then the vector work as three kernels.
static int enqueue_lz_step(Ctx& c, const MatvecFn& mv, int grid, double* V, double* w, double* xcur, long long N,
                           double* partial, LzState* s, const VecSplit& sp, cudaGraphConditionalHandle cond) {
    double* partB = partial + (size_t)grid * LZ_MAXK;
    TN_CHECK(step_matvec_dots(c, mv, grid, V, w, xcur, N, partial, s));
    TN_CHECK(launch_pdl(lz_update_kernel, grid, LZ_THREADS, 0, c.stream, (const double*)V, w, N,
                        (const double*)partial, partB, s));
    return launch_pdl(lz_next_kernel, grid, LZ_THREADS, 0, c.stream, V, (const double*)w, N, (const double*)partB, s,
                      xcur, sp, cond);
}

int lanczos_solve(Ctx& c, long long N, double* x, int m, int maxRestarts, double tol, const MatvecFn& mv,
                  LzResult* out, double tol_rel, unsigned long long graph_key, const VecSplit* split) {
    const VecSplit sp = split ? *split : VecSplit{};
    cudaStream_t st = c.stream;
    if (N <= 0) return TN_BAD_SHAPE;
    int mm = m;
    if (mm > LZ_MAXK - 1) mm = LZ_MAXK - 1;
    if ((long long)mm > N) mm = (int)N;
    if (mm < 1) mm = 1;
    const int grid = vec_grid(N, c.sm_count);
    // workspace: V (mm+1 vectors), w, xcur, partials
    size_t need = sizeof(double) * ((size_t)(mm + 3) * N + partial_doubles(N, c.sm_count) + 64);
    TN_CHECK(c.lz.ensure(need));
    TN_CHECK(c.lzstate.ensure(sizeof(LzState)));
    TN_CHECK(c.pinned.ensure(sizeof(LzState)));
    double* V = c.lz.as<double>();
    double* w = V + (size_t)(mm + 1) * N;
    double* xcur = w + N;
    double* partial = xcur + N;
    LzState* s = c.lzstate.as<LzState>();
    LzState* hs = reinterpret_cast<LzState*>(c.pinned.p);

    // one Lanczos step; cond != 0 inside the graph body
    auto enqueue_step = [&](cudaGraphConditionalHandle cond) -> int {
        return enqueue_lz_step(c, mv, grid, V, w, xcur, N, partial, s, sp, cond);
    };

    LzGraph* gr = nullptr;
    if (graph_key && c.use_graphs && st != nullptr) {
        unsigned long long key = graph_key;
        key = hash_val(key, N);
        key = hash_val(key, mm);
        key = hash_val(key, grid);
        key = hash_val(key, (const void*)sp.out);
        key = hash_val(key, (const void*)V);
        key = hash_val(key, (const void*)s);
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

    int restarts = 0;
    bool converged = false;
    double prev_resid = 1e300;
    if (c.prof) TN_CHECK(c.prof_events());
    for (restarts = 0; restarts < (maxRestarts > 0 ? maxRestarts : 1); ++restarts) {
        if (c.prof) TN_CUDA_CHECK(cudaEventRecord(c.pev[2], st));
        lz_reset_kernel<<<1, 32, 0, st>>>(s, tol, tol_rel, restarts == 0, mm);
        TN_LAUNCH_CHECK();
        lz_norm_kernel<<<grid, LZ_THREADS, 0, st>>>(x, N, partial, s);
        TN_LAUNCH_CHECK();
        lz_scale_kernel<<<grid, LZ_THREADS, 0, st>>>(x, V, N, s, 1, xcur, sp);
        TN_LAUNCH_CHECK();
        if (c.prof) TN_CUDA_CHECK(cudaEventRecord(c.pev[3], st));
        if (gr) {
            TN_CUDA_CHECK(cudaGraphLaunch(gr->exec, st));
        } else {
            for (int j = 0; j < mm; ++j) TN_CHECK(enqueue_step(0));
        }
        if (c.prof) TN_CUDA_CHECK(cudaEventRecord(c.pev[4], st));
        lz_ritz_coeffs_kernel<<<1, LZ_THREADS, 0, st>>>(s);
        TN_LAUNCH_CHECK();
        lz_ritz_vector_kernel<<<grid, LZ_THREADS, 0, st>>>(V, x, N, s);
        TN_LAUNCH_CHECK();
        if (c.prof) TN_CUDA_CHECK(cudaEventRecord(c.pev[5], st));
        TN_CUDA_CHECK(cudaMemcpyAsync(hs, s, sizeof(LzState), cudaMemcpyDeviceToHost, st));
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        if (c.prof) {
            float a = 0, b = 0, d = 0;
            cudaEventElapsedTime(&a, c.pev[2], c.pev[3]);
            cudaEventElapsedTime(&b, c.pev[3], c.pev[4]);
            cudaEventElapsedTime(&d, c.pev[4], c.pev[5]);
            c.prof_ms[1] += a;
            c.prof_ms[2] += b;
            c.prof_ms[3] += d;
            c.prof_steps += hs->nb;
            c.prof_restarts += 1;
        }
        if (gr)  // kernels the graph ran: one body per step taken
            for (int k = 0; k < hs->nb; ++k)
                for (unsigned long long q = 0; q < gr->kernels_per_iter; ++q) count_launch();
        if (hs->converged) { converged = true; ++restarts; break; }
        if ((long long)mm >= N) { converged = true; ++restarts; break; }  // full space spanned: exact
        if (tol_rel > 0) {
            // split-precision operator: stop at its noise floor (no real progress)
            if (restarts > 0 && hs->resid > 0.5 * prev_resid) { ++restarts; break; }
            prev_resid = hs->resid;
        }
    }
    // the Ritz vector V y is a unit vector already (orthonormal V, unit y)
    if (out) {
        out->theta = hs->theta;
        out->theta2 = hs->theta2;
        out->resid = hs->resid;
        out->matvecs = hs->matvecs;
        out->restarts = restarts;
        out->converged = converged ? 1 : 0;
    }
    if (!std::isfinite(hs->theta)) {
        set_error("lanczos: non-finite Ritz value");
        return TN_NAN_DETECTED;
    }
    return TN_OK;
}

// Records the enqueue calls of `fn` on stream st into graph g after the nodes
// deps; returns the capture's final frontier in `front` (when non-null).
template <class F>
int capture_into(cudaStream_t st, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, F&& fn,
                 std::vector<cudaGraphNode_t>* front) {
    TN_CUDA_CHECK(cudaStreamBeginCaptureToGraph(st, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                                cudaStreamCaptureModeRelaxed));
    int rc = fn();
    if (rc == TN_OK && front) {
        cudaStreamCaptureStatus status;
        const cudaGraphNode_t* d = nullptr;
        size_t nd = 0;
        if (cudaStreamGetCaptureInfo(st, &status, nullptr, nullptr, &d, &nd) != cudaSuccess) rc = TN_CUDA_ERROR;
        else front->assign(d, d + nd);
    }
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &out);
    if (rc != TN_OK) return rc;
    TN_CUDA_CHECK(e);
    return TN_OK;
}

// Adds a WHILE conditional node (handle created on `owner`, default 1) after
// deps; returns the node and its body graph.
int add_while(cudaGraph_t owner, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
              cudaGraphConditionalHandle* h, cudaGraphNode_t* node, cudaGraph_t* body) {
    TN_CUDA_CHECK(cudaGraphConditionalHandleCreate(h, owner, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = *h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    TN_CUDA_CHECK(cudaGraphAddNode(node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &cp));
    *body = cp.conditional.phGraph_out[0];
    return TN_OK;
}

int lanczos_solve_async(Ctx& c, long long N, double* x, int m, int maxRestarts, double tol, const MatvecFn& mv,
                        double tol_rel, unsigned long long graph_key, LzSummary* host_out, const VecSplit* split) {
    const VecSplit sp = split ? *split : VecSplit{};
    cudaStream_t st = c.stream;
    if (!graph_key || !c.use_graphs || st == nullptr || c.prof || N <= 0) return LZ_ASYNC_UNAVAILABLE;
    int mm = std::min(m, LZ_MAXK - 1);
    if ((long long)mm > N) mm = (int)N;
    if (mm < 1) mm = 1;
    const int maxR = maxRestarts > 0 ? maxRestarts : 1;
    const int grid = vec_grid(N, c.sm_count);
    // workspace: V (mm+1 vectors), w, xcur, the solve's copy of x, partials
    size_t need = sizeof(double) * ((size_t)(mm + 4) * N + partial_doubles(N, c.sm_count) + 64);
    TN_CHECK(c.lz.ensure(need));
    TN_CHECK(c.lzstate.ensure(sizeof(LzState)));
    TN_CHECK(c.lzsum.ensure(sizeof(LzSummary)));
    double* V = c.lz.as<double>();
    double* w = V + (size_t)(mm + 1) * N;
    double* xcur = w + N;
    double* xw = xcur + N;
    double* partial = xw + N;
    LzState* s = c.lzstate.as<LzState>();
    LzSummary* sum = c.lzsum.as<LzSummary>();
    unsigned long long key = hash_val(graph_key, 0x6e65737465644c5aULL);
    for (unsigned long long v : {(unsigned long long)N, (unsigned long long)mm, (unsigned long long)maxR,
                                 (unsigned long long)grid, alloc_generation()})
        key = hash_val(key, v);
    key = hash_val(key, tol);
    key = hash_val(key, tol_rel);
    key = hash_val(key, (const void*)V);
    key = hash_val(key, (const void*)s);
    key = hash_val(key, (const void*)sp.out);
    key = hash_val(key, st);
    auto it = c.lzgraphs.find(key);
    if (it == c.lzgraphs.end()) {
        if (c.lzgraphs.size() >= 1024) c.clear_graphs();
        LzGraph g;
        TN_CUDA_CHECK(cudaGraphCreate(&g.graph, 0));
        // whatever fails while the graph is built, the caller falls back to the host-driven loop
        auto fail = [&](int) {
            cudaGraphDestroy(g.graph);
            cudaGetLastError();
            return LZ_ASYNC_UNAVAILABLE;
        };
        std::vector<cudaGraphNode_t> front;
        // the whole solve's reset
        int rc = capture_into(st, g.graph, {}, [&]() -> int {
            lz_reset_kernel<<<1, 32, 0, st>>>(s, tol, tol_rel, 1, mm);
            return cudaGetLastError() == cudaSuccess ? TN_OK : TN_CUDA_ERROR;
        }, &front);
        if (rc != TN_OK) return fail(rc);
        cudaGraphConditionalHandle h_out, h_in;
        cudaGraphNode_t n_out, n_in;
        cudaGraph_t b_out, b_in;
        if (add_while(g.graph, g.graph, front, &h_out, &n_out, &b_out) != TN_OK) return fail(TN_OK);
        // a restart: reset (re-arming the steps loop), v0 = x / |x|, the steps, the Ritz vector, the decision
        if (cudaGraphConditionalHandleCreate(&h_in, g.graph, 1, cudaGraphCondAssignDefault) != cudaSuccess)
            return fail(TN_OK);
        rc = capture_into(st, b_out, {}, [&]() -> int {
            lz_reset_kernel<<<1, 32, 0, st>>>(s, tol, tol_rel, 0, mm, h_in);
            lz_norm_kernel<<<grid, LZ_THREADS, 0, st>>>(xw, N, partial, s);
            lz_scale_kernel<<<grid, LZ_THREADS, 0, st>>>(xw, V, N, s, 1, xcur, sp);
            return cudaGetLastError() == cudaSuccess ? TN_OK : TN_CUDA_ERROR;
        }, &front);
        if (rc != TN_OK) return fail(rc);
        {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h_in;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            if (cudaGraphAddNode(&n_in, b_out, front.data(), front.size(), &cp) != cudaSuccess) return fail(TN_OK);
            b_in = cp.conditional.phGraph_out[0];
        }
        const unsigned long long n0 = launch_count();
        rc = capture_into(st, b_in, {}, [&]() -> int {
            return enqueue_lz_step(c, mv, grid, V, w, xcur, N, partial, s, sp, h_in);
        }, nullptr);
        const unsigned long long kpi = launch_count() - n0;
        if (rc != TN_OK) return fail(rc);
        rc = capture_into(st, b_out, {n_in}, [&]() -> int {
            lz_ritz_coeffs_kernel<<<1, LZ_THREADS, 0, st>>>(s);
            lz_ritz_vector_kernel<<<grid, LZ_THREADS, 0, st>>>(V, xw, N, s);
            lz_decide_kernel<<<1, 32, 0, st>>>(s, h_out, maxR, N, mm);
            return cudaGetLastError() == cudaSuccess ? TN_OK : TN_CUDA_ERROR;
        }, nullptr);
        if (rc != TN_OK) return fail(rc);
        // the summary (the Ritz vector V y is a unit vector already)
        rc = capture_into(st, g.graph, {n_out}, [&]() -> int {
            lz_summary_kernel<<<1, 32, 0, st>>>(s, sum, (int)kpi);
            return cudaGetLastError() == cudaSuccess ? TN_OK : TN_CUDA_ERROR;
        }, nullptr);
        if (rc != TN_OK) return fail(rc);
        if (cudaGraphInstantiate(&g.exec, g.graph, 0) != cudaSuccess) return fail(TN_OK);
        g.kernels_per_iter = kpi;
        it = c.lzgraphs.emplace(key, g).first;
    }
    TN_CUDA_CHECK(cudaMemcpyAsync(xw, x, sizeof(double) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    TN_CUDA_CHECK(cudaGraphLaunch(it->second.exec, st));
    TN_CUDA_CHECK(cudaMemcpyAsync(x, xw, sizeof(double) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    TN_CUDA_CHECK(cudaMemcpyAsync(host_out, sum, sizeof(LzSummary), cudaMemcpyDeviceToHost, st));
    return TN_OK;
}

int rayleigh_residual(Ctx& c, long long N, const double* x, const double* y, double* theta, double* resid) {
    cudaStream_t st = c.stream;
    const int grid = vec_grid(N, c.sm_count);
    TN_CHECK(c.rq.ensure(sizeof(double) * (2 * (size_t)grid + 8) + sizeof(LzState)));
    LzState* s = reinterpret_cast<LzState*>(c.rq.p);
    double* partial = reinterpret_cast<double*>(c.rq.as<char>() + sizeof(LzState));
    TN_CHECK(c.pinned.ensure(sizeof(LzState)));
    TN_CUDA_CHECK(cudaMemsetAsync(&s->counter, 0, sizeof(unsigned int), st));
    rq_dots_kernel<<<grid, LZ_THREADS, 0, st>>>(x, y, N, partial, s);
    TN_LAUNCH_CHECK();
    rq_resid_kernel<<<grid, LZ_THREADS, 0, st>>>(x, y, N, partial, s);
    TN_LAUNCH_CHECK();
    LzState* hs = reinterpret_cast<LzState*>(c.pinned.p);
    TN_CUDA_CHECK(cudaMemcpyAsync(hs, s, sizeof(LzState), cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    *theta = hs->theta;
    *resid = hs->resid;
    return TN_OK;
}

size_t rayleigh_scratch_bytes(long long N, int sm_count) {
    return sizeof(LzState) + sizeof(double) * (2 * (size_t)vec_grid(N, sm_count) + 8);
}

int rayleigh_residual_async(cudaStream_t st, int sm_count, long long N, const double* x, const double* y, void* dev,
                            double* host_out) {
    const int grid = vec_grid(N, sm_count);
    LzState* s = reinterpret_cast<LzState*>(dev);
    double* partial = reinterpret_cast<double*>(reinterpret_cast<char*>(dev) + sizeof(LzState));
    TN_CUDA_CHECK(cudaMemsetAsync(&s->counter, 0, sizeof(unsigned int), st));
    rq_dots_kernel<<<grid, LZ_THREADS, 0, st>>>(x, y, N, partial, s);
    TN_LAUNCH_CHECK();
    rq_resid_kernel<<<grid, LZ_THREADS, 0, st>>>(x, y, N, partial, s);
    TN_LAUNCH_CHECK();
    static_assert(offsetof(LzState, theta2) == offsetof(LzState, theta) + sizeof(double) &&
                      offsetof(LzState, resid) == offsetof(LzState, theta) + 2 * sizeof(double),
                  "theta, theta2, resid are adjacent");
    TN_CUDA_CHECK(cudaMemcpyAsync(host_out, &s->theta, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    return TN_OK;
}

}  // namespace tnb
