// svd.cu -- one-sided (Hestenes) Jacobi SVD in FP64, one CTA per matrix.
//
// Replaces LapackSVDSolver<T>::Solve (zgesvd, LapackSVDSolver.C:42-90).  The
// columns of the tall working matrix are orthogonalised pairwise; pairs follow
// the round-robin (circle) ordering so that all n/2 pairs of a round are
// independent and run on different warps; rotation angles, dot products and
// convergence tests are FP64.  Small problems run entirely in shared memory.
// Singular values come out descending; zero singular values get orthonormal
// completion columns in U (as zgesvd provides), which the zero-padded bond
// growth of the sweep relies on.  A batch of matrices runs as one launch.
#include <algorithm>

#include "qr.h"

namespace tnb {

namespace {

constexpr int SVD_THREADS = 512;
constexpr int SVD_MAX_SWEEPS = 60;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int rr_pos(int q, int r, int ne) {
    return q == 0 ? 0 : ((q - 1 + r) % (ne - 1)) + 1;
}

__global__ void __launch_bounds__(SVD_THREADS) jacobi_svd_kernel(const SvdJob* __restrict__ jobs, int vectors,
                                                                   size_t smem_cap) {
    extern __shared__ double smem[];
    const SvdJob jb = jobs[blockIdx.x];
    const int m = jb.m, n = jb.n;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    __shared__ int s_rot;
    __shared__ int s_sweeps;
    __shared__ double red[32];

    // shared memory: norms (n), ranks (n ints), then A (m x n) and V (n x n) when they fit
    double* norms = smem;
    int* rank = reinterpret_cast<int*>(smem + n);
    double* tail = smem + n + (n + 1) / 2 + 1;
    size_t fixed = (size_t)n + (n + 1) / 2 + 1;
    size_t need = fixed + (size_t)m * n + (vectors ? (size_t)n * n : 0);
    bool in_smem = need * sizeof(double) <= smem_cap;
    double* A = in_smem ? tail : jb.W;
    double* V = vectors ? (in_smem ? tail + (size_t)m * n : jb.V) : nullptr;
    if (in_smem)
        for (size_t e = tid; e < (size_t)m * n; e += blockDim.x) A[e] = jb.W[e];
    if (vectors)
        for (size_t e = tid; e < (size_t)n * n; e += blockDim.x) V[e] = ((e % n) == (e / n)) ? 1.0 : 0.0;
    __syncthreads();

    const int ne = n + (n & 1);
    const double tol = 1e-15 * fmax(1.0, sqrt((double)m) / 4.0);
    int sweep = 0;
    for (sweep = 0; sweep < SVD_MAX_SWEEPS && n > 1; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        for (int r = 0; r < ne - 1; ++r) {
            for (int p = wid; p < ne / 2; p += nw) {
                int a = rr_pos(p, r, ne), b = rr_pos(ne - 1 - p, r, ne);
                if (a >= n || b >= n) continue;
                double* ca = A + (size_t)a * m;
                double* cb = A + (size_t)b * m;
                double al = 0, be = 0, ga = 0;
                for (int i = lane; i < m; i += 32) {
                    double x = ca[i], y = cb[i];
                    al = fma(x, x, al);
                    be = fma(y, y, be);
                    ga = fma(x, y, ga);
                }
                al = wsum(al);
                be = wsum(be);
                ga = wsum(ga);
                if (ga == 0.0 || fabs(ga) <= tol * sqrt(al * be)) continue;
                double zeta = (be - al) / (2.0 * ga);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                for (int i = lane; i < m; i += 32) {
                    double x = ca[i], y = cb[i];
                    ca[i] = c * x - s * y;
                    cb[i] = s * x + c * y;
                }
                if (vectors) {
                    double* va = V + (size_t)a * n;
                    double* vb = V + (size_t)b * n;
                    for (int i = lane; i < n; i += 32) {
                        double x = va[i], y = vb[i];
                        va[i] = c * x - s * y;
                        vb[i] = s * x + c * y;
                    }
                }
                if (lane == 0) s_rot = 1;
            }
            __syncthreads();
        }
        int rot = s_rot;
        __syncthreads();
        if (!rot) break;
    }
    if (tid == 0) s_sweeps = sweep;

    // column norms = singular values (unsorted)
    for (int j = wid; j < n; j += nw) {
        const double* cj = A + (size_t)j * m;
        double s = 0;
        for (int i = lane; i < m; i += 32) s = fma(cj[i], cj[i], s);
        s = wsum(s);
        if (lane == 0) norms[j] = sqrt(s);
    }
    __syncthreads();
    // descending rank, ties broken by column index
    for (int j = tid; j < n; j += blockDim.x) {
        double sj = norms[j];
        int rk = 0;
        for (int i = 0; i < n; ++i) {
            double si = norms[i];
            rk += (si > sj) || (si == sj && i < j);
        }
        rank[j] = rk;
        jb.s[rk] = sj;
    }
    __syncthreads();
    double smax = 0;
    for (int j = 0; j < n; ++j) smax = fmax(smax, norms[j]);
    const double cut = smax * 1e-13 * fmax(1.0, (double)m);
    if (vectors) {
        for (int j = wid; j < n; j += nw) {
            const int rk = rank[j];
            const double sj = norms[j];
            const double* cj = A + (size_t)j * m;
            double* uo = jb.U + (size_t)rk * jb.ldu;
            const bool good = sj > cut && sj > 0.0;
            for (int i = lane; i < m; i += 32) uo[i] = good ? cj[i] / sj : 0.0;
            const double* vj = V + (size_t)j * n;
            for (int i = lane; i < n; i += 32) jb.Vt[(size_t)i * jb.ldvt + rk] = vj[i];
        }
        __syncthreads();
        // orthonormal completion of U columns whose singular value is below the cut:
        // unit vectors, Gram-Schmidt (twice) against every accepted column
        int next_e = 0;
        for (int c = 0; c < n; ++c) {
            double sc = __ldcg(jb.s + c);
            if (sc > cut && sc > 0.0) continue;
            double* uc = jb.U + (size_t)c * jb.ldu;
            bool placed = false;
            while (!placed && next_e < m) {
                const int e = next_e++;
                for (int i = tid; i < m; i += blockDim.x) uc[i] = (i == e) ? 1.0 : 0.0;
                __syncthreads();
                for (int pass = 0; pass < 2; ++pass) {
                    for (int p = 0; p < n; ++p) {
                        if (p == c) continue;
                        double sp = __ldcg(jb.s + p);
                        if (!((sp > cut && sp > 0.0) || p < c)) continue;
                        const double* up = jb.U + (size_t)p * jb.ldu;
                        double part = 0;
                        for (int i = tid; i < m; i += blockDim.x) part = fma(up[i], uc[i], part);
                        part = wsum(part);
                        if (lane == 0) red[wid] = part;
                        __syncthreads();
                        double dotv = 0;
                        for (int w = 0; w < nw; ++w) dotv += red[w];
                        __syncthreads();
                        for (int i = tid; i < m; i += blockDim.x) uc[i] = fma(-dotv, up[i], uc[i]);
                        __syncthreads();
                    }
                }
                double part = 0;
                for (int i = tid; i < m; i += blockDim.x) part = fma(uc[i], uc[i], part);
                part = wsum(part);
                if (lane == 0) red[wid] = part;
                __syncthreads();
                double nr2 = 0;
                for (int w = 0; w < nw; ++w) nr2 += red[w];
                __syncthreads();
                double nr = sqrt(nr2);
                if (nr > 0.5) {
                    for (int i = tid; i < m; i += blockDim.x) uc[i] /= nr;
                    placed = true;
                }
                __syncthreads();
            }
        }
    }
    if (tid == 0 && jb.sweeps) *jb.sweeps = s_sweeps;
}

}  // namespace

int svd_batched(Ctx& c, const std::vector<SvdJob>& jobs, bool vectors) {
    if (jobs.empty()) return TN_OK;
    for (const auto& j : jobs) {
        if (j.m < j.n || j.n < 1) {
            set_error("svd: job needs m >= n >= 1 (got %d x %d)", j.m, j.n);
            return TN_BAD_SHAPE;
        }
        if ((size_t)j.n * 12 + 64 > 200 * 1024) {
            set_error("svd: n too large for the single-CTA Jacobi kernel (%d)", j.n);
            return TN_BAD_SHAPE;
        }
    }
    TN_CHECK(c.svdw.ensure(sizeof(SvdJob) * jobs.size()));
    TN_CUDA_CHECK(cudaMemcpyAsync(c.svdw.p, jobs.data(), sizeof(SvdJob) * jobs.size(), cudaMemcpyHostToDevice,
                                  c.stream));
    const size_t cap = 200 * 1024;
    TN_CUDA_CHECK(cudaFuncSetAttribute(jacobi_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
    jacobi_svd_kernel<<<(unsigned)jobs.size(), SVD_THREADS, cap, c.stream>>>(c.svdw.as<SvdJob>(), vectors ? 1 : 0,
                                                                             cap);
    TN_LAUNCH_CHECK();
    // the job array must stay valid until the kernel has read it
    TN_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return TN_OK;
}

}  // namespace tnb
