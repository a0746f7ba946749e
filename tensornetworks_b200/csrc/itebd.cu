// itebd.cu -- iTEBD gates path on the device (Vidal form, two-site unit cell).
//
// Follows the reference's gate application (iTEBDStateImp::Apply(MultigateType),
// TensorNetworksImp/iTEBD/iTEBDStateImp_iTime.C:119-135):
//   theta = lB GA[ma] lA GB[mb] lB                (ContractTheta lAlBl,
//                                                  iTEBDStateImp_Contractions.C:24-84)
//   theta'[na,nb] = sum_{ma,mb} expH(ma,na,mb,nb) theta[ma,mb]
//   M(i + Dl na, j + Dl nb) = theta'[na,nb](i, j) (ReshapeForSVD, iTEBDStateImp_OrthoNorm.C:24-42)
//   M = U s Vt (one-sided Jacobi), SVCompressor rule (SVCompressorImp.C:19-73),
//   lA = s / |s| (Bond::SetSingularValues), GA = lB^-1 U, GB = Vt lB^-1
//                                                 (Unpack, iTEBDStateImp_OrthoNorm.C:205-270)
// with the gates of the second-order Trotter step (iTEBDGates::InitGates,
// iTEBDGates.C:21-54) and the alternating centre (ReCenter).  The contractions
// are batched FP64 GEMMs, the SVD is the library's Jacobi SVD; only the
// truncation decision (a few doubles) goes through the host.
//
// The energy per bond is the infinite-chain expectation: left and right fixed
// points of the unit-cell transfer matrix by power iteration (FP64 GEMMs),
// then <l| sum h (B_p (x) B_q) |r> / <l| sum B_p (x) B_p |r> for both bonds.
#include "itebd.h"

#include <algorithm>
#include <cmath>
#include <random>

#include "qr.h"

namespace tnb {

namespace {

inline int g1d(long long n) {
    long long b = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(b, 148 * 8));
}

// out[n](i, j) = lrow[i] * G[n](i, j) * lcol[j]   (either scale may be null)
__global__ void scale_kernel(const double* __restrict__ G, int d, int Dl, int Dr, const double* __restrict__ lrow,
                             const double* __restrict__ lcol, double* __restrict__ out) {
    const long long total = (long long)d * Dl * Dr;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % Dl);
        const int j = (int)((e / Dl) % Dr);
        double v = G[e];
        if (lrow) v *= lrow[i];
        if (lcol) v *= lcol[j];
        out[e] = v;
    }
}

// M(i + Dl na, j + Dl nb) = sum_{ma,mb} gate[(ma d + mb) + (na d + nb) d^2] TH[(ma d + mb)](i, j)
__global__ void gate_reshape_kernel(const double* __restrict__ TH, int d, int Dl, const double* __restrict__ gate,
                                    double* __restrict__ M) {
    const int dd = d * d;
    const int m = d * Dl;
    const long long total = (long long)m * m;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e % m), c = (int)(e / m);
        const int i = r % Dl, na = r / Dl, j = c % Dl, nb = c / Dl;
        const int q = na * d + nb;
        double acc = 0;
        for (int p = 0; p < dd; ++p) acc = fma(gate[p + (size_t)q * dd], TH[(size_t)p * Dl * Dl + (size_t)j * Dl + i], acc);
        M[e] = acc;
    }
}

// GA[na](i, j) = U(i + Dl na, j) / lB[i]   (j < keep);  GB[nb](j, i) = Vt(j, i + Dl nb) / lB[i]
__global__ void unpack_kernel(const double* __restrict__ U, int ldu, const double* __restrict__ Vt, int ldvt, int d,
                              int Dl, int keep, const double* __restrict__ lB, double* __restrict__ GA,
                              double* __restrict__ GB) {
    const long long total = (long long)d * Dl * keep;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        // GA layout (d, Dl, keep): e = n*Dl*keep + j*Dl + i
        {
            const int i = (int)(e % Dl), j = (int)((e / Dl) % keep), n = (int)(e / ((long long)Dl * keep));
            GA[e] = U[(size_t)j * ldu + i + (size_t)Dl * n] / lB[i];
        }
        // GB layout (d, keep, Dl): e = n*keep*Dl + i*keep + j
        {
            const int j = (int)(e % keep), i = (int)((e / keep) % Dl), n = (int)(e / ((long long)Dl * keep));
            GB[e] = Vt[(size_t)(i + Dl * n) * ldvt + j] / lB[i];
        }
    }
}

// Frobenius normalisation of x (n <= a few thousand, one block); returns the norm in *nrm.
__global__ void normalize_kernel(double* __restrict__ x, int n, double* nrm) {
    __shared__ double sh[32];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(x[i], x[i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sh[0] = t;
    }
    __syncthreads();
    const double nr = sqrt(sh[0]);
    const double inv = nr > 0 ? 1.0 / nr : 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] *= inv;
    if (threadIdx.x == 0 && nrm) *nrm = nr;
}

// out[p*nq + q] = <C_p, E_q> (Frobenius) for p, q < dd; one block per pair
__global__ void pair_dots_kernel(const double* __restrict__ C, const double* __restrict__ E, int dd, int n,
                                 double* __restrict__ out) {
    const int p = blockIdx.x / dd, q = blockIdx.x % dd;
    __shared__ double sh[32];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(C[(size_t)p * n + i], E[(size_t)q * n + i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        out[blockIdx.x] = t;
    }
}

// |x - y|_max over n (one block), into *out
__global__ void maxdiff_kernel(const double* __restrict__ x, const double* __restrict__ y, int n, double* out) {
    __shared__ double sh[32];
    double m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(x[i] - y[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, sh[w]);
        *out = t;
    }
}

// M(i + D na, j + D nb) = lB[i] gam[na + d nb](i, j) lB[j]   (ReshapeForSVD of lambdaB gamma lambdaB)
__global__ void gamma_reshape_kernel(const double* __restrict__ gam, int d, int D, const double* __restrict__ lB,
                                     double* __restrict__ M) {
    const int m = d * D;
    const long long total = (long long)m * m;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e % m), c = (int)(e / m);
        const int i = r % D, na = r / D, j = c % D, nb = c / D;
        M[e] = lB[i] * gam[(size_t)(na + d * nb) * D * D + (size_t)j * D + i] * lB[j];
    }
}

// out = {Vr(0,0), Vl(0,0), min_i |Vr(i,i)|, min_i |Vl(i,i)|} (one block)
__global__ void norm_stats_kernel(const double* __restrict__ Vr, const double* __restrict__ Vl, int D, double* out) {
    __shared__ double sr[32], sl[32];
    double mr = 1e300, ml = 1e300;
    for (int i = threadIdx.x; i < D; i += blockDim.x) {
        mr = fmin(mr, fabs(Vr[(size_t)i * D + i]));
        ml = fmin(ml, fabs(Vl[(size_t)i * D + i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mr = fmin(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        ml = fmin(ml, __shfl_xor_sync(0xffffffffu, ml, o));
    }
    if ((threadIdx.x & 31) == 0) {
        sr[threadIdx.x >> 5] = mr;
        sl[threadIdx.x >> 5] = ml;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mr = fmin(mr, sr[w]);
            ml = fmin(ml, sl[w]);
        }
        out[0] = Vr[0];
        out[1] = Vl[0];
        out[2] = fmin(mr, sr[0]);
        out[3] = fmin(ml, sl[0]);
    }
}

// sq = sqrt(s), isq = 1/sqrt(s) for both factors; flag[0] = 1 when a value is not positive
__global__ void sqrt_pair_kernel(const double* __restrict__ sr, const double* __restrict__ sl, int D,
                                 double* __restrict__ out, double* flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D; i += gridDim.x * blockDim.x) {
        const double a = sr[i], b = sl[i];
        if (!(a > 1e-300) || !(b > 1e-300)) *flag = 1.0;
        out[i] = sqrt(a);
        out[D + i] = 1.0 / sqrt(a);
        out[2 * D + i] = sqrt(b);
        out[3 * D + i] = 1.0 / sqrt(b);
    }
}

__global__ void scal_kernel(double* __restrict__ x, long long n, double a) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        x[e] *= a;
}

// dst[n](i, j) = src[n](i, j) for i < Dl, j < Dr, else 0; dst is (d, D1, D2)
__global__ void pad_kernel(const double* __restrict__ src, int d, int Dl, int Dr, double* __restrict__ dst, int D1,
                           int D2) {
    const long long total = (long long)d * D1 * D2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % D1), j = (int)((e / D1) % D2), n = (int)(e / ((long long)D1 * D2));
        dst[e] = (i < Dl && j < Dr) ? src[(size_t)n * Dl * Dr + (size_t)j * Dl + i] : 0.0;
    }
}

// Symmetric eigen-decomposition by cyclic Jacobi (host, n <= 36): A = Q diag(w) Q^T.
void jacobi_eigh_host(std::vector<double> A, int n, std::vector<double>& w, std::vector<double>& Q) {
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += A[(size_t)q * n + p] * A[(size_t)q * n + p];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)q * n + p];
                if (std::fabs(apq) < 1e-300) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double tau = (aqq - app) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                const double c = 1 / std::sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double akp = A[(size_t)p * n + k], akq = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * akp - s * akq;
                    A[(size_t)q * n + k] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double apk = A[(size_t)k * n + p], aqk = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * apk - s * aqk;
                    A[(size_t)k * n + q] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double qkp = Q[(size_t)p * n + k], qkq = Q[(size_t)q * n + k];
                    Q[(size_t)p * n + k] = c * qkp - s * qkq;
                    Q[(size_t)q * n + k] = s * qkp + c * qkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = A[(size_t)i * n + i];
}

double spin_op(int which, int m, int n, double S) {
    // basis m = 0..d-1 with Sz = S - m; which: 0 Sz, 1 S+, 2 S-
    const double mz = S - m, nz = S - n;
    if (which == 0) return m == n ? mz : 0.0;
    if (which == 1) return (mz == nz + 1) ? std::sqrt(S * (S + 1) - nz * (nz + 1)) : 0.0;
    return (mz == nz - 1) ? std::sqrt(S * (S + 1) - nz * (nz - 1)) : 0.0;
}

}  // namespace

int ITebdState::init(Ctx& c, double S_, double Jxy_, double Jz_, double hz_, int D, unsigned long long seed) {
    ctx = &c;
    S = S_;
    Jxy = Jxy_;
    Jz = Jz_;
    hz = hz_;
    d = (int)std::lround(2 * S + 1);
    if (d < 2 || D < 1) return TN_BAD_ARG;
    // two-site Hamiltonian (Hamiltonian_1D_NN_Heisenberg::GetH convention: the
    // field term on both sites of the bond), rows (ma d + mb), columns (na d + nb)
    const int dd = d * d;
    h12.assign((size_t)dd * dd, 0.0);
    for (int ma = 0; ma < d; ++ma)
        for (int mb = 0; mb < d; ++mb)
            for (int na = 0; na < d; ++na)
                for (int nb = 0; nb < d; ++nb) {
                    const double v = 0.5 * Jxy * (spin_op(1, ma, na, S) * spin_op(2, mb, nb, S) +
                                                  spin_op(2, ma, na, S) * spin_op(1, mb, nb, S)) +
                                     Jz * spin_op(0, ma, na, S) * spin_op(0, mb, nb, S) +
                                     hz * (spin_op(0, ma, na, S) * (mb == nb) + (ma == na) * spin_op(0, mb, nb, S));
                    h12[(size_t)(na * d + nb) * dd + (ma * d + mb)] = v;
                }
    // uniform(-1,1) Gammas from a seeded generator, flat bond values
    std::mt19937_64 g(seed);
    for (int s = 0; s < 2; ++s) {
        const size_t n = (size_t)d * D * D;
        std::vector<double> h(n);
        for (auto& x : h) x = ((g() >> 11) * (1.0 / 9007199254740992.0)) * 2 - 1;
        TN_CHECK(G[s].ensure(sizeof(double) * n));
        TN_CUDA_CHECK(cudaMemcpy(G[s].p, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        lam_h[s].assign(D, 1.0 / std::sqrt((double)D));
        TN_CHECK(lam[s].ensure(sizeof(double) * D));
        TN_CUDA_CHECK(cudaMemcpy(lam[s].p, lam_h[s].data(), sizeof(double) * D, cudaMemcpyHostToDevice));
    }
    return TN_OK;
}

int ITebdState::set_gate(double dt) {
    const int dd = d * d;
    std::vector<double> w, Q;
    jacobi_eigh_host(h12, dd, w, Q);
    std::vector<double> Gt((size_t)dd * dd, 0.0);
    for (int r = 0; r < dd; ++r)
        for (int c = 0; c < dd; ++c) {
            double s = 0;
            for (int k = 0; k < dd; ++k) s += Q[(size_t)k * dd + r] * std::exp(-dt * w[k]) * Q[(size_t)k * dd + c];
            Gt[(size_t)c * dd + r] = s;
        }
    TN_CHECK(gate.ensure(sizeof(double) * dd * dd));
    TN_CUDA_CHECK(cudaMemcpyAsync(gate.p, Gt.data(), sizeof(double) * dd * dd, cudaMemcpyHostToDevice, ctx->stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    return TN_OK;
}

int ITebdState::apply_gate(int bond, int Dmax, double eps) {
    cudaStream_t st = ctx->stream;
    const int A = bond, B = 1 - bond;  // site A sits left of `bond`
    const int Dl = dim(B), Dm = dim(bond);
    const int dd = d * d;
    const int m = d * Dl;
    // X[ma] = lB GA[ma] lA (Dl x Dm), Y[mb] = GB[mb] lB (Dm x Dl)
    TN_CHECK(X.ensure(sizeof(double) * (size_t)d * Dl * Dm));
    TN_CHECK(Y.ensure(sizeof(double) * (size_t)d * Dm * Dl));
    TN_CHECK(TH.ensure(sizeof(double) * (size_t)dd * Dl * Dl));
    TN_CHECK(M.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(U.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(Vt.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(V.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(s.ensure(sizeof(double) * (size_t)m));
    scale_kernel<<<g1d((long long)d * Dl * Dm), 256, 0, st>>>(G[A].as<double>(), d, Dl, Dm, lam[B].as<double>(),
                                                              lam[bond].as<double>(), X.as<double>());
    TN_LAUNCH_CHECK();
    scale_kernel<<<g1d((long long)d * Dm * Dl), 256, 0, st>>>(G[B].as<double>(), d, Dm, Dl, nullptr,
                                                              lam[B].as<double>(), Y.as<double>());
    TN_LAUNCH_CHECK();
    // TH[ma d + mb] = X[ma] Y[mb]
    GemmArgs g;
    g.M = Dl; g.N = Dl; g.K = Dm; g.nb0 = d; g.nb1 = d;
    g.A.ptr = X.as<double>(); g.A.mn = idx(1); g.A.k = idx(Dl); g.A.sb0 = (long long)Dl * Dm; g.A.sb1 = 0;
    g.B.ptr = Y.as<double>(); g.B.k = idx(1); g.B.mn = idx(Dm); g.B.sb0 = 0; g.B.sb1 = (long long)Dm * Dl;
    g.C.ptr = TH.as<double>(); g.C.m = idx(1); g.C.n = idx(Dl); g.C.sb0 = (long long)d * Dl * Dl;
    g.C.sb1 = (long long)Dl * Dl;
    TN_CHECK(gemm_f64(g, st));
    gate_reshape_kernel<<<g1d((long long)m * m), 256, 0, st>>>(TH.as<double>(), d, Dl, gate.as<double>(),
                                                               M.as<double>());
    TN_LAUNCH_CHECK();
    TN_CHECK(svd_unpack(bond, Dl, Dmax, eps));
    ++gates_applied;
    return TN_OK;
}

int ITebdState::svd_unpack(int bond, int Dl, int Dmax, double eps) {
    cudaStream_t st = ctx->stream;
    const int A = bond, B = 1 - bond;
    const int m = d * Dl;
    TN_CHECK(U.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(Vt.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(V.ensure(sizeof(double) * (size_t)m * m));
    TN_CHECK(s.ensure(sizeof(double) * (size_t)m));
    SvdJob job{M.as<double>(), m, m, V.as<double>(), U.as<double>(), m, Vt.as<double>(), m, s.as<double>(), nullptr};
    TN_CHECK(svd_batched(*ctx, {job}, true));
    // SVCompressor rule on the host (a few values), then lambda normalised
    std::vector<double> sv(m);
    TN_CUDA_CHECK(cudaMemcpy(sv.data(), s.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
    int keep = m;
    if (eps > 0) {
        double tail = 0;
        for (keep = m; keep >= 2; --keep) {
            const double s2 = sv[keep - 1] * sv[keep - 1];
            if (tail + s2 >= eps) break;
            tail += s2;
        }
        if (Dmax > 0) keep = std::min(keep, Dmax);
    } else if (Dmax > 0) {
        keep = std::min(m, Dmax);
    }
    while (keep > 1 && !(sv[keep - 1] > 0)) --keep;  // the inverse bond values must stay finite
    double nrm = 0;
    for (int i = 0; i < keep; ++i) nrm += sv[i] * sv[i];
    nrm = std::sqrt(nrm);
    lam_h[bond].assign(sv.begin(), sv.begin() + keep);
    for (double& x : lam_h[bond]) x /= nrm;
    TN_CHECK(lam[bond].ensure(sizeof(double) * keep));
    TN_CUDA_CHECK(cudaMemcpyAsync(lam[bond].p, lam_h[bond].data(), sizeof(double) * keep, cudaMemcpyHostToDevice, st));
    // new Gammas: A (d, Dl, keep), B (d, keep, Dl)
    TN_CHECK(work.ensure(sizeof(double) * 2 * (size_t)d * Dl * keep));
    double* GA = work.as<double>();
    double* GB = GA + (size_t)d * Dl * keep;
    unpack_kernel<<<g1d((long long)d * Dl * keep), 256, 0, st>>>(U.as<double>(), m, Vt.as<double>(), m, d, Dl, keep,
                                                                 lam[B].as<double>(), GA, GB);
    TN_LAUNCH_CHECK();
    TN_CHECK(G[A].ensure(sizeof(double) * (size_t)d * Dl * keep));
    TN_CHECK(G[B].ensure(sizeof(double) * (size_t)d * Dl * keep));
    TN_CUDA_CHECK(cudaMemcpyAsync(G[A].p, GA, sizeof(double) * (size_t)d * Dl * keep, cudaMemcpyDeviceToDevice, st));
    TN_CUDA_CHECK(cudaMemcpyAsync(G[B].p, GB, sizeof(double) * (size_t)d * Dl * keep, cudaMemcpyDeviceToDevice, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    return TN_OK;
}

int ITebdState::step2(double dt, int Dmax) {
    TN_CHECK(set_gate(0.5 * dt));
    TN_CHECK(apply_gate(0, 0, 1e-7));
    TN_CHECK(set_gate(dt));
    TN_CHECK(apply_gate(1, Dmax, 1e-16));
    TN_CHECK(set_gate(0.5 * dt));
    TN_CHECK(apply_gate(0, Dmax, 1e-16));
    return TN_OK;
}

// iTEBDStateImp::OrthogonalizeI(comp, eps, niter), iTEBDStateImp_OrthoNorm.C:110-128,
// with the iteration of :511-637 (Phien, McCulloch, Vidal, PRB 91, 115137):
//   gamma[na + d nb] = GA[na] lA GB[nb]                  (ContractAlB)
//   repeat: Vr = sum_n (g_n l)(g_n l)^T, Vl = sum_n (l g_n)^T (l g_n) (GetNormMatrix),
//           bail when a diagonal is below 1e-10, Vr /= Vr(0,0), Vl /= Vl(0,0),
//           g /= sqrt(Vl(0,0)), Vr = X X^T, Vl = Yd Yd^T (Factor), SVD of
//           Yd^T l X = U l' VT, l' normalised, g_n = (VT X^-1) g_n (Yd^-T U),
//           until max |l - l'| < eps;  g /= sqrt(Vr(0,0))
//   lambdaB = l (normalised), then UnpackOrthonormal: lB g lB reshaped and
//   SVD-split into GA lA GB with the (Dmax, 1e-16) compressor.
// Factor takes the eigen-decomposition of the symmetric positive matrix; here
// it is the Jacobi SVD of that matrix (the same U and values), so the FP64
// rotations stay on the device.
int ITebdState::orthogonalize_i(int Dmax, double eps, int max_iter, double* delta, int* iters, bool* bailed) {
    cudaStream_t st = ctx->stream;
    const int D = dim(1), Dm = dim(0);
    const int dd = d * d;
    const size_t D2 = (size_t)D * D, nG = (size_t)dd * D2;
    if (delta) *delta = 0;
    if (iters) *iters = 0;
    if (bailed) *bailed = false;
    // workspace
    const size_t need = 2 * nG + 20 * D2 + 12 * (size_t)D + 16;
    TN_CHECK(og.ensure(sizeof(double) * need));
    double* gam = og.as<double>();
    double* tmp = gam + nG;
    double* Vr = tmp + nG;
    double* Vl = Vr + D2;
    double* Wr = Vl + D2;
    double* Wl = Wr + D2;
    double* Vwr = Wl + D2;
    double* Vwl = Vwr + D2;
    double* Ur = Vwl + D2;
    double* Ul = Ur + D2;
    double* Vtr = Ul + D2;
    double* Vtl = Vtr + D2;
    double* Z = Vtl + D2;
    double* Ys = Z + D2;
    double* YlX = Ys + D2;
    double* Vwy = YlX + D2;
    double* Up = Vwy + D2;
    double* VTp = Up + D2;
    double* Ri = VTp + D2;
    double* Li = Ri + D2;
    double* VX = Li + D2;
    double* YU = VX + D2;
    double* sr = YU + D2;
    double* sl = sr + D;
    double* sqv = sl + D;          // 4 D: sqrt(sr), 1/sqrt(sr), sqrt(sl), 1/sqrt(sl)
    double* lp = sqv + 4 * (size_t)D;
    double* lamv = lp + D;
    double* stats = lamv + D;      // 8 values
    auto gemm = [&](int M_, int N_, int K_, const double* a, IdxMap amn, IdxMap ak, const double* b, IdxMap bk,
                    IdxMap bmn, double* c) {
        GemmArgs g;
        g.M = M_; g.N = N_; g.K = K_;
        g.A.ptr = a; g.A.mn = amn; g.A.k = ak;
        g.B.ptr = b; g.B.k = bk; g.B.mn = bmn;
        g.C.ptr = c; g.C.m = idx(1); g.C.n = idx(M_);
        return gemm_f64(g, st);
    };
    // gamma[na + d nb] = (GA[na] lA) GB[nb]
    TN_CHECK(X.ensure(sizeof(double) * (size_t)d * D * Dm));
    scale_kernel<<<g1d((long long)d * D * Dm), 256, 0, st>>>(G[0].as<double>(), d, D, Dm, nullptr,
                                                             lam[0].as<double>(), X.as<double>());
    TN_LAUNCH_CHECK();
    {
        GemmArgs g;
        g.M = D; g.N = D; g.K = Dm; g.nb0 = d; g.nb1 = d;
        g.A.ptr = X.as<double>(); g.A.mn = idx(1); g.A.k = idx(D); g.A.sb0 = (long long)D * Dm; g.A.sb1 = 0;
        g.B.ptr = G[1].as<double>(); g.B.k = idx(1); g.B.mn = idx(Dm); g.B.sb0 = 0; g.B.sb1 = (long long)Dm * D;
        g.C.ptr = gam; g.C.m = idx(1); g.C.n = idx(D); g.C.sb0 = (long long)D2; g.C.sb1 = (long long)d * D2;
        TN_CHECK(gemm_f64(g, st));
    }
    TN_CUDA_CHECK(cudaMemcpyAsync(lamv, lam[1].p, sizeof(double) * D, cudaMemcpyDeviceToDevice, st));
    double er = 1.0;
    bool bail = false;
    int it = 0;
    double dl = 0.0;
    for (it = 0; it < max_iter; ++it) {
        // norm matrices
        scale_kernel<<<g1d((long long)nG), 256, 0, st>>>(gam, dd, D, D, nullptr, lamv, tmp);
        TN_LAUNCH_CHECK();
        TN_CHECK(gemm(D, D, dd * D, tmp, idx(1), idx2(D, D, (long long)D2), tmp, idx2(D, D, (long long)D2), idx(1), Vr));
        scale_kernel<<<g1d((long long)nG), 256, 0, st>>>(gam, dd, D, D, lamv, nullptr, tmp);
        TN_LAUNCH_CHECK();
        TN_CHECK(gemm(D, D, dd * D, tmp, idx(D), idx2(1, D, (long long)D2), tmp, idx2(1, D, (long long)D2), idx(D), Vl));
        norm_stats_kernel<<<1, 256, 0, st>>>(Vr, Vl, D, stats);
        TN_LAUNCH_CHECK();
        double hs[4];
        TN_CUDA_CHECK(cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, st));
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        if (!(hs[2] >= 1e-10) || !(hs[3] >= 1e-10)) {  // singular: bail out (as :547-554)
            bail = true;
            break;
        }
        er = hs[0];
        const double el = hs[1];
        scal_kernel<<<g1d((long long)D2), 256, 0, st>>>(Vr, (long long)D2, 1.0 / er);
        TN_LAUNCH_CHECK();
        scal_kernel<<<g1d((long long)D2), 256, 0, st>>>(Vl, (long long)D2, 1.0 / el);
        TN_LAUNCH_CHECK();
        scal_kernel<<<g1d((long long)nG), 256, 0, st>>>(gam, (long long)nG, 1.0 / std::sqrt(el));
        TN_LAUNCH_CHECK();
        // Factor: Vr = Ur sr Ur^T, Vl = Ul sl Ul^T
        TN_CUDA_CHECK(cudaMemcpyAsync(Wr, Vr, sizeof(double) * D2, cudaMemcpyDeviceToDevice, st));
        TN_CUDA_CHECK(cudaMemcpyAsync(Wl, Vl, sizeof(double) * D2, cudaMemcpyDeviceToDevice, st));
        TN_CUDA_CHECK(cudaMemsetAsync(stats + 4, 0, sizeof(double), st));
        {
            SvdJob jr{Wr, D, D, Vwr, Ur, D, Vtr, D, sr, nullptr};
            SvdJob jl{Wl, D, D, Vwl, Ul, D, Vtl, D, sl, nullptr};
            TN_CHECK(svd_batched(*ctx, {jr, jl}, true));
        }
        sqrt_pair_kernel<<<(D + 255) / 256, 256, 0, st>>>(sr, sl, D, sqv, stats + 4);
        TN_LAUNCH_CHECK();
        double flag = 0;
        TN_CUDA_CHECK(cudaMemcpyAsync(&flag, stats + 4, sizeof(double), cudaMemcpyDeviceToHost, st));
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        if (flag != 0.0) {  // a singular factor (the reference's isnan(X) / isnan(Yd) bail-out)
            bail = true;
            break;
        }
        const double* sqr = sqv;
        const double* isqr = sqv + D;
        const double* sql = sqv + 2 * D;
        const double* isql = sqv + 3 * D;
        // Z = l X = l Ur sqrt(sr);  Ys = Yd = Ul sqrt(sl);  YlX = Ys^T Z
        scale_kernel<<<g1d((long long)D2), 256, 0, st>>>(Ur, 1, D, D, lamv, sqr, Z);
        TN_LAUNCH_CHECK();
        scale_kernel<<<g1d((long long)D2), 256, 0, st>>>(Ul, 1, D, D, nullptr, sql, Ys);
        TN_LAUNCH_CHECK();
        TN_CHECK(gemm(D, D, D, Ys, idx(D), idx(1), Z, idx(1), idx(D), YlX));
        {
            SvdJob jy{YlX, D, D, Vwy, Up, D, VTp, D, lp, nullptr};
            TN_CHECK(svd_batched(*ctx, {jy}, true));
        }
        normalize_kernel<<<1, 256, 0, st>>>(lp, D, nullptr);
        TN_LAUNCH_CHECK();
        // VX = VT X^-1 = VTp (Ur / sqrt(sr))^T ;  YU = Yd^-T U = (Ul / sqrt(sl)) Up
        scale_kernel<<<g1d((long long)D2), 256, 0, st>>>(Ur, 1, D, D, nullptr, isqr, Ri);
        TN_LAUNCH_CHECK();
        scale_kernel<<<g1d((long long)D2), 256, 0, st>>>(Ul, 1, D, D, nullptr, isql, Li);
        TN_LAUNCH_CHECK();
        TN_CHECK(gemm(D, D, D, VTp, idx(1), idx(D), Ri, idx(D), idx(1), VX));
        TN_CHECK(gemm(D, D, D, Li, idx(1), idx(D), Up, idx(1), idx(D), YU));
        {
            GemmArgs g;  // tmp_n = VX gam_n
            g.M = D; g.N = D; g.K = D; g.nb0 = dd;
            g.A.ptr = VX; g.A.mn = idx(1); g.A.k = idx(D);
            g.B.ptr = gam; g.B.k = idx(1); g.B.mn = idx(D); g.B.sb0 = (long long)D2;
            g.C.ptr = tmp; g.C.m = idx(1); g.C.n = idx(D); g.C.sb0 = (long long)D2;
            TN_CHECK(gemm_f64(g, st));
            GemmArgs h;  // gam_n = tmp_n YU
            h.M = D; h.N = D; h.K = D; h.nb0 = dd;
            h.A.ptr = tmp; h.A.mn = idx(1); h.A.k = idx(D); h.A.sb0 = (long long)D2;
            h.B.ptr = YU; h.B.k = idx(1); h.B.mn = idx(D);
            h.C.ptr = gam; h.C.m = idx(1); h.C.n = idx(D); h.C.sb0 = (long long)D2;
            TN_CHECK(gemm_f64(h, st));
        }
        maxdiff_kernel<<<1, 256, 0, st>>>(lamv, lp, D, stats + 5);
        TN_LAUNCH_CHECK();
        TN_CUDA_CHECK(cudaMemcpyAsync(lamv, lp, sizeof(double) * D, cudaMemcpyDeviceToDevice, st));
        TN_CUDA_CHECK(cudaMemcpyAsync(&dl, stats + 5, sizeof(double), cudaMemcpyDeviceToHost, st));
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        if (dl < eps) {
            ++it;
            break;
        }
    }
    if (!bail) {
        scal_kernel<<<g1d((long long)nG), 256, 0, st>>>(gam, (long long)nG, 1.0 / std::sqrt(er));
        TN_LAUNCH_CHECK();
    }
    if (delta) *delta = dl;
    if (iters) *iters = it;
    if (bailed) *bailed = bail;
    // lambdaB = l / |l| (Bond::SetSingularValues)
    std::vector<double> hl(D);
    TN_CUDA_CHECK(cudaMemcpyAsync(hl.data(), lamv, sizeof(double) * D, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    double nrm = 0;
    for (double x : hl) nrm += x * x;
    nrm = std::sqrt(nrm);
    for (double& x : hl) x /= nrm;
    lam_h[1] = hl;
    TN_CUDA_CHECK(cudaMemcpyAsync(lam[1].p, hl.data(), sizeof(double) * D, cudaMemcpyHostToDevice, st));
    // UnpackOrthonormal
    const int m = d * D;
    TN_CHECK(M.ensure(sizeof(double) * (size_t)m * m));
    gamma_reshape_kernel<<<g1d((long long)m * m), 256, 0, st>>>(gam, d, D, lam[1].as<double>(), M.as<double>());
    TN_LAUNCH_CHECK();
    return svd_unpack(0, D, Dmax, 1e-16);
}

int ITebdState::grow(int D) {
    cudaStream_t st = ctx->stream;
    const int old[2] = {dim(0), dim(1)};
    if (old[0] >= D && old[1] >= D) return TN_OK;
    // Gammas: site 0 is (d, dim 1, dim 0), site 1 is (d, dim 0, dim 1); zero-padded to (d, D, D)
    for (int site = 0; site < 2; ++site) {
        const int Dl = site == 0 ? old[1] : old[0];
        const int Dr = site == 0 ? old[0] : old[1];
        const int N1 = std::max(D, Dl), N2 = std::max(D, Dr);
        TN_CHECK(work.ensure(sizeof(double) * (size_t)d * N1 * N2));
        pad_kernel<<<g1d((long long)d * N1 * N2), 256, 0, st>>>(G[site].as<double>(), d, Dl, Dr, work.as<double>(),
                                                                N1, N2);
        TN_LAUNCH_CHECK();
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        TN_CHECK(G[site].ensure(sizeof(double) * (size_t)d * N1 * N2));
        TN_CUDA_CHECK(cudaMemcpyAsync(G[site].p, work.p, sizeof(double) * (size_t)d * N1 * N2,
                                      cudaMemcpyDeviceToDevice, st));
    }
    // bond values: padded with min/10, renormalised (Bond::NewBondDimension, Bond.C:60-84)
    for (int b = 0; b < 2; ++b) {
        auto& l = lam_h[b];
        if ((int)l.size() >= D) continue;
        const double fill = *std::min_element(l.begin(), l.end()) / 10.0;
        l.resize(D, fill);
        double nrm = 0;
        for (double x : l) nrm += x * x;
        nrm = std::sqrt(nrm);
        for (double& x : l) x /= nrm;
        TN_CHECK(lam[b].ensure(sizeof(double) * D));
        TN_CUDA_CHECK(cudaMemcpyAsync(lam[b].p, l.data(), sizeof(double) * D, cudaMemcpyHostToDevice, st));
    }
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    return TN_OK;
}

int ITebdState::energy(double* E, int max_iters, double tol) {
    cudaStream_t st = ctx->stream;
    const int dd = d * d;
    double es[2];
    for (int b = 0; b < 2; ++b) {
        // cell P Q across bond b: P = G_b lam_b, Q = G_{1-b} lam_{1-b}
        const int P = b, Qs = 1 - b;
        const int Dl = dim(Qs), Dm = dim(b);  // P: (d, Dl, Dm), Q: (d, Dm, Dl)
        const size_t nP = (size_t)d * Dl * Dm;
        const size_t nB = (size_t)dd * Dl * Dl;
        TN_CHECK(X.ensure(sizeof(double) * nP));
        TN_CHECK(Y.ensure(sizeof(double) * nP));
        TN_CHECK(TH.ensure(sizeof(double) * nB));
        TN_CHECK(M.ensure(sizeof(double) * (2 * nB + 4 * (size_t)Dl * Dl + (size_t)dd * dd + 8)));
        scale_kernel<<<g1d((long long)nP), 256, 0, st>>>(G[P].as<double>(), d, Dl, Dm, nullptr, lam[b].as<double>(),
                                                         X.as<double>());
        TN_LAUNCH_CHECK();
        scale_kernel<<<g1d((long long)nP), 256, 0, st>>>(G[Qs].as<double>(), d, Dm, Dl, nullptr, lam[Qs].as<double>(),
                                                         Y.as<double>());
        TN_LAUNCH_CHECK();
        // B_p = P[m1] Q[m2], p = m1 d + m2 (Dl x Dl), stacked: B[p](i, j) at p*Dl*Dl + j*Dl + i
        GemmArgs g;
        g.M = Dl; g.N = Dl; g.K = Dm; g.nb0 = d; g.nb1 = d;
        g.A.ptr = X.as<double>(); g.A.mn = idx(1); g.A.k = idx(Dl); g.A.sb0 = (long long)Dl * Dm;
        g.B.ptr = Y.as<double>(); g.B.k = idx(1); g.B.mn = idx(Dm); g.B.sb1 = (long long)Dm * Dl;
        g.C.ptr = TH.as<double>(); g.C.m = idx(1); g.C.n = idx(Dl); g.C.sb0 = (long long)d * Dl * Dl;
        g.C.sb1 = (long long)Dl * Dl;
        TN_CHECK(gemm_f64(g, st));
        double* Bs = TH.as<double>();
        double* T1 = M.as<double>();      // dd blocks
        double* T2 = T1 + nB;             // dd blocks
        double* lv = T2 + nB;             // left fixed point
        double* rv = lv + (size_t)Dl * Dl;
        double* tmp = rv + (size_t)Dl * Dl;
        double* prev = tmp + (size_t)Dl * Dl;
        double* dots = prev + (size_t)Dl * Dl;
        double* scal = dots + (size_t)dd * dd;
        const int n2 = Dl * Dl;
        // start: identity
        std::vector<double> I0((size_t)n2, 0.0);
        for (int i = 0; i < Dl; ++i) I0[(size_t)i * Dl + i] = 1.0;
        TN_CUDA_CHECK(cudaMemcpyAsync(lv, I0.data(), sizeof(double) * n2, cudaMemcpyHostToDevice, st));
        TN_CUDA_CHECK(cudaMemcpyAsync(rv, I0.data(), sizeof(double) * n2, cudaMemcpyHostToDevice, st));
        for (int side = 0; side < 2; ++side) {
            double* v = side == 0 ? lv : rv;
            for (int it = 0; it < max_iters; ++it) {
                TN_CUDA_CHECK(cudaMemcpyAsync(prev, v, sizeof(double) * n2, cudaMemcpyDeviceToDevice, st));
                GemmArgs a, c;
                if (side == 0) {
                    // T1_p = l B_p ; l' = sum_p B_p^T T1_p
                    a.M = Dl; a.N = Dl; a.K = Dl; a.nb0 = dd;
                    a.A.ptr = v; a.A.mn = idx(1); a.A.k = idx(Dl);
                    a.B.ptr = Bs; a.B.k = idx(1); a.B.mn = idx(Dl); a.B.sb0 = n2;
                    a.C.ptr = T1; a.C.m = idx(1); a.C.n = idx(Dl); a.C.sb0 = n2;
                    TN_CHECK(gemm_f64(a, st));
                    c.M = Dl; c.N = Dl; c.K = dd * Dl;  // k = (i, p): B_p(i, j) T1_p(i, k)
                    c.A.ptr = Bs; c.A.mn = idx(Dl); c.A.k = idx2(1, Dl, n2);
                    c.B.ptr = T1; c.B.k = idx2(1, Dl, n2); c.B.mn = idx(Dl);
                    c.C.ptr = tmp; c.C.m = idx(1); c.C.n = idx(Dl);
                    TN_CHECK(gemm_f64(c, st));
                } else {
                    // T1_p = B_p r ; r' = sum_p T1_p B_p^T
                    a.M = Dl; a.N = Dl; a.K = Dl; a.nb0 = dd;
                    a.A.ptr = Bs; a.A.mn = idx(1); a.A.k = idx(Dl); a.A.sb0 = n2;
                    a.B.ptr = v; a.B.k = idx(1); a.B.mn = idx(Dl);
                    a.C.ptr = T1; a.C.m = idx(1); a.C.n = idx(Dl); a.C.sb0 = n2;
                    TN_CHECK(gemm_f64(a, st));
                    c.M = Dl; c.N = Dl; c.K = dd * Dl;  // k = (j, p): T1_p(i, j) B_p(k, j)
                    c.A.ptr = T1; c.A.mn = idx(1); c.A.k = idx2(Dl, Dl, n2);
                    c.B.ptr = Bs; c.B.k = idx2(Dl, Dl, n2); c.B.mn = idx(1);
                    c.C.ptr = tmp; c.C.m = idx(1); c.C.n = idx(Dl);
                    TN_CHECK(gemm_f64(c, st));
                }
                normalize_kernel<<<1, 256, 0, st>>>(tmp, n2, scal);
                TN_LAUNCH_CHECK();
                TN_CUDA_CHECK(cudaMemcpyAsync(v, tmp, sizeof(double) * n2, cudaMemcpyDeviceToDevice, st));
                if ((it + 1) % 50 == 0 || it + 1 == max_iters) {
                    maxdiff_kernel<<<1, 256, 0, st>>>(v, prev, n2, scal + 1);
                    TN_LAUNCH_CHECK();
                    double md = 0;
                    TN_CUDA_CHECK(cudaMemcpyAsync(&md, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
                    TN_CUDA_CHECK(cudaStreamSynchronize(st));
                    if (md < tol) break;
                }
            }
        }
        // C_p = l B_p, E_q = B_q r; num = sum h_pq <C_p, E_q>, den = sum_p <C_p, E_p>
        GemmArgs a;
        a.M = Dl; a.N = Dl; a.K = Dl; a.nb0 = dd;
        a.A.ptr = lv; a.A.mn = idx(Dl); a.A.k = idx(1);  // l^T B_p: <l| contracts the row index
        a.B.ptr = Bs; a.B.k = idx(1); a.B.mn = idx(Dl); a.B.sb0 = n2;
        a.C.ptr = T1; a.C.m = idx(1); a.C.n = idx(Dl); a.C.sb0 = n2;
        TN_CHECK(gemm_f64(a, st));
        GemmArgs e;
        e.M = Dl; e.N = Dl; e.K = Dl; e.nb0 = dd;
        e.A.ptr = Bs; e.A.mn = idx(1); e.A.k = idx(Dl); e.A.sb0 = n2;
        e.B.ptr = rv; e.B.k = idx(1); e.B.mn = idx(Dl);
        e.C.ptr = T2; e.C.m = idx(1); e.C.n = idx(Dl); e.C.sb0 = n2;
        TN_CHECK(gemm_f64(e, st));
        pair_dots_kernel<<<dd * dd, 256, 0, st>>>(T1, T2, dd, n2, dots);
        TN_LAUNCH_CHECK();
        std::vector<double> hd((size_t)dd * dd);
        TN_CUDA_CHECK(cudaMemcpyAsync(hd.data(), dots, sizeof(double) * dd * dd, cudaMemcpyDeviceToHost, st));
        TN_CUDA_CHECK(cudaStreamSynchronize(st));
        double num = 0, den = 0;
        for (int p = 0; p < dd; ++p) {
            den += hd[(size_t)p * dd + p];
            for (int q = 0; q < dd; ++q) num += h12[(size_t)q * dd + p] * hd[(size_t)p * dd + q];
        }
        es[b] = num / den;
    }
    *E = 0.5 * (es[0] + es[1]);
    return TN_OK;
}

}  // namespace tnb
