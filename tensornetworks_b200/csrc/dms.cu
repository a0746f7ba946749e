// dms.cu -- one- and two-site reduced density matrices of the MPS on the device
// (MPSImp::CalculateOneSiteDMs / CalculateTwoSiteDMs,
// TensorNetworksImp/MPS/MPSImp_ExpectationsAndDMs.C:59-117, with the site
// contractions of MPSSite_Contractions.C:516-580).
//
// Both walk the orthogonality centre from the left: the state is first
// right-normalised (Normalize(DRight)), each site ia is then the centre when
// its density matrices are formed, and is left-normalised (NormalizeSite(DLeft,
// ia)) before the next one, so that after the call the MPS is left-canonical,
// as the reference leaves it.
//   one site:  rho(m, n) = <A_m, A_n> (Frobenius over both bond indices)
//   two sites: for the pair (ia, ib) and every (m, n) of site ia the zipper
//     C_mn = A_m^T A_n (D2 x D2) is carried through the sites between
//     (C <- sum_n2 A_n2^T C A_n2) and closed at ib:
//     rho(m, m2; n, n2) = <A_m2, C_mn A_n2>.  For fixed ia all ib are served by
//     one pass: at each ib the closing product T = C A_n2 is also the first
//     half of the propagation through ib.
// The products are the library's FP64 batched GEMM; the closing dots one
// small kernel.
#include <algorithm>

#include "engine.h"

namespace tnb {

namespace {

// out[p * nb + q] = <X_p, Y_q> over n elements, X_p at X + p * xs, Y_q at Y + q * ys; one block per pair
__global__ void pair_dot_kernel(const double* __restrict__ X, long long xs, int na, const double* __restrict__ Y,
                                long long ys, int nb, long long n, double* __restrict__ out) {
    const int p = blockIdx.x / nb, q = blockIdx.x % nb;
    if (p >= na) return;
    __shared__ double sh[32];
    double s = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s = fma(X[p * xs + i], Y[q * ys + i], s);
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

}  // namespace

int MPSState::one_site_dms(double* out_host) {
    cudaStream_t st = ctx->stream;
    TN_CHECK(normalize_all(false));  // Normalize(DRight)
    // normalize_site reuses the state's scratch: the results get a buffer of their own
    DevBuf res;
    TN_CHECK(res.ensure(sizeof(double) * (size_t)L * d * d));
    for (int ia = 1; ia <= L; ++ia) {
        const long long blk = (long long)D1[ia] * D2[ia];
        pair_dot_kernel<<<d * d, 256, 0, st>>>(A[ia]->as<double>(), blk, d, A[ia]->as<double>(), blk, d, blk,
                                               res.as<double>() + (size_t)(ia - 1) * d * d);
        TN_LAUNCH_CHECK();
        TN_CHECK(normalize_site(ia, true));  // NormalizeSite(DLeft, ia)
    }
    TN_CUDA_CHECK(cudaMemcpyAsync(out_host, res.p, sizeof(double) * (size_t)L * d * d, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    return TN_OK;
}

int MPSState::two_site_dms(double* out_host) {
    cudaStream_t st = ctx->stream;
    TN_CHECK(normalize_all(false));
    const int dd = d * d, d4 = dd * dd;
    const size_t npairs = (size_t)L * (L - 1) / 2;
    DevBuf res, Cb, Tb, Cn;
    TN_CHECK(res.ensure(sizeof(double) * npairs * d4));
    const int Dmax = max_D();
    const size_t D2max = (size_t)Dmax * Dmax;
    TN_CHECK(Cb.ensure(sizeof(double) * dd * D2max));
    TN_CHECK(Cn.ensure(sizeof(double) * dd * D2max));
    TN_CHECK(Tb.ensure(sizeof(double) * (size_t)dd * d * D2max));
    size_t pair = 0;
    for (int ia = 1; ia < L; ++ia) {
        // C[m d + n](i2, j2) = sum_i1 A_m(i1, i2) A_n(i1, j2)   (InitializeTwoSiteDM)
        {
            const int a1 = D1[ia], a2 = D2[ia];
            const long long blk = (long long)a1 * a2;
            GemmArgs g;
            g.M = a2; g.N = a2; g.K = a1; g.nb0 = d; g.nb1 = d;
            g.A.ptr = A[ia]->as<double>(); g.A.mn = idx(a1); g.A.k = idx(1); g.A.sb0 = blk; g.A.sb1 = 0;
            g.B.ptr = A[ia]->as<double>(); g.B.k = idx(1); g.B.mn = idx(a1); g.B.sb0 = 0; g.B.sb1 = blk;
            g.C.ptr = Cb.as<double>(); g.C.m = idx(1); g.C.n = idx(a2);
            g.C.sb0 = (long long)d * a2 * a2; g.C.sb1 = (long long)a2 * a2;
            TN_CHECK(gemm_f64(g, st));
        }
        for (int ib = ia + 1; ib <= L; ++ib, ++pair) {
            const int b1 = D1[ib], b2 = D2[ib];
            const long long cblk = (long long)b1 * b1, blk = (long long)b1 * b2;
            // T[(mn) d + n2](i1, j2) = sum_j1 C_mn(i1, j1) A_n2(j1, j2)     (ContractCA)
            GemmArgs g;
            g.M = b1; g.N = b2; g.K = b1; g.nb0 = dd; g.nb1 = d;
            g.A.ptr = Cb.as<double>(); g.A.mn = idx(1); g.A.k = idx(b1); g.A.sb0 = cblk; g.A.sb1 = 0;
            g.B.ptr = A[ib]->as<double>(); g.B.k = idx(1); g.B.mn = idx(b1); g.B.sb0 = 0; g.B.sb1 = blk;
            g.C.ptr = Tb.as<double>(); g.C.m = idx(1); g.C.n = idx(b1);
            g.C.sb0 = (long long)d * blk; g.C.sb1 = blk;
            TN_CHECK(gemm_f64(g, st));
            // rho(m, m2; n, n2) = <A_m2, T[(mn) d + n2]>                       (FinializeTwoSiteDM)
            // dots[m2 * (dd d) + (mn) d + n2]
            DevBuf& dots = tmp;
            TN_CHECK(dots.ensure(sizeof(double) * (size_t)d * dd * d));
            pair_dot_kernel<<<d * dd * d, 256, 0, st>>>(A[ib]->as<double>(), blk, d, Tb.as<double>(), blk, dd * d,
                                                        blk, dots.as<double>());
            TN_LAUNCH_CHECK();
            TN_CHECK(dm_scatter(dots.as<double>(), res.as<double>() + pair * d4));
            if (ib < L) {
                // C'_mn(i2, j2) = sum_{n2, i1} A_n2(i1, i2) T[(mn) d + n2](i1, j2)   (IterateTwoSiteDM)
                GemmArgs h;
                h.M = b2; h.N = b2; h.K = d * b1; h.nb0 = dd;
                h.A.ptr = A[ib]->as<double>(); h.A.mn = idx(b1); h.A.k = idx2(1, b1, blk);
                h.B.ptr = Tb.as<double>(); h.B.k = idx2(1, b1, blk); h.B.mn = idx(b1); h.B.sb0 = (long long)d * blk;
                h.C.ptr = Cn.as<double>(); h.C.m = idx(1); h.C.n = idx(b2); h.C.sb0 = (long long)b2 * b2;
                TN_CHECK(gemm_f64(h, st));
                std::swap(Cb.p, Cn.p);
                std::swap(Cb.bytes, Cn.bytes);
            }
        }
        TN_CHECK(normalize_site(ia, true));
    }
    TN_CHECK(normalize_site(L, true));  // the last one, to keep things tidy (as the reference)
    TN_CUDA_CHECK(cudaMemcpyAsync(out_host, res.p, sizeof(double) * npairs * d4, cudaMemcpyDeviceToHost, st));
    TN_CUDA_CHECK(cudaStreamSynchronize(st));
    return TN_OK;
}

namespace {
// dots[m2 * (d^3) + (m d + n) d + n2] -> rho[((m d + m2) d + n) d + n2]
__global__ void dm_scatter_kernel(const double* __restrict__ dots, int d, double* __restrict__ rho) {
    const int d4 = d * d * d * d;
    for (int e = threadIdx.x; e < d4; e += blockDim.x) {
        const int n2 = e % d, n = (e / d) % d, m2 = (e / (d * d)) % d, m = e / (d * d * d);
        rho[e] = dots[(size_t)m2 * d * d * d + (size_t)(m * d + n) * d + n2];
    }
}
}  // namespace

int MPSState::dm_scatter(const double* dots, double* rho) {
    dm_scatter_kernel<<<1, 256, 0, ctx->stream>>>(dots, d, rho);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

}  // namespace tnb
