// itime.cu -- imaginary-time evolution of the finite MPS on the device:
// MPSImp::FindiTimeGroundState / Optimize / Sweep(psi2) / ApplyInPlace
// (TensorNetworksImp/MPS/MPSImp_iTime.C:18-198), MPSImp::NormalizeAndCompress
// (MPSImp_Normalization.C:34-53, with MPSSite::SVDNormalize,
// MPSSite_Normalization.C:45-78) and the Trotter operator of
// HamiltonianImp::CreateOperator (HamiltonianImp.C:52-86, first and second
// order).
//
// One iteration of a schedule line: |psi2> = W |psi> (W = the Trotter MPO of
// exp(-dt H); the site tensors grow to D Dw), then |psi> is SVD-normalised left
// to right and right to left with the line's compressor (Dmax, eps), and then
// varied towards |psi2> by alternating sweeps (site = L12 A2 R12^T with the
// overlap environments, then a gauge move), until the distance
// 2 - 2 <psi|psi2> / |psi2| changes by at most the line's norm epsilon.
//
// W is the exact product of the gate layers (odd bonds, even bonds, odd bonds
// for second order), each gate exp(-tau h12) split by an SVD into
// sum_k A_k (x) B_k; the reference compresses that product (Parker) to its
// MPO epsilon, which the tests set at 1e-6 .. 1e-14.  The field hz Sz of a
// site is shared by the bonds it belongs to (half on each for inner sites),
// so that the layers add up to the MPO's Hamiltonian.  The SVDs are the
// library's Jacobi SVD; products FP64 GEMMs.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "engine.h"
#include "host_linalg.h"

namespace tnb {

namespace {

double sz_of(int m, double S) { return m - S; }
double sp_el(int m, int n, double S) {  // <m|S+|n>
    return (m == n + 1) ? std::sqrt(S * (S + 1.0) - sz_of(m, S) * sz_of(n, S)) : 0.0;
}

// Gate exp(-tau h) of one bond (h with the field weights ca, cb of its two sites)
// as sum_k A_k (x) B_k: the SVD of M[(ma,na),(mb,nb)] = G(ma mb; na nb).
void gate_split(int d, double S, double Jxy, double Jz, double hz, double ca, double cb, double tau, int& r,
                std::vector<double>& Ak, std::vector<double>& Bk) {
    const int dd = d * d;
    std::vector<double> h((size_t)dd * dd, 0.0);  // h[(ma d + mb) + (na d + nb) dd]
    for (int ma = 0; ma < d; ++ma)
        for (int mb = 0; mb < d; ++mb)
            for (int na = 0; na < d; ++na)
                for (int nb = 0; nb < d; ++nb) {
                    double v = 0.5 * Jxy * (sp_el(ma, na, S) * sp_el(nb, mb, S) + sp_el(na, ma, S) * sp_el(mb, nb, S));
                    if (ma == na && mb == nb) v += Jz * sz_of(ma, S) * sz_of(mb, S);
                    if (ma == na && mb == nb) v += hz * (ca * sz_of(ma, S) + cb * sz_of(mb, S));
                    h[(size_t)(ma * d + mb) + (size_t)(na * d + nb) * dd] = v;
                }
    // G = exp(-tau h) from the eigen-decomposition of the symmetric h (host Jacobi SVD of h + c I)
    double shift = 0;
    for (int i = 0; i < dd; ++i) {
        double rs = 0;
        for (int j = 0; j < dd; ++j) rs += std::fabs(h[(size_t)i + (size_t)j * dd]);
        shift = std::max(shift, rs);
    }
    shift = 1.001 * shift + 1e-300;
    std::vector<double> hs = h;
    for (int i = 0; i < dd; ++i) hs[(size_t)i * dd + i] += shift;
    std::vector<double> Uh, sh, Vh;
    host_svd(hs, dd, dd, Uh, sh, Vh);
    std::vector<double> G((size_t)dd * dd, 0.0);
    for (int k = 0; k < dd; ++k) {
        const double e = std::exp(-tau * (sh[k] - shift));
        for (int i = 0; i < dd; ++i)
            for (int j = 0; j < dd; ++j) G[(size_t)i + (size_t)j * dd] += Uh[(size_t)k * dd + i] * e * Uh[(size_t)k * dd + j];
    }
    // M[(ma,na),(mb,nb)]: row ma d + na, column mb d + nb
    std::vector<double> M((size_t)dd * dd);
    for (int ma = 0; ma < d; ++ma)
        for (int mb = 0; mb < d; ++mb)
            for (int na = 0; na < d; ++na)
                for (int nb = 0; nb < d; ++nb)
                    M[(size_t)(ma * d + na) + (size_t)(mb * d + nb) * dd] =
                        G[(size_t)(ma * d + mb) + (size_t)(na * d + nb) * dd];
    std::vector<double> Um, sm, Vm;
    host_svd(M, dd, dd, Um, sm, Vm);
    const double smax = *std::max_element(sm.begin(), sm.end());
    r = 0;
    Ak.clear();
    Bk.clear();
    std::vector<int> order(dd);
    for (int k = 0; k < dd; ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return sm[a] > sm[b]; });
    for (int kk = 0; kk < dd; ++kk) {
        const int k = order[kk];
        if (!(sm[k] > 1e-14 * smax)) continue;
        const double rt = std::sqrt(sm[k]);
        for (int ma = 0; ma < d; ++ma)
            for (int na = 0; na < d; ++na) Ak.push_back(rt * Um[(size_t)k * dd + ma * d + na]);
        for (int mb = 0; mb < d; ++mb)
            for (int nb = 0; nb < d; ++nb) Bk.push_back(rt * Vm[(size_t)k * dd + mb * d + nb]);
        ++r;
    }
}

// (P Q)[(w1,v1),(w2,v2)](m,n) = sum_k P[w1,w2](m,k) Q[v1,v2](k,n): P applied after Q
SiteMPO mpo_mul(const SiteMPO& P, const SiteMPO& Q, int d) {
    SiteMPO R;
    R.Dw1 = P.Dw1 * Q.Dw1;
    R.Dw2 = P.Dw2 * Q.Dw2;
    R.W.assign((size_t)R.Dw1 * R.Dw2 * d * d, 0.0);
    for (int w1 = 0; w1 < P.Dw1; ++w1)
        for (int v1 = 0; v1 < Q.Dw1; ++v1)
            for (int w2 = 0; w2 < P.Dw2; ++w2)
                for (int v2 = 0; v2 < Q.Dw2; ++v2)
                    for (int m = 0; m < d; ++m)
                        for (int n = 0; n < d; ++n) {
                            double s = 0;
                            for (int k = 0; k < d; ++k)
                                s += P.W[(((size_t)w1 * P.Dw2 + w2) * d + m) * d + k] *
                                     Q.W[(((size_t)v1 * Q.Dw2 + v2) * d + k) * d + n];
                            R.W[(((size_t)(w1 * Q.Dw1 + v1) * R.Dw2 + (w2 * Q.Dw2 + v2)) * d + m) * d + n] = s;
                        }
    return R;
}

// A'[m](i1 Dw1 + w1, i2 Dw2 + w2) = sum_n W(w1, w2)(m, n) A[n](i1, i2)   (MPSSite::ApplyInPlace)
__global__ void apply_mpo_kernel(const double* __restrict__ A, int d, int D1, int D2, const double* __restrict__ W,
                                 int Dw1, int Dw2, double* __restrict__ out) {
    const int E1 = D1 * Dw1, E2 = D2 * Dw2;
    const long long total = (long long)d * E1 * E2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int I1 = (int)(e % E1), I2 = (int)((e / E1) % E2), m = (int)(e / ((long long)E1 * E2));
        const int i1 = I1 / Dw1, w1 = I1 % Dw1, i2 = I2 / Dw2, w2 = I2 % Dw2;
        double acc = 0;
        for (int n = 0; n < d; ++n)
            acc = fma(W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n], A[(size_t)n * D1 * D2 + (size_t)i2 * D1 + i1], acc);
        out[e] = acc;
    }
}

inline int g1d(long long n) {
    long long b = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(b, 148 * 8));
}

// M (rows x cols, column-major): row r scaled by s[r] (rows) or column c by s[c] (cols)
__global__ void scale_rc_kernel(double* __restrict__ M, int rows, int cols, const double* __restrict__ s, int by_row) {
    const long long total = (long long)rows * cols;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x)
        M[e] *= by_row ? s[e % rows] : s[e / rows];
}

int scale_rows(double* M, int rows, int cols, const double* s, cudaStream_t st) {
    scale_rc_kernel<<<g1d((long long)rows * cols), 256, 0, st>>>(M, rows, cols, s, 1);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

int scale_cols(double* M, int rows, int cols, const double* s, cudaStream_t st) {
    scale_rc_kernel<<<g1d((long long)rows * cols), 256, 0, st>>>(M, rows, cols, s, 0);
    TN_LAUNCH_CHECK();
    return TN_OK;
}

// SVCompressorImp::Compress (SVCompressorImp.C:19-73): kept count of descending s
int compress_keep(const std::vector<double>& s, int Dmax, double eps) {
    const int N = (int)s.size();
    int D = N;
    if (eps > 0) {
        double tail = 0;
        for (D = N; D >= 2; --D) {
            const double s2 = s[D - 1] * s[D - 1];
            if (tail + s2 >= eps) break;
            tail += s2;
        }
    }
    if (Dmax > 0) D = std::min(D, Dmax);
    while (D > 1 && !(s[D - 1] > 0)) --D;  // zero singular values carry nothing
    return std::max(D, 1);
}

}  // namespace

// Grow site ia's buffer to hold n doubles, keeping its contents.
int MPSState::site_reserve(int ia, size_t n) {
    if (A[ia]->bytes >= sizeof(double) * n) return TN_OK;
    DevBuf nb;
    TN_CHECK(nb.ensure(sizeof(double) * n));
    if (A[ia]->p) TN_CUDA_CHECK(cudaMemcpyAsync(nb.p, A[ia]->p, A[ia]->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    TN_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    std::swap(A[ia]->p, nb.p);
    std::swap(A[ia]->bytes, nb.bytes);
    return TN_OK;
}

// HamiltonianImp::CreateOperator (first / second order): per site the product MPO of the gate layers.
int MPSState::trotter_mpo(double dt, int order, std::vector<SiteMPO>& out) const {
    const double S = H->S;
    std::vector<SiteMPO> layer_odd(L + 1), layer_even(L + 1), layer_half(L + 1);
    auto build_layer = [&](int parity, double tau, std::vector<SiteMPO>& lay) {
        for (int i = 1; i <= L; ++i) {
            lay[i].Dw1 = lay[i].Dw2 = 1;
            lay[i].W.assign((size_t)d * d, 0.0);
            for (int m = 0; m < d; ++m) lay[i].W[(size_t)m * d + m] = 1.0;
        }
        for (int a = 1 + parity; a < L; a += 2) {  // bond (a, a+1)
            const double ca = (a == 1) ? 1.0 : 0.5, cb = (a + 1 == L) ? 1.0 : 0.5;
            int r = 0;
            std::vector<double> Ak, Bk;
            gate_split(d, S, H->Jxy, H->Jz, H->hz, ca, cb, tau, r, Ak, Bk);
            SiteMPO& wa = lay[a];
            SiteMPO& wb = lay[a + 1];
            wa.Dw1 = 1;
            wa.Dw2 = r;
            wa.W.assign((size_t)r * d * d, 0.0);
            wb.Dw1 = r;
            wb.Dw2 = 1;
            wb.W.assign((size_t)r * d * d, 0.0);
            for (int k = 0; k < r; ++k)
                for (int m = 0; m < d; ++m)
                    for (int n = 0; n < d; ++n) {
                        wa.W[(((size_t)0 * r + k) * d + m) * d + n] = Ak[(size_t)k * d * d + m * d + n];
                        wb.W[(((size_t)k * 1 + 0) * d + m) * d + n] = Bk[(size_t)k * d * d + m * d + n];
                    }
        }
    };
    out.assign(L + 1, SiteMPO());
    if (order == 1) {
        build_layer(0, dt, layer_odd);
        build_layer(1, dt, layer_even);
        for (int i = 1; i <= L; ++i) out[i] = mpo_mul(layer_odd[i], layer_even[i], d);
    } else if (order == 2) {
        build_layer(0, 0.5 * dt, layer_half);
        build_layer(1, dt, layer_even);
        for (int i = 1; i <= L; ++i) out[i] = mpo_mul(mpo_mul(layer_half[i], layer_even[i], d), layer_half[i], d);
    } else {
        set_error("imaginary time: Trotter order %d not provided (1 or 2)", order);
        return TN_BAD_ARG;
    }
    return TN_OK;
}

// MPSImp::ApplyInPlace: |psi> <- W |psi>
int MPSState::apply_mpo_inplace(const std::vector<SiteMPO>& W) {
    cudaStream_t st = ctx->stream;
    DevBuf wd;
    for (int ia = 1; ia <= L; ++ia) {
        const SiteMPO& op = W[ia];
        const int E1 = D1[ia] * op.Dw1, E2 = D2[ia] * op.Dw2;
        const size_t n = (size_t)d * E1 * E2;
        TN_CHECK(wd.ensure(sizeof(double) * op.W.size()));
        TN_CUDA_CHECK(cudaMemcpyAsync(wd.p, op.W.data(), sizeof(double) * op.W.size(), cudaMemcpyHostToDevice, st));
        TN_CHECK(tmp.ensure(sizeof(double) * n));
        apply_mpo_kernel<<<g1d((long long)n), 256, 0, st>>>(A[ia]->as<double>(), d, D1[ia], D2[ia], wd.as<double>(),
                                                            op.Dw1, op.Dw2, tmp.as<double>());
        TN_LAUNCH_CHECK();
        TN_CHECK(site_reserve(ia, n));
        TN_CUDA_CHECK(cudaMemcpyAsync(A[ia]->p, tmp.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        TN_CUDA_CHECK(cudaStreamSynchronize(st));  // wd and tmp are reused by the next site
        D1[ia] = E1;
        D2[ia] = E2;
    }
    for (int b = 1; b < L; ++b) bondK[b] = D2[b];
    return TN_OK;
}

// MPSImp::NormalizeAndCompress(lr, comp) with MPSSite::SVDNormalize(lr, comp):
// every site an SVD, truncated by the compressor rule, the bond factor moved
// into the neighbour; the edge site rescaled.  The kept singular values of
// every bond (normalised) land in svals[bond].
int MPSState::svd_compress_sweep(bool left, int Dmax, double eps, std::vector<std::vector<double>>* svals) {
    cudaStream_t st = ctx->stream;
    for (int step = 0; step < L; ++step) {
        const int ia = left ? 1 + step : L - step;
        if ((left && ia == L) || (!left && ia == 1)) {
            TN_CHECK(rescale_site(ia));
            continue;
        }
        const int a1 = D1[ia], a2 = D2[ia];
        const long long blk = (long long)a1 * a2;
        // M: left (d a1) x a2, rows n a1 + i1;  right a1 x (d a2), columns n a2 + i2
        const int m = left ? d * a1 : a1, n = left ? a2 : d * a2;
        const bool tall = m >= n;
        const int tm = tall ? m : n, tn = tall ? n : m;  // the SVD runs on the tall orientation
        TN_CHECK(Wqr.ensure(sizeof(double) * (size_t)tm * tn));
        TN_CHECK(svdw.ensure(sizeof(double) * ((size_t)tm * tn + 2 * (size_t)tn * tn + tn)));
        double* Ut = svdw.as<double>();      // tm x tn
        double* Vw = Ut + (size_t)tm * tn;   // tn x tn (work)
        double* Vt = Vw + (size_t)tn * tn;   // tn x tn
        double* sv = Vt + (size_t)tn * tn;   // tn
        double* Mw = Wqr.as<double>();
        const double* Aia = A[ia]->as<double>();
        if (left) {
            if (tall) TN_CHECK(copy2d(m, n, Aia, idx2(1, a1, blk), idx(a1), Mw, idx(1), idx(tm), 1.0, st));
            else TN_CHECK(copy2d(m, n, Aia, idx2(1, a1, blk), idx(a1), Mw, idx(tm), idx(1), 1.0, st));
        } else {
            if (tall) TN_CHECK(copy2d(m, n, Aia, idx(1), idx2(a1, a2, blk), Mw, idx(1), idx(tm), 1.0, st));
            else TN_CHECK(copy2d(m, n, Aia, idx(1), idx2(a1, a2, blk), Mw, idx(tm), idx(1), 1.0, st));
        }
        SvdJob job{Mw, tm, tn, Vw, Ut, tm, Vt, tn, sv, nullptr};
        TN_CHECK(svd_batched(*ctx, {job}, true));
        std::vector<double> hs(tn);
        TN_CUDA_CHECK(cudaMemcpy(hs.data(), sv, sizeof(double) * tn, cudaMemcpyDeviceToHost));
        const int k = compress_keep(hs, Dmax, eps);
        double nrm = 0;
        for (int i = 0; i < k; ++i) nrm += hs[i] * hs[i];
        nrm = std::sqrt(nrm);
        if (svals) {
            const int bond = left ? ia : ia - 1;
            std::vector<double>& bv = (*svals)[bond];
            bv.assign(hs.begin(), hs.begin() + k);
            for (double& x : bv) x /= (nrm > 0 ? nrm : 1.0);
        }
        // A = U s V^T (tall: U = Ut, V^T = Vt;  wide: A = (Ut s Vt)^T = Vt^T s Ut^T)
        // left:  site <- the m x k left factor;  right neighbour <- s (k x n right factor) . next
        // right: site <- the k x n right factor; left neighbour  <- prev . (m x k left factor) s
        // left factor L(i, c) = tall ? Ut(i, c) : Vt(c, i);  right factor R(c, j) = tall ? Vt(c, j) : Ut(j, c)
        const double* Lf = tall ? Ut : Vt;
        const IdxMap lr_row = tall ? idx(1) : idx(tn), lr_col = tall ? idx(tm) : idx(1);
        const double* Rf = tall ? Vt : Ut;
        const IdxMap rf_row = tall ? idx(1) : idx(tm), rf_col = tall ? idx(tn) : idx(1);
        DevBuf sk;
        TN_CHECK(sk.ensure(sizeof(double) * k));
        TN_CUDA_CHECK(cudaMemcpyAsync(sk.p, hs.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
        if (left) {
            // site ia <- L(:, :k) as (n, i1, c)
            TN_CHECK(copy2d(m, k, Lf, lr_row, lr_col, A[ia]->as<double>(), idx2(1, a1, (long long)a1 * k), idx(a1), 1.0,
                            st));
            D2[ia] = k;
            // next site: A'[n](c, j2) = sum_i2 s_c R(c, i2) A[n](i2, j2)
            const int b1 = D1[ia + 1], b2 = D2[ia + 1];
            TN_CHECK(tmp.ensure(sizeof(double) * ((size_t)k * n + (size_t)d * k * b2)));
            double* SR = tmp.as<double>();
            double* nxt = SR + (size_t)k * n;
            TN_CHECK(copy2d(k, n, Rf, rf_row, rf_col, SR, idx(1), idx(k), 1.0, st));
            TN_CHECK(scale_rows(SR, k, n, sk.as<double>(), st));
            GemmArgs g;
            g.M = k; g.N = b2; g.K = b1; g.nb0 = d;
            g.A.ptr = SR; g.A.mn = idx(1); g.A.k = idx(k);
            g.B.ptr = A[ia + 1]->as<double>(); g.B.k = idx(1); g.B.mn = idx(b1); g.B.sb0 = (long long)b1 * b2;
            g.C.ptr = nxt; g.C.m = idx(1); g.C.n = idx(k); g.C.sb0 = (long long)k * b2;
            TN_CHECK(gemm_f64(g, st));
            TN_CUDA_CHECK(cudaMemcpyAsync(A[ia + 1]->p, nxt, sizeof(double) * (size_t)d * k * b2, cudaMemcpyDeviceToDevice,
                                          st));
            D1[ia + 1] = k;
            bondK[ia] = k;
        } else {
            // site ia <- R(:k, :) as (n, c, i2): element (n, c, i2) = R(c, n a2 + i2)
            TN_CHECK(copy2d(k, n, Rf, rf_row, rf_col, A[ia]->as<double>(), idx(1), idx2(k, a2, (long long)k * a2), 1.0,
                            st));
            D1[ia] = k;
            // previous site: A'[n](i1, c) = sum_j A[n](i1, j) L(j, c) s_c
            const int p1 = D1[ia - 1], p2 = D2[ia - 1];
            TN_CHECK(tmp.ensure(sizeof(double) * ((size_t)m * k + (size_t)d * p1 * k)));
            double* LS = tmp.as<double>();
            double* prv = LS + (size_t)m * k;
            TN_CHECK(copy2d(m, k, Lf, lr_row, lr_col, LS, idx(1), idx(m), 1.0, st));
            TN_CHECK(scale_cols(LS, m, k, sk.as<double>(), st));
            GemmArgs g;
            g.M = p1; g.N = k; g.K = p2; g.nb0 = d;
            g.A.ptr = A[ia - 1]->as<double>(); g.A.mn = idx(1); g.A.k = idx(p1); g.A.sb0 = (long long)p1 * p2;
            g.B.ptr = LS; g.B.k = idx(1); g.B.mn = idx(m);
            g.C.ptr = prv; g.C.m = idx(1); g.C.n = idx(p1); g.C.sb0 = (long long)p1 * k;
            TN_CHECK(gemm_f64(g, st));
            TN_CUDA_CHECK(cudaMemcpyAsync(A[ia - 1]->p, prv, sizeof(double) * (size_t)d * p1 * k, cudaMemcpyDeviceToDevice,
                                          st));
            D2[ia - 1] = k;
            bondK[ia - 1] = k;
        }
        TN_CUDA_CHECK(cudaStreamSynchronize(st));  // sk and tmp are reused by the next site
    }
    return TN_OK;
}

// Overlap environments <psi|psi2>: Lo[ia] (D2(psi, ia) x D2(psi2, ia)) and Ro[ia]
// (D1(psi, ia) x D1(psi2, ia)); Lo[0] = Ro[L+1] = 1.
// Lo[ia](i2, j2) = sum_{n, i1, j1} A_n(i1, i2) Lo[ia-1](i1, j1) B_n(j1, j2)
int MPSState::overlap_left(int ia, const SiteSet& P2, std::vector<DevBuf*>& Lo) {
    cudaStream_t st = ctx->stream;
    const int a1 = D1[ia], a2 = D2[ia], b1 = P2.D1[ia], b2 = P2.D2[ia];
    TN_CHECK(tmp.ensure(sizeof(double) * (size_t)d * a1 * b2));
    // T[n](i1, j2) = Lo[ia-1](i1, j1) B_n(j1, j2)
    GemmArgs g;
    g.M = a1; g.N = b2; g.K = b1; g.nb0 = d;
    g.A.ptr = Lo[ia - 1]->as<double>(); g.A.mn = idx(1); g.A.k = idx(a1);
    g.B.ptr = P2.A[ia]->as<double>(); g.B.k = idx(1); g.B.mn = idx(b1); g.B.sb0 = (long long)b1 * b2;
    g.C.ptr = tmp.as<double>(); g.C.m = idx(1); g.C.n = idx(a1); g.C.sb0 = (long long)a1 * b2;
    TN_CHECK(gemm_f64(g, st));
    TN_CHECK(Lo[ia]->ensure(sizeof(double) * (size_t)a2 * b2));
    // Lo[ia](i2, j2) = sum_{(i1, n)} A_n(i1, i2) T[n](i1, j2)
    GemmArgs h;
    h.M = a2; h.N = b2; h.K = d * a1;
    h.A.ptr = A[ia]->as<double>(); h.A.mn = idx(a1); h.A.k = idx2(1, a1, (long long)a1 * a2);
    h.B.ptr = tmp.as<double>(); h.B.k = idx2(1, a1, (long long)a1 * b2); h.B.mn = idx(a1);
    h.C.ptr = Lo[ia]->as<double>(); h.C.m = idx(1); h.C.n = idx(a2);
    return gemm_f64(h, st);
}

// Ro[ia](i1, j1) = sum_{n, i2, j2} A_n(i1, i2) Ro[ia+1](i2, j2) B_n(j1, j2)
int MPSState::overlap_right(int ia, const SiteSet& P2, std::vector<DevBuf*>& Ro) {
    cudaStream_t st = ctx->stream;
    const int a1 = D1[ia], a2 = D2[ia], b1 = P2.D1[ia], b2 = P2.D2[ia];
    TN_CHECK(tmp.ensure(sizeof(double) * (size_t)d * a1 * b2));
    // T[n](i1, j2) = A_n(i1, i2) Ro[ia+1](i2, j2)
    GemmArgs g;
    g.M = a1; g.N = b2; g.K = a2; g.nb0 = d;
    g.A.ptr = A[ia]->as<double>(); g.A.mn = idx(1); g.A.k = idx(a1); g.A.sb0 = (long long)a1 * a2;
    g.B.ptr = Ro[ia + 1]->as<double>(); g.B.k = idx(1); g.B.mn = idx(a2);
    g.C.ptr = tmp.as<double>(); g.C.m = idx(1); g.C.n = idx(a1); g.C.sb0 = (long long)a1 * b2;
    TN_CHECK(gemm_f64(g, st));
    TN_CHECK(Ro[ia]->ensure(sizeof(double) * (size_t)a1 * b1));
    // Ro[ia](i1, j1) = sum_{(j2, n)} T[n](i1, j2) B_n(j1, j2)
    GemmArgs h;
    h.M = a1; h.N = b1; h.K = d * b2;
    h.A.ptr = tmp.as<double>(); h.A.mn = idx(1); h.A.k = idx2(a1, b2, (long long)a1 * b2);
    h.B.ptr = P2.A[ia]->as<double>(); h.B.k = idx2(b1, b2, (long long)b1 * b2); h.B.mn = idx(1);
    h.C.ptr = Ro[ia]->as<double>(); h.C.m = idx(1); h.C.n = idx(a1);
    return gemm_f64(h, st);
}

// MPSSite::Optimize (the closest site to psi2 given the others):
// A_n = Lo[ia-1] B_n Ro[ia+1]^T
int MPSState::overlap_site(int ia, const SiteSet& P2, std::vector<DevBuf*>& Lo, std::vector<DevBuf*>& Ro) {
    cudaStream_t st = ctx->stream;
    const int a1 = D1[ia], a2 = D2[ia], b1 = P2.D1[ia], b2 = P2.D2[ia];
    TN_CHECK(tmp.ensure(sizeof(double) * (size_t)d * a1 * b2));
    GemmArgs g;  // T[n] = Lo B_n   (a1 x b2)
    g.M = a1; g.N = b2; g.K = b1; g.nb0 = d;
    g.A.ptr = Lo[ia - 1]->as<double>(); g.A.mn = idx(1); g.A.k = idx(a1);
    g.B.ptr = P2.A[ia]->as<double>(); g.B.k = idx(1); g.B.mn = idx(b1); g.B.sb0 = (long long)b1 * b2;
    g.C.ptr = tmp.as<double>(); g.C.m = idx(1); g.C.n = idx(a1); g.C.sb0 = (long long)a1 * b2;
    TN_CHECK(gemm_f64(g, st));
    GemmArgs h;  // A_n = T[n] Ro^T   (a1 x a2): Ro is a2 x b2
    h.M = a1; h.N = a2; h.K = b2; h.nb0 = d;
    h.A.ptr = tmp.as<double>(); h.A.mn = idx(1); h.A.k = idx(a1); h.A.sb0 = (long long)a1 * b2;
    h.B.ptr = Ro[ia + 1]->as<double>(); h.B.k = idx(a2); h.B.mn = idx(1);
    h.C.ptr = A[ia]->as<double>(); h.C.m = idx(1); h.C.n = idx(a1); h.C.sb0 = (long long)a1 * a2;
    return gemm_f64(h, st);
}

// MPSImp::FindiTimeGroundState(H, schedule) (MPSImp_iTime.C:18-88).
int MPSState::itime_ground_state(const tn_itime_line* lines, int nlines, double* variance, int* iters_out) {
    cudaStream_t st = ctx->stream;
    double E1 = 0;
    TN_CHECK(expectation(H->ops, &E1));
    std::vector<std::vector<double>> sv_new(L), sv_old(L);
    // psi2's sites and the overlap environments, released on every return path
    std::vector<std::unique_ptr<DevBuf>> owned;
    auto fresh = [&owned]() {
        owned.emplace_back(new DevBuf());
        return owned.back().get();
    };
    SiteSet P2;
    P2.A.assign(L + 1, nullptr);
    for (int i = 1; i <= L; ++i) P2.A[i] = fresh();
    P2.D1.assign(L + 1, 0);
    P2.D2.assign(L + 1, 0);
    std::vector<DevBuf*> Lo(L + 2), Ro(L + 2);
    for (auto& p : Lo) p = fresh();
    for (auto& p : Ro) p = fresh();
    const double one = 1.0;
    int rc = TN_OK;
    for (int l = 0; l < nlines && rc == TN_OK; ++l) {
        const tn_itime_line& ln = lines[l];
        std::vector<SiteMPO> W;
        rc = trotter_mpo(ln.dt, ln.order, W);
        if (rc != TN_OK) break;
        int niter = 1;
        for (; niter < ln.max_iter && rc == TN_OK; ++niter) {
            sv_old = sv_new;
            // |psi2> = W |psi>
            rc = apply_mpo_inplace(W);
            if (rc != TN_OK) break;
            for (int ia = 1; ia <= L && rc == TN_OK; ++ia) {
                const size_t n = (size_t)d * D1[ia] * D2[ia];
                rc = P2.A[ia]->ensure(sizeof(double) * n);
                if (rc == TN_OK && cudaMemcpyAsync(P2.A[ia]->p, A[ia]->p, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                                   st) != cudaSuccess)
                    rc = TN_CUDA_ERROR;
                P2.D1[ia] = D1[ia];
                P2.D2[ia] = D2[ia];
            }
            if (rc != TN_OK) break;
            // compress both ways (the line's compressor), then vary towards psi2
            if ((rc = svd_compress_sweep(true, ln.Dmax, ln.eps_mps_compress, nullptr)) != TN_OK) break;
            if ((rc = svd_compress_sweep(false, ln.Dmax, ln.eps_mps_compress, &sv_new)) != TN_OK) break;
            // |psi2|^2 by the overlap sweep of psi2 with itself
            double n22 = 1.0;
            {
                // a temporary view of psi2 as "this": swap the site pointers in
                std::vector<DevBuf*> keepA = A;
                std::vector<int> k1 = D1, k2 = D2;
                for (int ia = 1; ia <= L; ++ia) {
                    A[ia] = P2.A[ia];
                    D1[ia] = P2.D1[ia];
                    D2[ia] = P2.D2[ia];
                }
                rc = Lo[0]->ensure(sizeof(double));
                if (rc == TN_OK && cudaMemcpyAsync(Lo[0]->p, &one, sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
                    rc = TN_CUDA_ERROR;
                for (int ia = 1; ia <= L && rc == TN_OK; ++ia) rc = overlap_left(ia, P2, Lo);
                if (rc == TN_OK && cudaMemcpyAsync(&n22, Lo[L]->p, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
                    rc = TN_CUDA_ERROR;
                cudaStreamSynchronize(st);
                A = keepA;
                D1 = k1;
                D2 = k2;
                if (rc != TN_OK) break;
            }
            const double nrm2 = std::sqrt(std::max(n22, 1e-300));
            // Optimize(Psi2): load the right caches, then sweep pairs
            TN_CUDA_CHECK(cudaMemcpyAsync(Lo[0]->p, &one, sizeof(double), cudaMemcpyHostToDevice, st));
            if ((rc = Ro[L + 1]->ensure(sizeof(double))) != TN_OK) break;
            TN_CUDA_CHECK(cudaMemcpyAsync(Ro[L + 1]->p, &one, sizeof(double), cudaMemcpyHostToDevice, st));
            for (int ia = L; ia >= 2 && rc == TN_OK; --ia) rc = overlap_right(ia, P2, Ro);
            if (rc != TN_OK) break;
            for (int it = 0; it < std::max(1, ln.max_opt_iter) && rc == TN_OK; ++it) {
                double ov[2] = {0, 0};
                for (int dir = 0; dir < 2 && rc == TN_OK; ++dir) {
                    const bool left = dir == 0;
                    for (int step = 0; step < L && rc == TN_OK; ++step) {
                        const int ia = left ? 1 + step : L - step;
                        if ((rc = overlap_site(ia, P2, Lo, Ro)) != TN_OK) break;
                        if ((rc = normalize_site(ia, left)) != TN_OK) break;
                        if (left) rc = overlap_left(ia, P2, Lo);
                        else rc = overlap_right(ia, P2, Ro);
                    }
                    if (rc != TN_OK) break;
                    double o = 0;
                    TN_CUDA_CHECK(cudaMemcpyAsync(&o, left ? Lo[L]->p : Ro[1]->p, sizeof(double), cudaMemcpyDeviceToHost,
                                                  st));
                    TN_CUDA_CHECK(cudaStreamSynchronize(st));
                    ov[dir] = 2.0 - 2.0 * o / nrm2;
                }
                if (rc != TN_OK) break;
                const double dO = std::fabs(ov[1] - ov[0]);
                if (dO <= ln.eps_norm) break;
            }
            if (rc != TN_OK) break;
            double Enew = 0;
            if ((rc = expectation(H->ops, &Enew)) != TN_OK) break;
            const double dE = Enew - E1;
            E1 = Enew;
            double dl = 0;
            for (int b = 1; b < L; ++b) {
                const auto& o = sv_old[b];
                const auto& x = sv_new[b];
                if (o.size() != x.size()) {
                    dl = 1.0;
                    continue;
                }
                for (size_t i = 0; i < x.size(); ++i) dl = std::max(dl, std::fabs(o[i] - x[i]));
            }
            if (std::fabs(dE) <= ln.eps_energy && dl < ln.eps_lambda) break;
            if (dE > 0.0 && niter > 1) break;
        }
        if (iters_out) iters_out[l] = niter;
    }
    TN_CHECK(rc);
    // bond bookkeeping of the sweep engine: the shapes changed
    for (int b = 1; b < L; ++b) {
        bondK[b] = D2[b];
        bond_s[b] = sv_new[b].empty() ? std::vector<double>(D2[b], 1.0 / std::sqrt((double)D2[b])) : sv_new[b];
        bondDirty[b] = 0;
    }
    if (variance) {
        double E2 = 0;
        TN_CHECK(expectation(H->ops2, &E2));
        *variance = E2 - E1 * E1;
    }
    return TN_OK;
}

}  // namespace tnb
