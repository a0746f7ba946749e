// tn_oracle.cpp -- FP64 CPU oracle for the variational ground-state sweep.
//
// TEST INFRASTRUCTURE ONLY (see tn_oracle.h).  Every routine below restates
// the reference algorithm of JanReimers/TensorNetworks; the citation next to
// each function names the reference file:line it follows.  The product CUDA
// library never loads this code.
#include "tn_oracle.h"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <limits>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

using std::vector;
typedef vector<double> Vec;

// ---------------------------------------------------------------------------
// Column-major dense matrix helpers
// ---------------------------------------------------------------------------
struct Mat {
    int r = 0, c = 0;
    Vec a;
    Mat() {}
    Mat(int r_, int c_) : r(r_), c(c_), a((size_t)r_ * c_, 0.0) {}
    double& operator()(int i, int j) { return a[(size_t)j * r + i]; }
    double operator()(int i, int j) const { return a[(size_t)j * r + i]; }
    double* col(int j) { return a.data() + (size_t)j * r; }
    const double* col(int j) const { return a.data() + (size_t)j * r; }
};

// C(MxN) = alpha*op(A)*op(B) + beta*C, column-major with leading dimensions.
static void gemm(bool ta, bool tb, int M, int N, int K, double alpha,
                 const double* A, int lda, const double* B, int ldb,
                 double beta, double* C, int ldc) {
    if (M <= 0 || N <= 0) return;
    // Pack op(A) as column-major M x K so the inner loop is unit stride.
    Vec Ap;
    const double* Ac = A;
    int ldac = lda;
    if (ta) {
        Ap.resize((size_t)M * K);
        for (int k = 0; k < K; ++k)
            for (int i = 0; i < M; ++i) Ap[(size_t)k * M + i] = A[(size_t)i * lda + k];
        Ac = Ap.data();
        ldac = M;
    }
    long long work = (long long)M * N * K;
#pragma omp parallel for schedule(static) if (work > 200000)
    for (int j = 0; j < N; ++j) {
        double* cj = C + (size_t)j * ldc;
        if (beta == 0.0) {
            for (int i = 0; i < M; ++i) cj[i] = 0.0;
        } else if (beta != 1.0) {
            for (int i = 0; i < M; ++i) cj[i] *= beta;
        }
        for (int k = 0; k < K; ++k) {
            double b = tb ? B[(size_t)k * ldb + j] : B[(size_t)j * ldb + k];
            if (b == 0.0) continue;
            b *= alpha;
            const double* ak = Ac + (size_t)k * ldac;
            for (int i = 0; i < M; ++i) cj[i] += ak[i] * b;
        }
    }
}

static double dot(const double* x, const double* y, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

// ---------------------------------------------------------------------------
// Seeded uniform(-1,1): mt19937_64, 53-bit mantissa.
// The reference's FillRandom comes from the un-vendored oml library
// (MPSSite.C:119-127); this generator is this project's documented stand-in.
// ---------------------------------------------------------------------------
static void uniform_fill(unsigned long long seed, long long offset, long long count, double* out) {
    std::mt19937_64 g(seed);
    if (offset > 0) g.discard((unsigned long long)offset);
    for (long long i = 0; i < count; ++i) {
        unsigned long long x = g();
        double u = (double)(x >> 11) * (1.0 / 9007199254740992.0);
        out[i] = 2.0 * u - 1.0;
    }
}

// ---------------------------------------------------------------------------
// Spin operators (SpinCalculator.C:20-70): basis index n <-> Sz = n - S.
// ---------------------------------------------------------------------------
static double spin_of(int n, double S) { return n - S; }
static double op_sp(int m, int n, double S) {
    return (m == n + 1) ? std::sqrt(S * (S + 1.0) - spin_of(m, S) * spin_of(n, S)) : 0.0;
}
static double op_sm(int m, int n, double S) {
    return (m + 1 == n) ? std::sqrt(S * (S + 1.0) - spin_of(m, S) * spin_of(n, S)) : 0.0;
}
static double op_sz(int m, int n, double S) { return (m == n) ? spin_of(m, S) : 0.0; }
static double op_i(int m, int n) { return (m == n) ? 1.0 : 0.0; }

static int d_of(double S) { return (int)std::lround(2.0 * S + 1.0); }

// Bulk W of the nearest-neighbour Heisenberg/XXZ chain
// (Hamiltonian_1D_NN_Heisenberg.C:35-79).  form 1 = RegularUpper, 2 = RegularLower.
static Vec heisenberg_w(double S, int form, double Jxy, double Jz, double hz) {
    const int d = d_of(S), Dw = 5;
    Vec W((size_t)Dw * Dw * d * d, 0.0);
    auto set = [&](int w1, int w2, int which, double f) {
        for (int m = 0; m < d; ++m)
            for (int n = 0; n < d; ++n) {
                double v = 0;
                switch (which) {
                    case 0: v = op_i(m, n); break;
                    case 1: v = op_sp(m, n, S); break;
                    case 2: v = op_sm(m, n, S); break;
                    case 3: v = op_sz(m, n, S); break;
                }
                W[(((size_t)w1 * Dw + w2) * d + m) * d + n] = f * v;
            }
    };
    if (form == 2) {  // RegularLower
        set(0, 0, 0, 1.0);
        set(1, 0, 1, 1.0);
        set(2, 0, 2, 1.0);
        set(3, 0, 3, 1.0);
        set(4, 0, 3, hz);
        set(4, 1, 2, Jxy / 2.0);
        set(4, 2, 1, Jxy / 2.0);
        set(4, 3, 3, Jz);
        set(4, 4, 0, 1.0);
    } else {  // RegularUpper
        set(0, 0, 0, 1.0);
        set(0, 1, 1, 1.0);
        set(0, 2, 2, 1.0);
        set(0, 3, 3, 1.0);
        set(0, 4, 3, hz);
        set(1, 4, 2, Jxy / 2.0);
        set(2, 4, 1, Jxy / 2.0);
        set(3, 4, 3, Jz);
        set(4, 4, 0, 1.0);
    }
    return W;
}

// Site operator with the open-boundary rows/columns applied
// (SiteOperatorImp.C:33-51 and Init_lr :109-134): the left edge keeps row
// Dw-1 (lower) / row 0 (upper); the right edge keeps column 0 (lower) /
// column Dw-1 (upper).
struct SiteOp {
    int Dw1 = 1, Dw2 = 1, d = 2;
    Vec W;  // (w1,w2,m,n)
    double at(int w1, int w2, int m, int n) const {
        return W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
    }
};

static SiteOp make_site_op(int L, double S, int form, double Jxy, double Jz, double hz, int site) {
    const int d = d_of(S), Dw = 5;
    Vec Wb = heisenberg_w(S, form, Jxy, Jz, hz);
    SiteOp op;
    op.d = d;
    int rowKeep = (form == 2) ? Dw - 1 : 0;
    int colKeep = (form == 2) ? 0 : Dw - 1;
    bool left = (site == 1), right = (site == L);
    op.Dw1 = left ? 1 : Dw;
    op.Dw2 = right ? 1 : Dw;
    op.W.assign((size_t)op.Dw1 * op.Dw2 * d * d, 0.0);
    for (int a = 0; a < op.Dw1; ++a)
        for (int b = 0; b < op.Dw2; ++b) {
            int w1 = left ? rowKeep : a;
            int w2 = right ? colKeep : b;
            for (int m = 0; m < d; ++m)
                for (int n = 0; n < d; ++n)
                    op.W[(((size_t)a * op.Dw2 + b) * d + m) * d + n] =
                        Wb[(((size_t)w1 * Dw + w2) * d + m) * d + n];
        }
    return op;
}

// Product MPO site operator (MPO::Product, MPO.C:73-79): (W*W)[(w1,v1),(w2,v2)](m,n)
// = sum_k W[w1,w2](m,k) W[v1,v2](k,n).  Used for <H^2> (Hamiltonian.C:8-16);
// the reference then Parker-compresses it, which leaves the expectation value
// unchanged to its compression epsilon, so the uncompressed product is used.
static SiteOp product_op(const SiteOp& A, const SiteOp& B) {
    SiteOp P;
    P.d = A.d;
    int d = A.d;
    P.Dw1 = A.Dw1 * B.Dw1;
    P.Dw2 = A.Dw2 * B.Dw2;
    P.W.assign((size_t)P.Dw1 * P.Dw2 * d * d, 0.0);
    for (int w1 = 0; w1 < A.Dw1; ++w1)
        for (int v1 = 0; v1 < B.Dw1; ++v1)
            for (int w2 = 0; w2 < A.Dw2; ++w2)
                for (int v2 = 0; v2 < B.Dw2; ++v2) {
                    int r = w1 * B.Dw1 + v1, c = w2 * B.Dw2 + v2;
                    for (int m = 0; m < d; ++m)
                        for (int n = 0; n < d; ++n) {
                            double s = 0;
                            for (int k = 0; k < d; ++k) s += A.at(w1, w2, m, k) * B.at(v1, v2, k, n);
                            P.W[(((size_t)r * P.Dw2 + c) * d + m) * d + n] = s;
                        }
                }
    return P;
}

// ---------------------------------------------------------------------------
// Environments and the effective Hamiltonian
// ---------------------------------------------------------------------------
// Left environment recursion (MPSSite::IterateLeft_F, MPSSite_Contractions.C:292-345):
//   F'(w2,i2,j2) = sum_{m,i1} A(m,i1,i2) sum_{n,w1} W(w1,w2)(m,n) sum_{j1} F(w1,i1,j1) A(n,j1,j2)
// staged as P[w1][n] = F_w1 A_n ; Q[m][w2] = sum W P ; F'_w2 = sum_m A_m^T Q[m][w2].
static void env_left(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                     const double* A, const double* F, double* Fout) {
    size_t blk = (size_t)D1 * D2;
    Vec P((size_t)Dw1 * d * blk), Q((size_t)d * Dw2 * blk);
    for (int w1 = 0; w1 < Dw1; ++w1)
        for (int n = 0; n < d; ++n)
            gemm(false, false, D1, D2, D1, 1.0, F + (size_t)w1 * D1 * D1, D1, A + n * blk, D1, 0.0,
                 P.data() + ((size_t)w1 * d + n) * blk, D1);
    std::fill(Q.begin(), Q.end(), 0.0);
    for (int w1 = 0; w1 < Dw1; ++w1)
        for (int w2 = 0; w2 < Dw2; ++w2)
            for (int m = 0; m < d; ++m)
                for (int n = 0; n < d; ++n) {
                    double c = W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
                    if (c == 0.0) continue;
                    double* q = Q.data() + ((size_t)m * Dw2 + w2) * blk;
                    const double* p = P.data() + ((size_t)w1 * d + n) * blk;
                    for (size_t t = 0; t < blk; ++t) q[t] += c * p[t];
                }
    for (int w2 = 0; w2 < Dw2; ++w2) {
        double* out = Fout + (size_t)w2 * D2 * D2;
        for (int m = 0; m < d; ++m)
            gemm(true, false, D2, D2, D1, 1.0, A + m * blk, D1, Q.data() + ((size_t)m * Dw2 + w2) * blk,
                 D1, m == 0 ? 0.0 : 1.0, out, D2);
    }
}

// Right environment recursion (MPSSite::IterateRightF, MPSSite_Contractions.C:352-400):
//   G'(w1,i1,j1) = sum_{m,i2} A(m,i1,i2) sum_{n,w2} W(w1,w2)(m,n) sum_{j2} G(w2,i2,j2) A(n,j1,j2)
// staged as P[w2][n] = G_w2 A_n^T ; Q[m][w1] = sum W P ; G'_w1 = sum_m A_m Q[m][w1].
static void env_right(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                      const double* A, const double* G, double* Gout) {
    size_t blk = (size_t)D1 * D2;
    Vec P((size_t)Dw2 * d * blk), Q((size_t)d * Dw1 * blk);
    for (int w2 = 0; w2 < Dw2; ++w2)
        for (int n = 0; n < d; ++n)
            gemm(false, true, D2, D1, D2, 1.0, G + (size_t)w2 * D2 * D2, D2, A + n * blk, D1, 0.0,
                 P.data() + ((size_t)w2 * d + n) * blk, D2);
    std::fill(Q.begin(), Q.end(), 0.0);
    for (int w1 = 0; w1 < Dw1; ++w1)
        for (int w2 = 0; w2 < Dw2; ++w2)
            for (int m = 0; m < d; ++m)
                for (int n = 0; n < d; ++n) {
                    double c = W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
                    if (c == 0.0) continue;
                    double* q = Q.data() + ((size_t)m * Dw1 + w1) * blk;
                    const double* p = P.data() + ((size_t)w2 * d + n) * blk;
                    for (size_t t = 0; t < blk; ++t) q[t] += c * p[t];
                }
    for (int w1 = 0; w1 < Dw1; ++w1) {
        double* out = Gout + (size_t)w1 * D1 * D1;
        for (int m = 0; m < d; ++m)
            gemm(false, false, D1, D1, D2, 1.0, A + m * blk, D1, Q.data() + ((size_t)m * Dw1 + w1) * blk,
                 D2, m == 0 ? 0.0 : 1.0, out, D1);
    }
}

// Heff x = sum_{w1,w2,n} W(w1,w2)(m,n) F_w1 x_n G_w2^T, the matrix-free form of
// MPSSite::GetHeff (MPSSite_Contractions.C:155-193).
static void heff_matvec(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                        const double* F, const double* G, const double* x, double* y) {
    size_t blk = (size_t)D1 * D2;
    Vec P((size_t)Dw1 * d * blk), Q((size_t)d * Dw2 * blk);
    for (int w1 = 0; w1 < Dw1; ++w1)
        for (int n = 0; n < d; ++n)
            gemm(false, false, D1, D2, D1, 1.0, F + (size_t)w1 * D1 * D1, D1, x + n * blk, D1, 0.0,
                 P.data() + ((size_t)w1 * d + n) * blk, D1);
    std::fill(Q.begin(), Q.end(), 0.0);
    for (int w1 = 0; w1 < Dw1; ++w1)
        for (int w2 = 0; w2 < Dw2; ++w2)
            for (int m = 0; m < d; ++m)
                for (int n = 0; n < d; ++n) {
                    double c = W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
                    if (c == 0.0) continue;
                    double* q = Q.data() + ((size_t)m * Dw2 + w2) * blk;
                    const double* p = P.data() + ((size_t)w1 * d + n) * blk;
                    for (size_t t = 0; t < blk; ++t) q[t] += c * p[t];
                }
    for (int m = 0; m < d; ++m) {
        double* ym = y + m * blk;
        for (int w2 = 0; w2 < Dw2; ++w2)
            gemm(false, true, D1, D2, D2, 1.0, Q.data() + ((size_t)m * Dw2 + w2) * blk, D1,
                 G + (size_t)w2 * D2 * D2, D2, w2 == 0 ? 0.0 : 1.0, ym, D1);
    }
}

// ---------------------------------------------------------------------------
// Symmetric eigenproblems
// ---------------------------------------------------------------------------
// Sturm count: number of eigenvalues of the tridiagonal (a,b) below x.
static int sturm_count(int n, const double* a, const double* b, double x) {
    int cnt = 0;
    double q = a[0] - x;
    const double tiny = 1e-300;
    if (q < 0) ++cnt;
    for (int i = 1; i < n; ++i) {
        if (std::fabs(q) < tiny) q = (q < 0 ? -tiny : tiny);
        q = (a[i] - x) - b[i - 1] * b[i - 1] / q;
        if (q < 0) ++cnt;
    }
    return cnt;
}

// k-th smallest eigenvalue (0-based) of a symmetric tridiagonal by bisection
// (the dstebz step of zheevx RANGE='I', LapackEigenSolver.C:62-109).
static double tridiag_bisect(int n, const double* a, const double* b, int k) {
    double lo = a[0], hi = a[0];
    for (int i = 0; i < n; ++i) {
        double r = (i > 0 ? std::fabs(b[i - 1]) : 0) + (i < n - 1 ? std::fabs(b[i]) : 0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    double scale = std::max(std::fabs(lo), std::fabs(hi));
    lo -= 1e-14 * scale + 1e-300;
    hi += 1e-14 * scale + 1e-300;
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(n, a, b, mid) > k) hi = mid; else lo = mid;
    }
    return 0.5 * (lo + hi);
}

// Tridiagonal solve (T - shift) x = rhs with partial pivoting (LU of a
// tridiagonal as in LAPACK dlagtf/dlagts), overwriting rhs.
static void tridiag_solve_shifted(int n, const double* a, const double* b, double shift, double pivmin, double* rhs) {
    vector<double> dl(n), dd(n), du(n), du2(n);
    vector<int> piv(n);
    for (int i = 0; i < n; ++i) dd[i] = a[i] - shift;
    for (int i = 0; i < n - 1; ++i) { dl[i] = b[i]; du[i] = b[i]; }
    for (int i = 0; i < n - 1; ++i) {
        du2[i] = 0;
        if (std::fabs(dd[i]) >= std::fabs(dl[i])) {
            piv[i] = 0;
            if (std::fabs(dd[i]) < pivmin) dd[i] = (dd[i] < 0 ? -pivmin : pivmin);
            double f = dl[i] / dd[i];
            dl[i] = f;
            dd[i + 1] -= f * du[i];
        } else {
            piv[i] = 1;
            double f = dd[i] / dl[i];
            dd[i] = dl[i];
            dl[i] = f;
            double t = du[i];
            du[i] = dd[i + 1];
            dd[i + 1] = t - f * du[i];
            if (i < n - 2) {
                du2[i] = du[i + 1];
                du[i + 1] = -f * du[i + 1];
            }
        }
    }
    if (std::fabs(dd[n - 1]) < pivmin) dd[n - 1] = (dd[n - 1] < 0 ? -pivmin : pivmin);
    // forward
    for (int i = 0; i < n - 1; ++i) {
        if (piv[i] == 0) rhs[i + 1] -= dl[i] * rhs[i];
        else { double t = rhs[i]; rhs[i] = rhs[i + 1]; rhs[i + 1] = t - dl[i] * rhs[i]; }
    }
    // back
    rhs[n - 1] /= dd[n - 1];
    if (n > 1) rhs[n - 2] = (rhs[n - 2] - du[n - 2] * rhs[n - 1]) / dd[n - 2];
    for (int i = n - 3; i >= 0; --i)
        rhs[i] = (rhs[i] - du[i] * rhs[i + 1] - du2[i] * rhs[i + 2]) / dd[i];
}

// Lowest k eigenpairs of a symmetric tridiagonal: bisection + inverse
// iteration with reorthogonalisation inside the found set (dstebz + dstein).
static void tridiag_lowest(int n, const double* a, const double* b, int k, double* theta, double* Y) {
    for (int j = 0; j < k; ++j) {
        theta[j] = tridiag_bisect(n, a, b, j);
        double* y = Y + (size_t)j * n;
        double scale = 0;
        for (int i = 0; i < n; ++i) scale = std::max(scale, std::fabs(a[i]) + (i < n - 1 ? std::fabs(b[i]) : 0));
        scale = std::max(scale, 1e-300);
        // The shift sits a few ulps of ||T|| off the eigenvalue and tiny pivots
        // are floored at eps*||T|| (as dstein), so the solve never overflows.
        double pert = 4e-15 * scale;
        double pivmin = 2.2e-16 * scale;
        for (int i = 0; i < n; ++i) y[i] = 1.0 / std::sqrt((double)n) * (1.0 + 0.1 * ((i * 7919 + j * 104729) % 97) / 97.0);
        for (int it = 0; it < 3; ++it) {
            tridiag_solve_shifted(n, a, b, theta[j] + pert, pivmin, y);
            double mx = 0;
            for (int i = 0; i < n; ++i) mx = std::max(mx, std::fabs(y[i]));
            if (mx > 0) for (int i = 0; i < n; ++i) y[i] /= mx;
            for (int p = 0; p < j; ++p) {
                double c = dot(y, Y + (size_t)p * n, n);
                for (int i = 0; i < n; ++i) y[i] -= c * Y[(size_t)p * n + i];
            }
            double nr = std::sqrt(dot(y, y, n));
            if (nr == 0) { y[j % n] = 1; nr = 1; }
            for (int i = 0; i < n; ++i) y[i] /= nr;
        }
        // Deterministic sign: largest-magnitude component positive.
        int im = 0;
        for (int i = 1; i < n; ++i) if (std::fabs(y[i]) > std::fabs(y[im])) im = i;
        if (y[im] < 0) for (int i = 0; i < n; ++i) y[i] = -y[i];
    }
}

// Householder tridiagonalisation of a dense symmetric matrix (the zhetrd step
// of zheevx): returns the diagonal/off-diagonal and the reflectors so that
// eigenvectors can be back-transformed (zunmtr).
struct Tridiag {
    int n;
    Vec a, b;
    Mat V;   // reflector vectors, column k acts on rows k+1..n-1
    Vec tau;
};

static Tridiag householder_tridiag(Mat A) {
    int n = A.r;
    Tridiag T;
    T.n = n;
    T.a.assign(n, 0);
    T.b.assign(std::max(n - 1, 0), 0);
    T.V = Mat(n, std::max(n - 1, 1));
    T.tau.assign(std::max(n - 1, 1), 0);
    Vec v(n), p(n), w(n);
    for (int k = 0; k < n - 2; ++k) {
        double alpha = 0;
        for (int i = k + 1; i < n; ++i) alpha += A(i, k) * A(i, k);
        alpha = std::sqrt(alpha);
        double x0 = A(k + 1, k);
        if (alpha == 0) { T.tau[k] = 0; continue; }
        double beta = (x0 >= 0) ? -alpha : alpha;
        // v = x - beta e1, tau = (beta - x0)/beta, scaled so v[k+1] = 1
        double v0 = x0 - beta;
        for (int i = 0; i < n; ++i) v[i] = 0;
        v[k + 1] = 1.0;
        for (int i = k + 2; i < n; ++i) v[i] = A(i, k) / v0;
        double tau = (beta - x0) / beta;
        T.tau[k] = tau;
        for (int i = k + 1; i < n; ++i) T.V(i, k) = v[i];
        // A <- H A H with H = I - tau v v^T on the trailing block
        for (int i = k; i < n; ++i) {
            double s = 0;
            for (int j = k + 1; j < n; ++j) s += A(i, j) * v[j];
            p[i] = tau * s;
        }
        double K = 0;
        for (int i = k + 1; i < n; ++i) K += v[i] * p[i];
        K *= 0.5 * tau;
        for (int i = k; i < n; ++i) w[i] = p[i] - K * v[i];
        w[k] = p[k];
        for (int i = k + 1; i < n; ++i)
            for (int j = k + 1; j < n; ++j) A(i, j) -= v[i] * w[j] + w[i] * v[j];
        A(k + 1, k) = beta;
        A(k, k + 1) = beta;
        for (int i = k + 2; i < n; ++i) { A(i, k) = 0; A(k, i) = 0; }
    }
    for (int i = 0; i < n; ++i) T.a[i] = A(i, i);
    for (int i = 0; i < n - 1; ++i) T.b[i] = A(i + 1, i);
    return T;
}

// Lowest k eigenpairs of a dense symmetric matrix: restates zheevx with
// RANGE='I', IL=1, IU=k (LapackEigenSolver.C:62-109).
static void dense_lowest(const Mat& A, int k, Vec& w, Mat& U) {
    int n = A.r;
    w.assign(k, 0);
    U = Mat(n, k);
    if (n == 1) { w[0] = A(0, 0); U(0, 0) = 1; return; }
    Tridiag T = householder_tridiag(A);
    Vec Y((size_t)k * n);
    tridiag_lowest(n, T.a.data(), T.b.data(), k, w.data(), Y.data());
    for (int j = 0; j < k; ++j) {
        double* u = U.col(j);
        for (int i = 0; i < n; ++i) u[i] = Y[(size_t)j * n + i];
        // back-transform: u = H_0 H_1 ... H_{n-3} y
        for (int r = n - 3; r >= 0; --r) {
            double tau = T.tau[r];
            if (tau == 0) continue;
            double s = u[r + 1];
            for (int i = r + 2; i < n; ++i) s += T.V(i, r) * u[i];
            s *= tau;
            u[r + 1] -= s;
            for (int i = r + 2; i < n; ++i) u[i] -= s * T.V(i, r);
        }
    }
}

// Cyclic Jacobi for all eigenpairs (small matrices only; used by tests).
static void jacobi_eigh(Mat A, Vec& w, Mat& V) {
    int n = A.r;
    V = Mat(n, n);
    for (int i = 0; i < n; ++i) V(i, i) = 1;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, tot = 0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) { tot += A(i, j) * A(i, j); if (i != j) off += A(i, j) * A(i, j); }
        if (off <= 1e-30 * std::max(tot, 1e-300)) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A(p, q);
                if (std::fabs(apq) < 1e-300) continue;
                double theta = (A(q, q) - A(p, p)) / (2 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V(k, p), vkq = V(k, q);
                    V(k, p) = c * vkp - s * vkq;
                    V(k, q) = s * vkp + c * vkq;
                }
            }
    }
    vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return A(x, x) < A(y, y); });
    w.assign(n, 0);
    Mat Vs(n, n);
    for (int j = 0; j < n; ++j) {
        w[j] = A(idx[j], idx[j]);
        for (int i = 0; i < n; ++i) Vs(i, j) = V(i, idx[j]);
    }
    V = Vs;
}

// ---------------------------------------------------------------------------
// QR and SVD
// ---------------------------------------------------------------------------
// Thin Householder QR (the dgeqrf + dorgqr pair of LapackQRSolver::SolveThinQR,
// LapackQRSolver.C:116-160): A (m x n) = Q (m x k) R (k x n), k = min(m,n).
// A zero column yields a zero R row and an orthonormal completion column of Q.
static void householder_qr(const Mat& Ain, Mat& Q, Mat& R) {
    int m = Ain.r, n = Ain.c, k = std::min(m, n);
    Mat A = Ain;
    Vec tau(k, 0.0);
    for (int j = 0; j < k; ++j) {
        // dlarfg convention: no reflection when the sub-column is already zero
        double xn2 = 0;
        for (int i = j + 1; i < m; ++i) xn2 += A(i, j) * A(i, j);
        double x0 = A(j, j);
        if (xn2 == 0.0) { tau[j] = 0; continue; }
        double nrm = std::sqrt(x0 * x0 + xn2);
        double beta = (x0 >= 0) ? -nrm : nrm;
        double v0 = x0 - beta;
        for (int i = j + 1; i < m; ++i) A(i, j) /= v0;
        tau[j] = (beta - x0) / beta;
        A(j, j) = beta;
        for (int c = j + 1; c < n; ++c) {
            double s = A(j, c);
            for (int i = j + 1; i < m; ++i) s += A(i, j) * A(i, c);
            s *= tau[j];
            A(j, c) -= s;
            for (int i = j + 1; i < m; ++i) A(i, c) -= s * A(i, j);
        }
    }
    R = Mat(k, n);
    for (int c = 0; c < n; ++c)
        for (int r = 0; r <= std::min(c, k - 1); ++r) R(r, c) = A(r, c);
    Q = Mat(m, k);
    for (int i = 0; i < k; ++i) Q(i, i) = 1.0;
    for (int j = k - 1; j >= 0; --j) {
        if (tau[j] == 0) continue;
        for (int c = j; c < k; ++c) {
            double s = Q(j, c);
            for (int i = j + 1; i < m; ++i) s += A(i, j) * Q(i, c);
            s *= tau[j];
            Q(j, c) -= s;
            for (int i = j + 1; i < m; ++i) Q(i, c) -= s * A(i, j);
        }
    }
}

static Mat transpose(const Mat& A) {
    Mat T(A.c, A.r);
    for (int j = 0; j < A.c; ++j)
        for (int i = 0; i < A.r; ++i) T(j, i) = A(i, j);
    return T;
}

// Complete the columns of U flagged in `bad` to an orthonormal set, by
// Gram-Schmidt (twice) of unit vectors against the columns already present.
static void complete_columns(Mat& U, const vector<char>& bad) {
    int m = U.r, k = U.c;
    vector<char> have(k);
    for (int j = 0; j < k; ++j) have[j] = !bad[j];
    int e = 0;
    for (int j = 0; j < k; ++j) {
        if (have[j]) continue;
        Vec v(m);
        for (; e < m; ++e) {
            std::fill(v.begin(), v.end(), 0.0);
            v[e] = 1.0;
            for (int pass = 0; pass < 2; ++pass)
                for (int p = 0; p < k; ++p) {
                    if (!have[p]) continue;
                    double c = dot(U.col(p), v.data(), m);
                    for (int i = 0; i < m; ++i) v[i] -= c * U(i, p);
                }
            double nr = std::sqrt(dot(v.data(), v.data(), m));
            if (nr > 0.5) {
                for (int i = 0; i < m; ++i) U(i, j) = v[i] / nr;
                have[j] = 1;
                ++e;
                break;
            }
        }
    }
}

// One-sided (Hestenes) Jacobi SVD of a tall matrix (m >= n):
// A V = U diag(s); returns U (m x n), s (n, descending), V (n x n).
static void jacobi_svd_tall(const Mat& Ain, Mat& U, Vec& s, Mat& V, bool wantVectors) {
    int m = Ain.r, n = Ain.c;
    Mat A = Ain;
    V = Mat(n, n);
    for (int i = 0; i < n; ++i) V(i, i) = 1.0;
    const double eps = 1e-15;
    for (int sweep = 0; sweep < 80; ++sweep) {
        int rotated = 0;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double alpha = dot(A.col(p), A.col(p), m);
                double beta = dot(A.col(q), A.col(q), m);
                double gamma = dot(A.col(p), A.col(q), m);
                if (std::fabs(gamma) <= eps * std::sqrt(alpha * beta) || gamma == 0.0) continue;
                ++rotated;
                double zeta = (beta - alpha) / (2.0 * gamma);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                double c = 1.0 / std::sqrt(1.0 + t * t), sn = c * t;
                double* ap = A.col(p);
                double* aq = A.col(q);
                for (int i = 0; i < m; ++i) {
                    double x = ap[i], y = aq[i];
                    ap[i] = c * x - sn * y;
                    aq[i] = sn * x + c * y;
                }
                if (wantVectors) {
                    double* vp = V.col(p);
                    double* vq = V.col(q);
                    for (int i = 0; i < n; ++i) {
                        double x = vp[i], y = vq[i];
                        vp[i] = c * x - sn * y;
                        vq[i] = sn * x + c * y;
                    }
                }
            }
        if (!rotated) break;
    }
    Vec nrm(n);
    for (int j = 0; j < n; ++j) nrm[j] = std::sqrt(dot(A.col(j), A.col(j), m));
    vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return nrm[x] > nrm[y]; });
    s.assign(n, 0);
    for (int j = 0; j < n; ++j) s[j] = nrm[idx[j]];
    if (!wantVectors) return;
    U = Mat(m, n);
    Mat Vs(n, n);
    vector<char> bad(n, 0);
    double smax = n > 0 ? s[0] : 0;
    double cut = smax * 1e-13 * std::max(1, m);
    for (int j = 0; j < n; ++j) {
        int src = idx[j];
        for (int i = 0; i < n; ++i) Vs(i, j) = V(i, src);
        if (s[j] > cut && s[j] > 0) {
            for (int i = 0; i < m; ++i) U(i, j) = A(i, src) / s[j];
        } else {
            bad[j] = 1;
        }
    }
    complete_columns(U, bad);
    V = Vs;
}

// Thin SVD A = U s Vt (LapackSVDSolver::Solve, LapackSVDSolver.C:42-90).
static void svd_thin(const Mat& A, Mat& U, Vec& s, Mat& Vt) {
    int m = A.r, n = A.c;
    if (m >= n) {
        Mat V;
        jacobi_svd_tall(A, U, s, V, true);
        Vt = transpose(V);
    } else {
        Mat U2, V2;
        jacobi_svd_tall(transpose(A), U2, s, V2, true);
        U = V2;                 // m x m
        Vt = transpose(U2);     // m x n
    }
}

static Vec svd_values(const Mat& A) {
    Mat U, V;
    Vec s;
    if (A.r >= A.c) jacobi_svd_tall(A, U, s, V, false);
    else jacobi_svd_tall(transpose(A), U, s, V, false);
    return s;
}

// ---------------------------------------------------------------------------
// Restarted Lanczos for the lowest eigenpair of Heff (the CUDA path's
// eigensolver; replaces the dense zheevx of MPSSite::Refine,
// MPSSite_Variational.C:18-33).  Full reorthogonalisation, classical
// Gram-Schmidt applied twice, FP64 tridiagonal eigenproblem.
// ---------------------------------------------------------------------------
template <class MV>
static int lanczos(MV matvec, size_t N, double* x, int m, int maxRestarts, double tol,
                   double* thetaOut, double* residOut, double* theta2Out) {
    int matvecs = 0;
    double nx = std::sqrt(dot(x, x, N));
    if (!(nx > 0)) {
        uniform_fill(0x9E3779B97F4A7C15ULL, 0, (long long)N, x);
        nx = std::sqrt(dot(x, x, N));
    }
    if (N == 1) {
        double y;
        matvec(x, &y);
        *thetaOut = y / x[0];
        x[0] = 1.0;
        if (residOut) *residOut = 0;
        if (theta2Out) *theta2Out = *thetaOut;
        return 1;
    }
    int mm = (int)std::min<size_t>((size_t)m, N);
    Vec V((size_t)(mm + 1) * N), w(N), h(mm + 1), alpha(mm + 1), beta(mm + 1), theta(2), Y(2 * (mm + 1));
    double th = 0, resid = 1e300, th2 = 0;
    for (int restart = 0; restart < std::max(1, maxRestarts); ++restart) {
        nx = std::sqrt(dot(x, x, N));
        for (size_t i = 0; i < N; ++i) V[i] = x[i] / nx;
        int j = 0;
        bool done = false;
        for (j = 0; j < mm; ++j) {
            double* vj = V.data() + (size_t)j * N;
            matvec(vj, w.data());
            ++matvecs;
            double a = 0;
            for (int pass = 0; pass < 2; ++pass) {
                for (int k = 0; k <= j; ++k) h[k] = dot(V.data() + (size_t)k * N, w.data(), N);
                for (int k = 0; k <= j; ++k) {
                    const double* vk = V.data() + (size_t)k * N;
                    double c = h[k];
                    for (size_t i = 0; i < N; ++i) w[i] -= c * vk[i];
                }
                a += h[j];
            }
            alpha[j] = a;
            double b = std::sqrt(dot(w.data(), w.data(), N));
            beta[j] = b;
            int kk = std::min(2, j + 1);
            tridiag_lowest(j + 1, alpha.data(), beta.data(), kk, theta.data(), Y.data());
            th = theta[0];
            th2 = kk > 1 ? theta[1] : theta[0];
            resid = b * std::fabs(Y[j]);
            double tolEff = std::max(tol, 1e-13 * std::max(1.0, std::fabs(th)));
            if (resid <= tolEff || b <= 1e-14 * std::max(1.0, std::fabs(th))) { done = true; ++j; break; }
            if (j + 1 < mm) {
                double* vn = V.data() + (size_t)(j + 1) * N;
                for (size_t i = 0; i < N; ++i) vn[i] = w[i] / b;
            }
        }
        int nb = std::min(j, mm);
        // Ritz vector x = V y
        for (size_t i = 0; i < N; ++i) x[i] = 0;
        for (int k = 0; k < nb; ++k) {
            const double* vk = V.data() + (size_t)k * N;
            double c = Y[k];
            for (size_t i = 0; i < N; ++i) x[i] += c * vk[i];
        }
        double nr = std::sqrt(dot(x, x, N));
        for (size_t i = 0; i < N; ++i) x[i] /= nr;
        if (done) break;
    }
    *thetaOut = th;
    if (residOut) *residOut = resid;
    if (theta2Out) *theta2Out = th2;
    return matvecs;
}

// ---------------------------------------------------------------------------
// MPS with the reference's sweep semantics
// ---------------------------------------------------------------------------
struct Site {
    int D1, D2;
    Vec A;  // d*D1*D2, per-n column-major
    double Emin = 0.0, iterDE = 1.0, gapE = 0.0;
};
struct Bond {
    int D;
    Vec s;
    double maxDelta = 0.0;
};

struct Model {
    int L, d;
    double S;
    int form;
    double Jxy, Jz, hz;
    vector<SiteOp> ops;  // 1-based, ops[0] unused
};

struct MPS {
    int L, d;
    vector<Site> sites;  // 1-based
    vector<Bond> bonds;  // 1-based: bond b between sites b and b+1
    vector<Vec> Lenv;    // Lenv[ia]: left env including site ia (Dw2(ia), D2, D2); Lenv[0] boundary
    vector<Vec> Renv;    // Renv[ia]: right env including site ia; Renv[L+1] boundary
    vector<int> LenvDw, RenvDw, LenvD, RenvD;
    orc_options opt;
    long long matvecs = 0;
};

// MPSImp::InitSitesAndBonds (MPSImp.C:69-90) and MPSSite::InitializeWith(Random)
// (MPSSite.C:119-127) with the documented uniform(-1,1) generator.
static void mps_init(MPS& psi, int L, int d, int D, unsigned long long seed) {
    psi.L = L;
    psi.d = d;
    psi.sites.assign(L + 2, Site());
    psi.bonds.assign(L + 1, Bond());
    for (int b = 1; b < L; ++b) {
        psi.bonds[b].D = D;
        psi.bonds[b].s.assign(D, 1.0 / D);
    }
    long long off = 0;
    for (int ia = 1; ia <= L; ++ia) {
        Site& s = psi.sites[ia];
        s.D1 = (ia == 1) ? 1 : D;
        s.D2 = (ia == L) ? 1 : D;
        if (L == 1) { s.D1 = 1; s.D2 = 1; }
        size_t cnt = (size_t)d * s.D1 * s.D2;
        s.A.resize(cnt);
        uniform_fill(seed, off, (long long)cnt, s.A.data());
        off += (long long)cnt;
        double sc = 1.0 / std::sqrt((double)d * s.D1 * s.D2);
        for (auto& v : s.A) v *= sc;
    }
    psi.Lenv.assign(L + 2, Vec());
    psi.Renv.assign(L + 2, Vec());
    psi.LenvDw.assign(L + 2, 1);
    psi.RenvDw.assign(L + 2, 1);
    psi.LenvD.assign(L + 2, 1);
    psi.RenvD.assign(L + 2, 1);
    psi.Lenv[0] = Vec(1, 1.0);
    psi.Renv[L + 1] = Vec(1, 1.0);
}

// MPSSite::NewBondDimensions (MPSSite.C:156-171): resize keeping the old
// top-left block; new entries are zero.
static void site_resize(Site& s, int d, int D1, int D2) {
    if (s.D1 == D1 && s.D2 == D2) return;
    Vec B((size_t)d * D1 * D2, 0.0);
    for (int n = 0; n < d; ++n)
        for (int i2 = 0; i2 < std::min(D2, s.D2); ++i2)
            for (int i1 = 0; i1 < std::min(D1, s.D1); ++i1)
                B[(size_t)n * D1 * D2 + (size_t)i2 * D1 + i1] = s.A[(size_t)n * s.D1 * s.D2 + (size_t)i2 * s.D1 + i1];
    s.A.swap(B);
    s.D1 = D1;
    s.D2 = D2;
}

// Bond::SetSingularValues (Bond.C:86-106).
static void bond_set_sv(Bond& b, const Vec& s) {
    double nrm = std::sqrt(dot(s.data(), s.data(), s.size()));
    Vec sn(s.size());
    for (size_t i = 0; i < s.size(); ++i) sn[i] = nrm > 0 ? s[i] / nrm : 0.0;
    Vec old = b.s;
    old.resize(sn.size(), 0.0);
    double md = 0;
    for (size_t i = 0; i < sn.size(); ++i) md = std::max(md, std::fabs(sn[i] - old[i]));
    b.maxDelta = md;
    b.s = sn;
    b.D = (int)sn.size();
}

// Bond::NewBondDimension (Bond.C:60-84).
static void bond_new_dim(Bond& b, int D) {
    if (D > b.D) {
        double mn = *std::min_element(b.s.begin(), b.s.end());
        b.s.resize(D, mn / 10.0);
    } else {
        b.s.resize(D);
    }
    b.D = D;
    double nrm = std::sqrt(dot(b.s.data(), b.s.data(), b.s.size()));
    for (auto& v : b.s) v /= nrm;
}

// A reshaped as (d*D1) x D2 with row (n,i1) (ReshapeBeforeSVD DLeft,
// MPSSite_Contractions.C:18-33) or D1 x (d*D2) with column (n,i2) (DRight :34-44).
static Mat reshape_before(const Site& s, int d, bool left) {
    if (left) {
        Mat A(d * s.D1, s.D2);
        for (int n = 0; n < d; ++n)
            for (int i2 = 0; i2 < s.D2; ++i2)
                for (int i1 = 0; i1 < s.D1; ++i1)
                    A(n * s.D1 + i1, i2) = s.A[(size_t)n * s.D1 * s.D2 + (size_t)i2 * s.D1 + i1];
        return A;
    }
    Mat A(s.D1, d * s.D2);
    for (int n = 0; n < d; ++n)
        for (int i2 = 0; i2 < s.D2; ++i2)
            for (int i1 = 0; i1 < s.D1; ++i1)
                A(i1, n * s.D2 + i2) = s.A[(size_t)n * s.D1 * s.D2 + (size_t)i2 * s.D1 + i1];
    return A;
}

// ReshapeAfter_SVD (MPSSite_Contractions.C:49-80).
static void reshape_after(Site& s, int d, bool left, const Mat& UV) {
    if (left) {
        if (UV.c < s.D2) site_resize(s, d, s.D1, UV.c);
        for (int n = 0; n < d; ++n)
            for (int i2 = 0; i2 < s.D2; ++i2)
                for (int i1 = 0; i1 < s.D1; ++i1)
                    s.A[(size_t)n * s.D1 * s.D2 + (size_t)i2 * s.D1 + i1] = UV(n * s.D1 + i1, i2);
    } else {
        if (UV.r < s.D1) site_resize(s, d, UV.r, s.D2);
        for (int n = 0; n < d; ++n)
            for (int i2 = 0; i2 < s.D2; ++i2)
                for (int i1 = 0; i1 < s.D1; ++i1)
                    s.A[(size_t)n * s.D1 * s.D2 + (size_t)i2 * s.D1 + i1] = UV(i1, n * s.D2 + i2);
    }
}

// Neighbour update of MPSSite::SVDTransfer (MPSSite_Contractions.C:402-458):
// DLeft: M_n <- X * M_n (X = s*Vdagger or R); DRight: M_n <- M_n * X (X = U*s or L).
static void transfer(Site& nb, int d, bool left, const Mat& X) {
    if (left) {
        int k = X.r;
        Vec B((size_t)d * k * nb.D2);
        for (int n = 0; n < d; ++n)
            gemm(false, false, k, nb.D2, nb.D1, 1.0, X.a.data(), X.r, nb.A.data() + (size_t)n * nb.D1 * nb.D2,
                 nb.D1, 0.0, B.data() + (size_t)n * k * nb.D2, k);
        nb.A.swap(B);
        nb.D1 = k;
    } else {
        int k = X.c;
        Vec B((size_t)d * nb.D1 * k);
        for (int n = 0; n < d; ++n)
            gemm(false, false, nb.D1, k, nb.D2, 1.0, nb.A.data() + (size_t)n * nb.D1 * nb.D2, nb.D1, X.a.data(),
                 X.r, 0.0, B.data() + (size_t)n * nb.D1 * k, nb.D1);
        nb.A.swap(B);
        nb.D2 = k;
    }
}

// MPSSite::HandleEdges (MPSSite_Normalization.C:20-43).
static bool handle_edges(MPS& psi, int ia, bool left) {
    int L = psi.L, d = psi.d;
    Site& s = psi.sites[ia];
    bool edge = false;
    if (!left && ia == 1) {
        if (L > 1) {
            int newD2 = std::max(psi.bonds[1].D, d);
            if (newD2 < s.D2) site_resize(s, d, s.D1, newD2);
        }
        edge = true;
    }
    if (left && ia == L) {
        if (L > 1) {
            int newD1 = std::max(psi.bonds[L - 1].D, d);
            if (newD1 < s.D1) site_resize(s, d, newD1, s.D2);
        }
        edge = true;
    }
    if (edge) {
        double nrm2 = dot(s.A.data(), s.A.data(), s.A.size());
        double sc = std::sqrt(nrm2);  // Rescale(sqrt(GetNorm(lr)(1,1))): GetNorm is the 1x1 sum of squares
        if (sc > 0) for (auto& v : s.A) v /= sc;
    }
    return edge;
}

// MPSSite::SVDNormalize / NormalizeQR (MPSSite_Normalization.C:45-107) with the
// bond and neighbour updates of Bond::SVDTransfer (Bond.C:162-168).
static void normalize_site(MPS& psi, int ia, bool left, int gauge) {
    int d = psi.d;
    if (handle_edges(psi, ia, left)) return;
    Site& s = psi.sites[ia];
    Mat A = reshape_before(s, d, left);
    if (gauge == 0) {
        Mat U, Vt;
        Vec sv;
        svd_thin(A, U, sv, Vt);
        int k = (int)sv.size();
        if (left) {
            bond_set_sv(psi.bonds[ia], sv);
            Mat X = Vt;  // s * Vdagger
            for (int j = 0; j < X.c; ++j)
                for (int i = 0; i < k; ++i) X(i, j) *= sv[i];
            transfer(psi.sites[ia + 1], d, true, X);
            reshape_after(s, d, true, U);
        } else {
            bond_set_sv(psi.bonds[ia - 1], sv);
            Mat X = U;  // U * s
            for (int j = 0; j < k; ++j)
                for (int i = 0; i < X.r; ++i) X(i, j) *= sv[j];
            transfer(psi.sites[ia - 1], d, false, X);
            reshape_after(s, d, false, Vt);
        }
    } else {
        if (left) {
            Mat Q, R;
            householder_qr(A, Q, R);
            bond_set_sv(psi.bonds[ia], svd_values(R));
            transfer(psi.sites[ia + 1], d, true, R);
            reshape_after(s, d, true, Q);
        } else {
            Mat Qt, Rt;
            householder_qr(transpose(A), Qt, Rt);   // A = Rt^T Qt^T = L Q
            Mat Lm = transpose(Rt), Qm = transpose(Qt);
            bond_set_sv(psi.bonds[ia - 1], svd_values(Lm));
            transfer(psi.sites[ia - 1], d, false, Lm);
            reshape_after(s, d, false, Qm);
        }
    }
}

static void compute_left_env(MPS& psi, const Model& H, int ia) {
    const SiteOp& op = H.ops[ia];
    Site& s = psi.sites[ia];
    Vec out((size_t)op.Dw2 * s.D2 * s.D2);
    env_left(psi.d, op.Dw1, op.Dw2, s.D1, s.D2, op.W.data(), s.A.data(), psi.Lenv[ia - 1].data(), out.data());
    psi.Lenv[ia].swap(out);
    psi.LenvDw[ia] = op.Dw2;
    psi.LenvD[ia] = s.D2;
}

static void compute_right_env(MPS& psi, const Model& H, int ia) {
    const SiteOp& op = H.ops[ia];
    Site& s = psi.sites[ia];
    Vec out((size_t)op.Dw1 * s.D1 * s.D1);
    env_right(psi.d, op.Dw1, op.Dw2, s.D1, s.D2, op.W.data(), s.A.data(), psi.Renv[ia + 1].data(), out.data());
    psi.Renv[ia].swap(out);
    psi.RenvDw[ia] = op.Dw1;
    psi.RenvD[ia] = s.D1;
}

// MPSImp::LoadHeffCaches / CalcHeffRight (MPSImp_Variational.C:120-149).  The
// left caches it also builds are never read before the left-to-right sweep
// rebuilds them, so only the right caches are formed.
static void load_heff_caches(MPS& psi, const Model& H) {
    for (int ia = psi.L; ia >= 2; --ia) compute_right_env(psi, H, ia);
}

// MPSImp::Normalize(DRight) -> NormalizeAndCompress (MPSImp_Normalization.C:34-38).
static void normalize_all(MPS& psi, bool left, int gauge) {
    if (left) for (int ia = 1; ia <= psi.L; ++ia) normalize_site(psi, ia, true, gauge);
    else for (int ia = psi.L; ia >= 1; --ia) normalize_site(psi, ia, false, gauge);
}

// MPSSite::Refine (MPSSite_Variational.C:18-44).
static void refine_site(MPS& psi, const Model& H, int ia, double epsEigen) {
    int d = psi.d;
    Site& s = psi.sites[ia];
    const SiteOp& op = H.ops[ia];
    const Vec& F = psi.Lenv[ia - 1];
    const Vec& G = psi.Renv[ia + 1];
    int N = d * s.D1 * s.D2;
    double lam = 0, lam2 = 0;
    if (psi.opt.eig_mode == 0) {
        Mat Hd(N, N);
        orc_heff_dense(d, op.Dw1, op.Dw2, s.D1, s.D2, op.W.data(), F.data(), G.data(), Hd.a.data());
        Vec w;
        Mat U;
        int k = std::min(2, N);
        dense_lowest(Hd, k, w, U);
        lam = w[0];
        lam2 = k > 1 ? w[1] : w[0];
        for (int i = 0; i < N; ++i) s.A[i] = U(i, 0);
    } else {
        auto mv = [&](const double* x, double* y) {
            heff_matvec(d, op.Dw1, op.Dw2, s.D1, s.D2, op.W.data(), F.data(), G.data(), x, y);
        };
        double resid = 0;
        int nmv = lanczos(mv, (size_t)N, s.A.data(), psi.opt.krylov, psi.opt.max_restarts, epsEigen, &lam, &resid, &lam2);
        psi.matvecs += nmv;
    }
    s.iterDE = lam - s.Emin;
    s.Emin = lam;
    s.gapE = lam2 - lam;
}

// MPSImp::Sweep + MPSImp::Refine (MPSImp_Variational.C:64-99).
static void sweep(MPS& psi, const Model& H, bool left, double epsEigen) {
    int L = psi.L;
    if (left) {
        for (int ia = 1; ia <= L; ++ia) {
            refine_site(psi, H, ia, epsEigen);
            normalize_site(psi, ia, true, psi.opt.gauge);
            compute_left_env(psi, H, ia);
        }
    } else {
        for (int ia = L; ia >= 1; --ia) {
            refine_site(psi, H, ia, epsEigen);
            normalize_site(psi, ia, false, psi.opt.gauge);
            compute_right_env(psi, H, ia);
        }
    }
}

static double max_delta_e(const MPS& psi) {
    double m = 0;
    for (int ia = 1; ia <= psi.L; ++ia) m = std::max(m, std::fabs(psi.sites[ia].iterDE));
    return m;
}
static double max_delta_l(const MPS& psi) {
    double m = 0;
    for (int b = 1; b < psi.L; ++b) m = std::max(m, psi.bonds[b].maxDelta);
    return m;
}
static int max_D(const MPS& psi) {
    int D = 0;
    for (int ia = 1; ia <= psi.L; ++ia) D = std::max(D, psi.sites[ia].D2);
    return D;
}

// MPSImp::IncreaseBondDimensions (MPSImp.C:123-147).
static void increase_bond_dims(MPS& psi, int D) {
    int L = psi.L, d = psi.d;
    // Dideal = d^k saturates at D (the reference's int product overflows beyond L ~ 60)
    long long Dideal = 1;
    int ia = 1;
    for (; ia <= L / 2; ++ia) {
        int D1 = (int)std::min<long long>(Dideal, D), D2 = (int)std::min<long long>(Dideal * d, D);
        site_resize(psi.sites[ia], d, D1, D2);
        bond_new_dim(psi.bonds[ia], D2);
        Dideal = std::min<long long>(Dideal * d, D);
    }
    Dideal = 1;
    for (int ib = L; ib >= ia; --ib) {
        int D2 = (int)std::min<long long>(Dideal, D), D1 = (int)std::min<long long>(Dideal * d, D);
        site_resize(psi.sites[ib], d, D1, D2);
        bond_new_dim(psi.bonds[ib - 1], D1);
        Dideal = std::min<long long>(Dideal * d, D);
    }
}

// MPSImp::GetExpectation (MPSImp_ExpectationsAndDMs.C:33-45).
static double expectation(const MPS& psi, const vector<SiteOp>& ops) {
    Vec F(1, 1.0);
    for (int ia = 1; ia <= psi.L; ++ia) {
        const Site& s = psi.sites[ia];
        const SiteOp& op = ops[ia];
        Vec out((size_t)op.Dw2 * s.D2 * s.D2);
        env_left(psi.d, op.Dw1, op.Dw2, s.D1, s.D2, op.W.data(), s.A.data(), F.data(), out.data());
        F.swap(out);
    }
    return F[0];
}

static Model make_model(int L, double S, int form, double Jxy, double Jz, double hz) {
    Model H;
    H.L = L;
    H.S = S;
    H.d = d_of(S);
    H.form = form;
    H.Jxy = Jxy;
    H.Jz = Jz;
    H.hz = hz;
    H.ops.resize(L + 1);
    for (int ia = 1; ia <= L; ++ia) H.ops[ia] = make_site_op(L, S, form, Jxy, Jz, hz, ia);
    return H;
}

}  // namespace orc

using namespace orc;

// ===========================================================================
// extern "C" surface
// ===========================================================================
extern "C" {

void orc_uniform(unsigned long long seed, long long offset, long long count, double* out) {
    uniform_fill(seed, offset, count, out);
}

int orc_mpo_dims(int L, double S, int site, int* Dw1, int* Dw2) {
    (void)S;
    if (site < 1 || site > L) return -1;
    *Dw1 = (site == 1) ? 1 : 5;
    *Dw2 = (site == L) ? 1 : 5;
    return 0;
}

int orc_mpo_site(int L, double S, int form, double Jxy, double Jz, double hz, int site, double* W) {
    if (site < 1 || site > L) return -1;
    SiteOp op = make_site_op(L, S, form, Jxy, Jz, hz, site);
    std::memcpy(W, op.W.data(), op.W.size() * sizeof(double));
    return 0;
}

// Hamiltonian_1D_NN_Heisenberg::GetH (Hamiltonian_1D_NN_Heisenberg.C:28-33).
int orc_local_h12(double S, double Jxy, double Jz, double hz, double* H12) {
    int d = d_of(S);
    for (int ma = 0; ma < d; ++ma)
        for (int mb = 0; mb < d; ++mb)
            for (int na = 0; na < d; ++na)
                for (int nb = 0; nb < d; ++nb) {
                    double v = 0.5 * Jxy * (op_sp(ma, na, S) * op_sm(mb, nb, S) + op_sm(ma, na, S) * op_sp(mb, nb, S)) +
                               Jz * op_sz(ma, na, S) * op_sz(mb, nb, S) +
                               hz * (op_sz(ma, na, S) * op_i(mb, nb) + op_i(ma, na) * op_sz(mb, nb, S));
                    int r = ma * d + mb, c = na * d + nb;
                    H12[(size_t)c * d * d + r] = v;
                }
    return 0;
}

int orc_env_left(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* A,
                 const double* F, double* Fout) {
    env_left(d, Dw1, Dw2, D1, D2, W, A, F, Fout);
    return 0;
}
int orc_env_right(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* A,
                  const double* G, double* Gout) {
    env_right(d, Dw1, Dw2, D1, D2, W, A, G, Gout);
    return 0;
}

// Literal ContractAWFA/WFA/FA loops (MPSSite_Contractions.C:292-345).
int orc_env_left_literal(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* A,
                         const double* F, double* Fout) {
    auto Aat = [&](int n, int i1, int i2) { return A[(size_t)n * D1 * D2 + (size_t)i2 * D1 + i1]; };
    auto Fat = [&](int w, int i, int j) { return F[(size_t)w * D1 * D1 + (size_t)j * D1 + i]; };
    auto Wat = [&](int w1, int w2, int m, int n) { return W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n]; };
    for (int w2 = 0; w2 < Dw2; ++w2)
        for (int i2 = 0; i2 < D2; ++i2)
            for (int j2 = 0; j2 < D2; ++j2) {
                double awfa = 0;
                for (int m = 0; m < d; ++m)
                    for (int i1 = 0; i1 < D1; ++i1) {
                        double wfa = 0;
                        for (int n = 0; n < d; ++n)
                            for (int w1 = 0; w1 < Dw1; ++w1) {
                                double w = Wat(w1, w2, m, n);
                                if (w == 0.0) continue;
                                double fa = 0;
                                for (int j1 = 0; j1 < D1; ++j1) fa += Fat(w1, i1, j1) * Aat(n, j1, j2);
                                wfa += w * fa;
                            }
                        awfa += Aat(m, i1, i2) * wfa;
                    }
                Fout[(size_t)w2 * D2 * D2 + (size_t)j2 * D2 + i2] = awfa;
            }
    return 0;
}

// Literal ContractBWFB/WFB/FB loops (MPSSite_Contractions.C:352-400).
int orc_env_right_literal(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* A,
                          const double* G, double* Gout) {
    auto Aat = [&](int n, int i1, int i2) { return A[(size_t)n * D1 * D2 + (size_t)i2 * D1 + i1]; };
    auto Gat = [&](int w, int i, int j) { return G[(size_t)w * D2 * D2 + (size_t)j * D2 + i]; };
    auto Wat = [&](int w1, int w2, int m, int n) { return W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n]; };
    for (int w1 = 0; w1 < Dw1; ++w1)
        for (int i1 = 0; i1 < D1; ++i1)
            for (int j1 = 0; j1 < D1; ++j1) {
                double bwfb = 0;
                for (int m = 0; m < d; ++m)
                    for (int i2 = 0; i2 < D2; ++i2) {
                        double wfb = 0;
                        for (int n = 0; n < d; ++n)
                            for (int w2 = 0; w2 < Dw2; ++w2) {
                                double w = Wat(w1, w2, m, n);
                                if (w == 0.0) continue;
                                double fb = 0;
                                for (int j2 = 0; j2 < D2; ++j2) fb += Gat(w2, i2, j2) * Aat(n, j1, j2);
                                wfb += w * fb;
                            }
                        bwfb += Aat(m, i1, i2) * wfb;
                    }
                Gout[(size_t)w1 * D1 * D1 + (size_t)j1 * D1 + i1] = bwfb;
            }
    return 0;
}

int orc_heff_matvec(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* F,
                    const double* G, const double* x, double* y) {
    heff_matvec(d, Dw1, Dw2, D1, D2, W, F, G, x, y);
    return 0;
}

// Dense Heff of MPSSite::GetHeff (MPSSite_Contractions.C:155-193):
//   Heff(m,i1,i2; n,j1,j2) = sum_{w1,w2} L(w1,i1,j1) W(w1,w2)(m,n) R(w2,i2,j2),
// flattened with the site-tensor index n*D1*D2 + i2*D1 + i1.
int orc_heff_dense(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* F,
                   const double* G, double* H) {
    size_t N = (size_t)d * D1 * D2;
    for (int m = 0; m < d; ++m)
        for (int n = 0; n < d; ++n)
            for (int i2 = 0; i2 < D2; ++i2)
                for (int j2 = 0; j2 < D2; ++j2) {
                    vector<double> WR(Dw1, 0.0);
                    for (int w1 = 0; w1 < Dw1; ++w1)
                        for (int w2 = 0; w2 < Dw2; ++w2) {
                            double w = W[(((size_t)w1 * Dw2 + w2) * d + m) * d + n];
                            if (w != 0.0) WR[w1] += w * G[(size_t)w2 * D2 * D2 + (size_t)j2 * D2 + i2];
                        }
                    for (int i1 = 0; i1 < D1; ++i1)
                        for (int j1 = 0; j1 < D1; ++j1) {
                            double v = 0;
                            for (int w1 = 0; w1 < Dw1; ++w1) v += F[(size_t)w1 * D1 * D1 + (size_t)j1 * D1 + i1] * WR[w1];
                            size_t r = (size_t)m * D1 * D2 + (size_t)i2 * D1 + i1;
                            size_t c = (size_t)n * D1 * D2 + (size_t)j2 * D1 + j1;
                            H[c * N + r] = v;
                        }
                }
    return 0;
}

int orc_heff_diag(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* F,
                  const double* G, double* diag) {
    for (int m = 0; m < d; ++m)
        for (int i2 = 0; i2 < D2; ++i2)
            for (int i1 = 0; i1 < D1; ++i1) {
                double v = 0;
                for (int w1 = 0; w1 < Dw1; ++w1)
                    for (int w2 = 0; w2 < Dw2; ++w2) {
                        double w = W[(((size_t)w1 * Dw2 + w2) * d + m) * d + m];
                        if (w == 0.0) continue;
                        v += F[(size_t)w1 * D1 * D1 + (size_t)i1 * D1 + i1] * w * G[(size_t)w2 * D2 * D2 + (size_t)i2 * D2 + i2];
                    }
                diag[(size_t)m * D1 * D2 + (size_t)i2 * D1 + i1] = v;
            }
    return 0;
}

int orc_svd(int m, int n, const double* A, double* U, double* s, double* Vt) {
    Mat M(m, n);
    std::memcpy(M.a.data(), A, sizeof(double) * (size_t)m * n);
    Mat Uo, Vto;
    Vec so;
    svd_thin(M, Uo, so, Vto);
    std::memcpy(U, Uo.a.data(), sizeof(double) * Uo.a.size());
    std::memcpy(s, so.data(), sizeof(double) * so.size());
    std::memcpy(Vt, Vto.a.data(), sizeof(double) * Vto.a.size());
    return 0;
}

int orc_svd_values(int m, int n, const double* A, double* s) {
    Mat M(m, n);
    std::memcpy(M.a.data(), A, sizeof(double) * (size_t)m * n);
    Vec so = svd_values(M);
    std::memcpy(s, so.data(), sizeof(double) * so.size());
    return 0;
}

int orc_qr(int m, int n, const double* A, double* Q, double* R) {
    Mat M(m, n);
    std::memcpy(M.a.data(), A, sizeof(double) * (size_t)m * n);
    Mat Qo, Ro;
    householder_qr(M, Qo, Ro);
    std::memcpy(Q, Qo.a.data(), sizeof(double) * Qo.a.size());
    std::memcpy(R, Ro.a.data(), sizeof(double) * Ro.a.size());
    return 0;
}

// LapackQRSolver::SolveThinLQ (LapackQRSolver.C:277-320) as QR of the transpose.
int orc_lq(int m, int n, const double* A, double* Lout, double* Qout) {
    Mat M(m, n);
    std::memcpy(M.a.data(), A, sizeof(double) * (size_t)m * n);
    Mat Qt, Rt;
    householder_qr(transpose(M), Qt, Rt);
    Mat Lm = transpose(Rt), Qm = transpose(Qt);
    std::memcpy(Lout, Lm.a.data(), sizeof(double) * Lm.a.size());
    std::memcpy(Qout, Qm.a.data(), sizeof(double) * Qm.a.size());
    return 0;
}

int orc_eigh(int N, const double* A, double* w, double* V) {
    Mat M(N, N);
    std::memcpy(M.a.data(), A, sizeof(double) * (size_t)N * N);
    Vec wo;
    Mat Vo;
    jacobi_eigh(M, wo, Vo);
    std::memcpy(w, wo.data(), sizeof(double) * N);
    std::memcpy(V, Vo.a.data(), sizeof(double) * (size_t)N * N);
    return 0;
}

int orc_tridiag_lowest(int n, const double* alpha, const double* beta, int k, double* theta, double* Y) {
    if (k > n || n < 1) return -1;
    tridiag_lowest(n, alpha, beta, k, theta, Y);
    return 0;
}

int orc_lanczos_heff(int d, int Dw1, int Dw2, int D1, int D2, const double* W, const double* F,
                     const double* G, double* x, int krylov, int max_restarts, double tol,
                     double* theta_out, double* resid_out) {
    auto mv = [&](const double* xi, double* yo) { heff_matvec(d, Dw1, Dw2, D1, D2, W, F, G, xi, yo); };
    double th2 = 0;
    return lanczos(mv, (size_t)d * D1 * D2, x, krylov, max_restarts, tol, theta_out, resid_out, &th2);
}

// SVCompressorImp<T>::Compress(U,s,Vdagger) (SVCompressorImp.C:19-73).
double orc_compress(int Dmax, double eps, int m, int n, int k, double* U, double* s, double* Vt, int* k_out) {
    int N = k, D = N;
    double integratedS2 = 0.0;
    if (eps == 0.0) {
        D = Dmax;
        for (int id = D; id < N; ++id) integratedS2 += s[id] * s[id];
    } else {
        for (; D >= 1; --D) {
            double s2 = s[D - 1] * s[D - 1];
            if (integratedS2 + s2 >= eps) break;
            integratedS2 += s2;
        }
        if (Dmax > 0 && D > Dmax) D = Dmax;
    }
    if (D < N) {
        double before = 0, after = 0;
        for (int i = 0; i < N; ++i) before += s[i] * s[i];
        for (int i = 0; i < D; ++i) after += s[i] * s[i];
        double rescale = after > 0 ? before / after : 1.0;  // ratio of squares, as the reference
        for (int i = 0; i < D; ++i) s[i] *= rescale;
        // U: m x D keeps its first D columns (already contiguous).
        // Vt: k x n with leading dimension k -> D x n with leading dimension D.
        Vec tmp((size_t)D * n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < D; ++i) tmp[(size_t)j * D + i] = Vt[(size_t)j * k + i];
        std::memcpy(Vt, tmp.data(), sizeof(double) * tmp.size());
    }
    (void)m;
    *k_out = std::min(D, N);
    return integratedS2;
}

// MPSImp::FindVariationalGroundState(H,IterationSchedule) and the per-line
// driver (MPSImp_Variational.C:16-62).
int orc_find_ground_state(int L, double S, int form, double Jxy, double Jz, double hz, int Dstart,
                          unsigned long long seed, const orc_sched_line* lines, int nlines,
                          const orc_options* opt, orc_result* res, double* site_energies) {
    if (L < 2 || Dstart < 1 || !lines || nlines < 1 || !opt || !res) return -1;
#ifdef _OPENMP
    if (opt->nthreads > 0) omp_set_num_threads(opt->nthreads);
#endif
    Model H = make_model(L, S, form, Jxy, Jz, hz);
    vector<SiteOp> H2ops(L + 1);
    for (int ia = 1; ia <= L; ++ia) H2ops[ia] = product_op(H.ops[ia], H.ops[ia]);
    MPS psi;
    psi.opt = *opt;
    if (psi.opt.krylov <= 0) psi.opt.krylov = 20;
    if (psi.opt.max_restarts <= 0) psi.opt.max_restarts = 10;
    mps_init(psi, L, H.d, Dstart, seed);
    normalize_all(psi, false, psi.opt.gauge);
    load_heff_caches(psi, H);
    double E1 = 0, E2 = 0, DE2 = 0, dE = 0, dl = 0;
    int total = 0;
    for (int li = 0; li < nlines; ++li) {
        const orc_sched_line& isl = lines[li];
        int Dmax = max_D(psi);
        for (int D = Dmax; D <= isl.Dmax; D += std::max(1, isl.deltaD)) {
            if (D > Dmax) {
                increase_bond_dims(psi, D);
                normalize_all(psi, false, psi.opt.gauge);
                load_heff_caches(psi, H);
            }
            int in = 0;
            for (; in < isl.max_sweeps; ++in) {
                sweep(psi, H, true, isl.eps_eigen);
                sweep(psi, H, false, isl.eps_eigen);
                ++total;
                dE = max_delta_e(psi);
                dl = max_delta_l(psi);
                if (opt->verbose) std::printf("%4d %4d %.1e %.1e\n", in, D, dE, dl);
                if (dE < isl.eps_energy && dl < isl.eps_lambda) break;
            }
            E1 = expectation(psi, H.ops);
            E2 = expectation(psi, H2ops);
            DE2 = E2 - E1 * E1;
            if (opt->verbose)
                std::printf("Variational GS D=%4d, %4d iterations, <E>=%.11f, <E^2>-<E>^2=%.2e\n", D, in + 1,
                            E1 / (L - 1), DE2);
        }
    }
    res->energy = E1;
    res->energy2 = E2;
    res->variance = DE2;
    res->total_sweeps = total;
    res->matvecs = psi.matvecs;
    res->final_D = max_D(psi);
    res->last_dE = dE;
    res->last_dlambda = dl;
    if (site_energies)
        for (int ia = 1; ia <= L; ++ia) site_energies[ia - 1] = psi.sites[ia].Emin;
    return 0;
}

int orc_sweep_sample(int L, double S, int form, double Jxy, double Jz, double hz, const int* D1s,
                     const int* D2s, const double* sites, int first, int nsites, int krylov, int max_restarts,
                     double tol, int nthreads, double* seconds, long long* matvecs) {
    if (L < 2 || first < 1 || first + nsites - 1 > L - 1 || nsites < 1) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Model H = make_model(L, S, form, Jxy, Jz, hz);
    MPS psi;
    psi.opt.eig_mode = 1;
    psi.opt.gauge = 1;
    psi.opt.krylov = krylov > 0 ? krylov : 20;
    psi.opt.max_restarts = max_restarts > 0 ? max_restarts : 10;
    mps_init(psi, L, H.d, 1, 0);
    size_t off = 0;
    for (int ia = 1; ia <= L; ++ia) {
        Site& st = psi.sites[ia];
        st.D1 = D1s[ia - 1];
        st.D2 = D2s[ia - 1];
        size_t cnt = (size_t)H.d * st.D1 * st.D2;
        st.A.assign(sites + off, sites + off + cnt);
        off += cnt;
    }
    for (int b = 1; b < L; ++b) {
        psi.bonds[b].D = psi.sites[b].D2;
        psi.bonds[b].s.assign(psi.bonds[b].D, 1.0 / psi.bonds[b].D);
    }
    // untimed preparation: left-normalise 1..first-1, build the environments
    for (int ia = 1; ia < first; ++ia) {
        Site& s = psi.sites[ia];
        Mat A = reshape_before(s, H.d, true);
        Mat Q, R;
        householder_qr(A, Q, R);
        transfer(psi.sites[ia + 1], H.d, true, R);
        reshape_after(s, H.d, true, Q);
        compute_left_env(psi, H, ia);
    }
    for (int ia = L; ia > first; --ia) compute_right_env(psi, H, ia);
    auto t0 = std::chrono::steady_clock::now();
    for (int ia = first; ia < first + nsites; ++ia) {
        refine_site(psi, H, ia, tol);
        normalize_site(psi, ia, true, 1);
        compute_left_env(psi, H, ia);
    }
    auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    *matvecs = psi.matvecs;
    return 0;
}

// Exact diagonalisation: H = sum_bonds H12 (FullStateImp::ContractOverLattice,
// FullStateImp.C:91-133) with a Lanczos ground-state solve
// (FullStateImp::FindGroundState, FullStateImp.C:184-199).
int orc_ed_ground(int L, double S, double Jxy, double Jz, double hz, int field_mode, double tol, double* E) {
    int d = d_of(S);
    size_t N = 1;
    for (int i = 0; i < L; ++i) N *= d;
    if (N > (size_t)1 << 26) return -1;
    int dd = d * d;
    Vec H12((size_t)dd * dd);
    orc_local_h12(S, Jxy, Jz, field_mode == 1 ? hz : 0.0, H12.data());
    vector<size_t> stride(L);
    stride[L - 1] = 1;
    for (int i = L - 2; i >= 0; --i) stride[i] = stride[i + 1] * d;
    auto mv = [&](const double* x, double* y) {
#pragma omp parallel for schedule(static)
        for (long long t = 0; t < (long long)N; ++t) {
            size_t idx = (size_t)t;
            double acc = 0;
            for (int b = 0; b + 1 < L; ++b) {
                int ma = (int)((idx / stride[b]) % d), mb = (int)((idx / stride[b + 1]) % d);
                size_t base = idx - ma * stride[b] - mb * stride[b + 1];
                int r = ma * d + mb;
                for (int na = 0; na < d; ++na)
                    for (int nb = 0; nb < d; ++nb) {
                        double h = H12[(size_t)(na * d + nb) * dd + r];
                        if (h != 0.0) acc += h * x[base + na * stride[b] + nb * stride[b + 1]];
                    }
            }
            if (field_mode == 0 && hz != 0.0)
                for (int b = 0; b < L; ++b) acc += hz * spin_of((int)((idx / stride[b]) % d), S) * x[idx];
            y[idx] = acc;
        }
    };
    Vec x(N);
    uniform_fill(12345, 0, (long long)N, x.data());
    double th = 0, resid = 0, th2 = 0;
    lanczos(mv, N, x.data(), 60, 60, tol, &th, &resid, &th2);
    *E = th;
    return 0;
}

int orc_itebd(double S, double Jxy, double Jz, double hz, int D, const double* dts, const int* nsteps,
              int nlines, unsigned long long seed, double eps_sv, double* E_bond) {
    (void)S; (void)Jxy; (void)Jz; (void)hz; (void)D; (void)dts; (void)nsteps; (void)nlines; (void)seed;
    (void)eps_sv; (void)E_bond;
    return -2;  // not built yet
}

}  // extern "C"
