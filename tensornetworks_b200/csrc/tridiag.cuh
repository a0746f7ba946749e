// tridiag.cuh -- device helpers for the small symmetric tridiagonal
// eigenproblems of the Krylov solvers (Sturm multisection, last eigenvector
// component, pivoted tridiagonal solve for inverse iteration).
#pragma once
#include <cuda_runtime.h>

namespace tnb {
namespace {

// Number of eigenvalues of the symmetric tridiagonal (a, b) below x: the sign
// changes of p_0 = 1, p_k = (a_{k-1} - x) p_{k-1} - b_{k-2}^2 p_{k-2}, the
// leading principal minors of T - x.  The three-term recurrence needs no
// division (the ratio form q_k = p_k / p_{k-1} spends an FP64 division, a long
// serial latency, on every step); the pair is rescaled to stay in range.  A
// zero minor takes its predecessor's sign, as the ratio form's +pivmin does.
__device__ int sturm_count(int n, const double* a, const double* b, double x) {
    double pm = 1.0, p = a[0] - x;
    bool neg = p < 0;
    int cnt = neg;
    for (int i = 1; i < n; ++i) {
        const double pn = fma(a[i] - x, p, -(b[i - 1] * b[i - 1]) * pm);
        pm = p;
        p = pn;
        const bool ng = p < 0 ? true : (p > 0 ? false : neg);
        cnt += (ng != neg);
        neg = ng;
        const double mx = fmax(fabs(p), fabs(pm));
        if (mx > 1e150) {
            p *= 1e-150;
            pm *= 1e-150;
        } else if (mx < 1e-150 && mx > 0) {
            p *= 1e150;
            pm *= 1e150;
        }
    }
    return cnt;
}

// k-th smallest eigenvalue by block-wide multisection: every round each
// thread evaluates one Sturm count, shrinking the bracket by blockDim+1.
__device__ double block_eig_k(int n, const double* a, const double* b, int k) {
    __shared__ double s_lo, s_hi;
    double lo = a[0], hi = a[0];
    for (int i = 0; i < n; ++i) {
        double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < n - 1 ? fabs(b[i]) : 0.0);
        lo = fmin(lo, a[i] - r);
        hi = fmax(hi, a[i] + r);
    }
    double scale = fmax(fabs(lo), fabs(hi));
    lo -= 1e-14 * scale + 1e-300;
    hi += 1e-14 * scale + 1e-300;
    const int T = blockDim.x;
    // the trial points' fractions of the bracket, divided once rather than every round
    const double inv = 1.0 / (double)(T + 1), frac = (double)(threadIdx.x + 1) * inv;
    for (int round = 0; round < 12; ++round) {
        double x = lo + (hi - lo) * frac;
        int ok = sturm_count(n, a, b, x) <= k;
        int cnt = __syncthreads_count(ok);
        if (threadIdx.x == 0) {
            double nlo = cnt > 0 ? lo + (hi - lo) * ((double)cnt * inv) : lo;
            double nhi = cnt < T ? lo + (hi - lo) * ((double)(cnt + 1) * inv) : hi;
            s_lo = nlo;
            s_hi = nhi;
        }
        __syncthreads();
        lo = s_lo;
        hi = s_hi;
        __syncthreads();
        if (hi - lo <= 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300) break;
    }
    return 0.5 * (lo + hi);
}

// k-th smallest eigenvalue by multisection in ONE warp (every lane of the
// calling warp must call it; a, b may be in shared or global memory): 32 Sturm
// counts per round shrink the bracket 33-fold, so ~11 rounds reach rounding
// level from the Gershgorin interval.  The block version spends 16 warps of
// one SM on the same ~300-instruction counts per round; one warp costs a
// sixteenth of the issue slots for one more round.
__device__ double warp_eig_k(int n, const double* a, const double* b, int k) {
    const int lane = threadIdx.x & 31;
    double lo = a[0], hi = a[0];
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < n - 1 ? fabs(b[i]) : 0.0);
        lo = fmin(lo, a[i] - r);
        hi = fmax(hi, a[i] + r);
    }
    const double scale = fmax(fabs(lo), fabs(hi));
    lo -= 1e-14 * scale + 1e-300;
    hi += 1e-14 * scale + 1e-300;
    const double inv = 1.0 / 33.0, frac = (double)(lane + 1) * inv;
    for (int round = 0; round < 24; ++round) {
        const double x = lo + (hi - lo) * frac;
        const int ok = sturm_count(n, a, b, x) <= k;
        const int cnt = __popc(__ballot_sync(0xffffffffu, ok));  // trial points with at most k eigenvalues below
        const double nlo = cnt > 0 ? lo + (hi - lo) * ((double)cnt * inv) : lo;
        const double nhi = cnt < 32 ? lo + (hi - lo) * ((double)(cnt + 1) * inv) : hi;
        lo = nlo;
        hi = nhi;
        if (hi - lo <= 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300) break;
    }
    return 0.5 * (lo + hi);
}

// |last component| of the normalised eigenvector of T for eigenvalue th:
// y_n^2 = p_{n-1}(th) / p_n'(th) with the monic characteristic polynomials of
// the leading blocks (scaled recurrences; the ratio is scale-free).
__device__ double last_component(int n, const double* a, const double* b, double th) {
    if (n == 1) return 1.0;
    double pm2 = 1.0, pm1 = th - a[0];  // p0, p1
    double dm2 = 0.0, dm1 = 1.0;        // p0', p1'
    for (int k = 2; k <= n; ++k) {
        double bb = b[k - 2] * b[k - 2];
        double p = (th - a[k - 1]) * pm1 - bb * pm2;
        double dp = pm1 + (th - a[k - 1]) * dm1 - bb * dm2;
        pm2 = pm1; pm1 = p;
        dm2 = dm1; dm1 = dp;
        double mx = fmax(fmax(fabs(pm1), fabs(pm2)), fmax(fabs(dm1), fabs(dm2)));
        if (mx > 1e150) { pm1 *= 1e-150; pm2 *= 1e-150; dm1 *= 1e-150; dm2 *= 1e-150; }
        else if (mx < 1e-150 && mx > 0) { pm1 *= 1e150; pm2 *= 1e150; dm1 *= 1e150; dm2 *= 1e150; }
    }
    // after the loop: pm2 = p_{n-1}, dm1 = p_n'
    double r = (dm1 != 0.0) ? pm2 / dm1 : 1.0;
    return sqrt(fabs(r));
}

// Tridiagonal (T - shift) y = rhs with partial pivoting (dlagtf/dlagts style).
__device__ void tri_solve(int n, const double* a, const double* b, double shift, double pivmin, double* rhs,
                          double* dl, double* dd, double* du, double* du2, int* piv) {
    for (int i = 0; i < n; ++i) dd[i] = a[i] - shift;
    for (int i = 0; i < n - 1; ++i) { dl[i] = b[i]; du[i] = b[i]; }
    for (int i = 0; i < n - 1; ++i) {
        du2[i] = 0;
        if (fabs(dd[i]) >= fabs(dl[i])) {
            piv[i] = 0;
            if (fabs(dd[i]) < pivmin) dd[i] = (dd[i] < 0 ? -pivmin : pivmin);
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
            if (i < n - 2) { du2[i] = du[i + 1]; du[i + 1] = -f * du[i + 1]; }
        }
    }
    if (fabs(dd[n - 1]) < pivmin) dd[n - 1] = (dd[n - 1] < 0 ? -pivmin : pivmin);
    for (int i = 0; i < n - 1; ++i) {
        if (piv[i] == 0) rhs[i + 1] -= dl[i] * rhs[i];
        else { double t = rhs[i]; rhs[i] = rhs[i + 1]; rhs[i + 1] = t - dl[i] * rhs[i]; }
    }
    rhs[n - 1] /= dd[n - 1];
    if (n > 1) rhs[n - 2] = (rhs[n - 2] - du[n - 2] * rhs[n - 1]) / dd[n - 2];
    for (int i = n - 3; i >= 0; --i) rhs[i] = (rhs[i] - du[i] * rhs[i + 1] - du2[i] * rhs[i + 2]) / dd[i];
}

}  // namespace
}  // namespace tnb
