// contract.h -- contraction building blocks shared by the sweep and the C ABI.
#pragma once
#include "tn_internal.h"

namespace tnb {

struct ContractShape {
    int d, Dw1, Dw2, D1, D2;
};

// One nonzero of the MPO in slab form: out[out] += c * in[in].
struct WTermDev {
    int in, out;
    double c;
};

std::vector<WTermDev> build_terms(const double* W, int d, int Dw1, int Dw2, bool leftToRight);

int wcombine(const double* P, double* Q, const WTermDev* terms, int nterms, long long blk, const int* skip,
             cudaStream_t st);
int copy2d(int rows, int cols, const double* src, IdxMap sr, IdxMap sc, double* dst, IdxMap dr, IdxMap dc,
           double scale, cudaStream_t st);
int fill(double* p, long long n, double v, cudaStream_t st);
// W = A + sigma I (N x N, W with leading dimension N) with sigma = 1.001 times
// the Gershgorin bound max_i sum_j |A_ij| of A's spectrum (plus a tiny floor),
// written to *sigma on the device: W is then symmetric positive definite.
int dense_shift_spd(int N, const double* A, int lda, double* W, double* sigma, cudaStream_t st);
// p[i] += v
int shift_vector(double* p, long long n, double v, cudaStream_t st);
int slab_sum(const double* in, int nslab, long long slab, double* out, const int* skip, cudaStream_t st);
int slab_sum_skip(const double* in, int nslab, long long slab, double* out, const int* skip, cudaStream_t st);
int heff_diag(const ContractShape& s, const double* Wdev, const double* F, const double* G, double* diag,
              cudaStream_t st);
int heff_matvec_f64(const ContractShape& s, const WTermDev* termsLR, int nLR, const double* F, const double* G,
                    const double* x, double* y, double* P, double* Q, const int* skip, cudaStream_t st);
int env_left_f64(const ContractShape& s, const WTermDev* termsLR, int nLR, const double* A, const double* F,
                 double* Fout, double* P, double* Q, cudaStream_t st);
int env_right_f64(const ContractShape& s, const WTermDev* termsRL, int nRL, const double* A, const double* G,
                  double* Gout, double* P, double* Q, cudaStream_t st);

// Doubles each of the two contraction scratch buffers (P, Q) must hold.
inline size_t contract_scratch_doubles(const ContractShape& s) {
    size_t Dm = (size_t)(s.D1 > s.D2 ? s.D1 : s.D2);
    size_t Dw = (size_t)(s.Dw1 > s.Dw2 ? s.Dw1 : s.Dw2);
    return (size_t)s.d * Dw * Dm * Dm;
}

// Algorithmic flops of one Heff application (dense W, as counted in the
// measurement plan): 2 d Dw D1 D2 (D1+D2) + 2 d^2 Dw^2 D1 D2, with Dw1/Dw2.
inline double heff_flops(const ContractShape& s) {
    return 2.0 * s.d * s.Dw1 * (double)s.D1 * s.D1 * s.D2 + 2.0 * s.d * s.Dw2 * (double)s.D1 * s.D2 * s.D2 +
           2.0 * s.d * s.d * (double)s.Dw1 * s.Dw2 * s.D1 * s.D2;
}

}  // namespace tnb
