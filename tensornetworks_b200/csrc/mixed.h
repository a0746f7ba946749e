// mixed.h -- split-precision (BF16 pieces on tcgen05) Heff matvec.
#pragma once
#include <vector>

#include "contract.h"
#include "tc_chain.h"

namespace tnb {

// Up to this many distinct (w2, coefficient) pairs of an MPO tensor: the scaled
// right-environment copies of the second GEMM.
constexpr int MIXED_MAX_SCALED = 48;

// Device state of one site's mixed-precision operator (valid until the
// environments or the site shape change).
struct MixedSite {
    DevBuf Fs;      // F pieces, [w1][i1][j1] (j1 contiguous)
    DevBuf Gc;      // scaled G pieces, [u][i2][j2]: c_u G_{w2_u} (j2 contiguous)
    DevBuf Xs;      // x pieces, the site layout [n][j2][j1]
    DevBuf Ps;      // stage-1 pieces, [(w1, n)][i1][j2]
    DevBuf segs;    // segment tables of the two GEMMs (ints)
    DevBuf shifts, err;
    DevBuf tune;    // input and output vectors of the split-K measurement
    ContractShape shape{};
    int nsplit = 2;
    int nU = 0;
    size_t nF = 0, nG = 0, nX = 0, nP = 0;  // piece strides (elements)
    std::vector<int> seg_host;               // last uploaded segment table
    TcChainPlan plan1, plan2;
    int splitk1 = 1, splitk2 = 1;  // chosen split-K factors of the two GEMMs
    bool ready = false;
    // the input vector's pieces are already in Xs, written by the kernels that
    // produced the vector (the Lanczos steps): heff_matvec_mixed skips its split
    bool presplit = false;
};

inline bool mixed_supported(const ContractShape& s) {
    return s.D1 % 16 == 0 && s.D2 % 16 == 0 && s.D1 >= 16 && s.D2 >= 16;
}

// Split F and the scaled copies of G into nsplit BF16 pieces (the complete-
// energy channels wshiftF / wshiftG shifted by their mean diagonals) and plan
// the two GEMMs from the host MPO tensor W (Dw1 x Dw2 blocks of d x d,
// ((w1 Dw2 + w2) d + m) d + n).
int mixed_prepare_site(Ctx& c, MixedSite& ms, const ContractShape& s, const double* W_host, const double* F,
                       const double* G, int wshiftF, int wshiftG, int nsplit);
// y = (Heff - sigma I) x with sigma the sum of the two shifts; x, y FP64 site layout.
int heff_matvec_mixed(Ctx& c, MixedSite& ms, const double* x, double* y, const int* skip);
int mixed_check_error(MixedSite& ms, cudaStream_t st);
double mixed_shift_host(MixedSite& ms, cudaStream_t st);

}  // namespace tnb
