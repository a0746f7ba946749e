// mixed.h -- split-precision (BF16x3, tcgen05) Heff matvec.
#pragma once
#include "contract.h"
#include "tc_gemm.h"

namespace tnb {

// Device state of one site's mixed-precision operator (valid until the
// environments or the site shape change).
struct MixedSite {
    DevBuf Fs, Gs, Xs, P32, Qs, shifts, err;
    ContractShape shape{};
    const WTermDev* termsLR = nullptr;
    int nLR = 0;
    int nsplit = 2;
    size_t nX = 0, nQ = 0;  // piece strides (elements)
    TcGemmPlan plan1, plan3;
    bool ready = false;
};

inline bool mixed_supported(const ContractShape& s) {
    return s.D1 % 16 == 0 && s.D2 % 16 == 0 && s.D1 >= 16 && s.D2 >= 16;
}

// Split F, G into nsplit BF16 pieces (shifting the complete-energy channels wshiftF / wshiftG) and plan the GEMMs.
int mixed_prepare_site(Ctx& c, MixedSite& ms, const ContractShape& s, const WTermDev* termsLR, int nLR,
                       const double* F, const double* G, int wshiftF, int wshiftG, int nsplit);
// y = (Heff - sigma I) x with sigma the sum of the two shifts; x, y FP64 site layout.
int heff_matvec_mixed(Ctx& c, MixedSite& ms, const double* x, double* y, const int* skip);
int mixed_check_error(MixedSite& ms, cudaStream_t st);
double mixed_shift_host(MixedSite& ms, cudaStream_t st);

}  // namespace tnb
