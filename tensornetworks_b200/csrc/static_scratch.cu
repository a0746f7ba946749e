// static_scratch.cu -- tn_heff_matvec_static: the FP64 Heff matvec with its
// scratch (MPO term list + the two stage buffers) in a fixed device array, so
// the call allocates no memory at all.
//
// The scratch is one file-scope __device__ array per device.  The first call
// through a context on a device makes that device current, looks up its
// copy's address (cudaGetSymbolAddress) and caches it per device ordinal;
// later calls only enqueue copies and kernels on the context's stream.  The
// kernel chain is the one of tn_heff_matvec (stage-1 GEMM, sparse MPO
// combination, split stage-3 GEMM, deterministic slab sum): it writes every
// scratch element it reads, so nothing has to start at zero.
#include <algorithm>
#include <array>
#include <cstring>
#include <mutex>

#include "contract.h"

namespace tnb {
namespace {

constexpr size_t STATIC_SCRATCH_DOUBLES = (size_t)TN_HEFF_STATIC_MAX_DOUBLES;
constexpr int STATIC_MAX_TERMS = 4096;  // MPO terms (d^2 Dw1 Dw2 + d Dw at most)

static __device__ __align__(256) double g_heff_scratch[STATIC_SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_scratch_ptr[MAX_DEVICES] = {};

// Address of this device's copy of the array.  The caller has made `dev`
// current: the symbol address is per device, and a kernel given another
// device's copy would run on the wrong memory.
int scratch_for_device(int dev, double** out) {
    if (dev < 0 || dev >= MAX_DEVICES) {
        set_error("tn_heff_matvec_static: device ordinal %d out of range", dev);
        return TN_BAD_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_heff_scratch);
        if (e != cudaSuccess || !p) {
            set_error("tn_heff_matvec_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return TN_CUDA_ERROR;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return TN_OK;
}

}  // namespace
}  // namespace tnb

using namespace tnb;

extern "C" int tn_heff_matvec_static(tn_ctx c, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host,
                                     const double* F, const double* G, const double* x, double* y) {
    if (!c || !W_host || !F || !G || !x || !y) return TN_BAD_ARG;
    if (d < 1 || Dw1 < 1 || Dw2 < 1 || D1 < 1 || D2 < 1) return TN_BAD_SHAPE;
    Ctx& cx = c->c;
    // Bound every dimension before any product is formed (no size_t wrap-around
    // can then slip past the capacity check) and before the term loop reads W.
    {
        const double Dm = (double)std::max(D1, D2), Dw = (double)std::max(Dw1, Dw2);
        const double stage = (double)d * Dw * Dm * Dm;
        const double nterm_max = (double)d * d * Dw1 * Dw2 + (double)d * Dw2;
        if (stage * 2.0 + nterm_max * 2.0 > (double)STATIC_SCRATCH_DOUBLES) {
            set_error("tn_heff_matvec_static: shape d=%d Dw=%dx%d D=%dx%d needs about %.0f doubles of scratch, the "
                      "static scratch holds %zu",
                      d, Dw1, Dw2, D1, D2, stage * 2.0, STATIC_SCRATCH_DOUBLES);
            return TN_BAD_SHAPE;
        }
    }
    // MPO term list (left-to-right slab form) in a fixed host array
    std::array<WTermDev, STATIC_MAX_TERMS> terms;
    int nt = 0;
    for (int m = 0; m < d; ++m)
        for (int wo = 0; wo < Dw2; ++wo) {
            const int o = m * Dw2 + wo;
            bool any = false;
            for (int wi = 0; wi < Dw1; ++wi)
                for (int n = 0; n < d; ++n) {
                    const double v = W_host[(((size_t)wi * Dw2 + wo) * d + m) * d + n];
                    if (v == 0.0) continue;
                    if (nt >= STATIC_MAX_TERMS) {
                        set_error("tn_heff_matvec_static: more than %d MPO terms", STATIC_MAX_TERMS);
                        return TN_BAD_SHAPE;
                    }
                    terms[nt++] = WTermDev{wi * d + n, o, v};
                    any = true;
                }
            if (!any) {
                if (nt >= STATIC_MAX_TERMS) {
                    set_error("tn_heff_matvec_static: more than %d MPO terms", STATIC_MAX_TERMS);
                    return TN_BAD_SHAPE;
                }
                terms[nt++] = WTermDev{0, o, 0.0};
            }
        }
    ContractShape s{d, Dw1, Dw2, D1, D2};
    const size_t term_doubles = ((sizeof(WTermDev) * (size_t)nt + 255) / 256) * 256 / sizeof(double);
    const size_t stage = ((contract_scratch_doubles(s) + 31) / 32) * 32;
    const size_t need = term_doubles + 2 * stage;
    if (need > STATIC_SCRATCH_DOUBLES) {
        set_error("tn_heff_matvec_static: shape d=%d Dw=%dx%d D=%dx%d needs %zu doubles of scratch, the static "
                  "scratch holds %zu",
                  d, Dw1, Dw2, D1, D2, need, STATIC_SCRATCH_DOUBLES);
        return TN_BAD_SHAPE;
    }
    TN_ON_DEVICE(cx.device);
    double* base = nullptr;
    TN_CHECK(scratch_for_device(cx.device, &base));
    WTermDev* tdev = reinterpret_cast<WTermDev*>(base);
    double* P = base + term_doubles;
    double* Q = P + stage;
    // pageable source: the copy is staged before cudaMemcpyAsync returns
    TN_CUDA_CHECK(cudaMemcpyAsync(tdev, terms.data(), sizeof(WTermDev) * (size_t)nt, cudaMemcpyHostToDevice,
                                  cx.stream));
    TN_CHECK(heff_matvec_f64(s, tdev, nt, F, G, x, y, P, Q, nullptr, cx.stream));
    return TN_OK;
}
