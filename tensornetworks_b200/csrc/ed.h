// ed.h -- full-state (exact) wave function of an open spin chain on the device:
// the FullState accelerator (TensorNetworksImp/FullStateImp.C).
#pragma once
#include <vector>

#include "tn_internal.h"

namespace tnb {

struct FullStateDev {
    Ctx* ctx = nullptr;
    int L = 0, d = 2;
    double S = 0.5;
    long long N = 0;             // d^L amplitudes, site 1 the most significant digit (StateIterator::GetIndex)
    DevBuf amp;                  // amplitudes
    DevBuf work;                 // second vector + reduction scratch
    DevBuf hl;                   // sparse local two-site matrix: per column (na d + nb) its nonzero rows
    double E = 0.0;
    int nnz_max = 0;
    double hz_site = 0.0;        // field per site (MPO convention: hz Sz once per site)
    std::vector<int> cnt_;       // nonzeros per column of the local matrix

    int init(Ctx& c, int L, double S, unsigned long long seed);
    // Hlocal of the bond term (Hamiltonian::GetLocalMatrix without the field, which is added per site)
    int set_hamiltonian(double Jxy, double Jz, double hz);
    // y = H x: sum over the L-1 bonds of the local matrix, plus the site field
    int matvec(const double* x, double* y, const int* skip);
    // Lanczos ground state (FullStateImp::FindGroundState, :190-205)
    int find_ground_state(double epsE, int krylov, int max_restarts, double* E_out, int* matvecs);
    // power iteration |psi'> = H|psi> / E (FullStateImp::PowerIterate, :155-188)
    int power_iterate(double epsE, double epsPsi, int max_iter, double* E_out, int* iters);
};

}  // namespace tnb
