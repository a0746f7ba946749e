// itebd.h -- infinite-chain imaginary-time evolution (iTEBD, Vidal form,
// two-site unit cell) on the device.
#pragma once
#include <vector>

#include "tn_internal.h"

namespace tnb {

struct ITebdState {
    Ctx* ctx = nullptr;
    int d = 2;
    double S = 0.5, Jxy = 1, Jz = 1, hz = 0;
    // site s: Gamma_s (d, Dl, Dr), Gamma_s[n](i, j) at n*Dl*Dr + j*Dl + i.
    // bond 0 joins site 0 -> site 1, bond 1 joins site 1 -> site 0 (next cell);
    // site 0 has Dl = dim(bond 1), Dr = dim(bond 0); site 1 the reverse.
    DevBuf G[2];
    DevBuf lam[2];
    std::vector<double> lam_h[2];
    DevBuf gate;                 // exp(-dt h), d^2 x d^2 (symmetric)
    DevBuf X, Y, TH, M, U, Vt, V, s, work;
    DevBuf og;                   // OrthogonalizeI workspace
    std::vector<double> h12;     // two-site Hamiltonian, rows (ma d + mb), columns (na d + nb)
    long long gates_applied = 0;

    int dim(int bond) const { return (int)lam_h[bond].size(); }
    int init(Ctx& c, double S, double Jxy, double Jz, double hz, int D, unsigned long long seed);
    // exp(-dt h12) on the device
    int set_gate(double dt);
    // one gate on `bond` with the SVCompressor rule (Dmax, eps)
    int apply_gate(int bond, int Dmax, double eps);
    // second-order Trotter step: gates dt/2, dt, dt/2 on bonds 0, 1, 0; eps-only
    // compression (1e-7) on the first, Dmax on the last two
    int step2(double dt, int Dmax);
    // SVD of the (d Dl) x (d Dl) matrix in M, SVCompressor rule (Dmax, eps),
    // new bond values on `bond`, Gammas unpacked with the other bond's values
    int svd_unpack(int bond, int Dl, int Dmax, double eps);
    // OrthogonalizeI at centre 1 (the iterative re-orthogonalisation); the
    // largest change of the bond values in the last iteration in *delta, the
    // iterations run in *iters, *bailed when the norm matrices were singular
    int orthogonalize_i(int Dmax, double eps, int max_iter, double* delta, int* iters, bool* bailed);
    // IncreaseBondDimensions: Gammas zero-padded to D x D, bond values padded
    // with min/10 and renormalised
    int grow(int D);
    // energy per bond from the unit-cell transfer-matrix fixed points
    int energy(double* E, int max_iters, double tol);
};

}  // namespace tnb
