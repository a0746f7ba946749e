// A C++ client of libtn_cuda through include/tn_cuda.h only, as a reference-side
// adapter would call it: the Heisenberg chain of PyTensorNetworks/test_Unittest1.py
// (L = 10, S = 1/2, D grown from 2 to 8, epsilons 1e-12, 100 sweeps at most)
// through Factory -> Hamiltonian -> MPS -> FindVariationalGroundState, then a
// thin QR through the QRSolver entry point.  Exits 0 when the energy per bond
// matches the reference's golden value (-0.473113399629092,
// test_Unittest1.py:22) to 1e-11 and Q R reproduces the matrix.
#include <cmath>
#include <cstdio>
#include <vector>

#include <cuda_runtime.h>

#include "tn_cuda.h"

#define CHECK(x)                                                                                  \
    do {                                                                                          \
        int st_ = (x);                                                                            \
        if (st_ != TN_OK) {                                                                       \
            std::fprintf(stderr, "%s failed: %s (%s)\n", #x, tn_status_string(st_), tn_last_error()); \
            return 2;                                                                             \
        }                                                                                         \
    } while (0)

int main() {
    tn_ctx ctx = nullptr;
    CHECK(tn_ctx_create(0, &ctx));
    const int L = 10, Dstart = 2, Dfinal = 8;
    tn_hamiltonian H = nullptr;
    CHECK(tn_hamiltonian_create_heisenberg(ctx, L, 0.5, TN_FORM_REGULAR_LOWER, 1.0, 1.0, 0.0, &H));
    tn_mps psi = nullptr;
    CHECK(tn_mps_create(H, Dstart, 1e-12, 1e-12, &psi));
    CHECK(tn_mps_initialize_random(psi, 1234));
    tn_sched_line line{100, Dfinal, 1, 1e-12, 1e-12, 1e-12};
    tn_solver_options opt{};
    opt.precision = TN_PREC_FP64;
    opt.eigensolver = TN_EIG_LANCZOS;
    opt.krylov = 20;
    opt.max_restarts = 10;
    tn_sweep_stats stats{};
    double variance = 0.0, E = 0.0;
    CHECK(tn_mps_find_variational_ground_state(psi, H, &line, 1, &opt, &stats, &variance));
    CHECK(tn_mps_get_expectation(psi, H, &E));
    const double e = E / (L - 1), golden = -0.473113399629092;
    std::printf("E/(L-1) = %.15f (golden %.15f), variance %.3e, sweeps %d, matvecs %lld\n", e, golden, variance,
                stats.total_sweeps, stats.matvecs);
    // QRSolver::SolveThinQR on a device matrix
    const int m = 64, n = 32;
    std::vector<double> A(m * n);
    for (int i = 0; i < m * n; ++i) A[i] = std::sin(0.37 * i + 1.0);
    double *dA = nullptr, *dQ = nullptr, *dR = nullptr;
    if (cudaMalloc(&dA, sizeof(double) * m * n) != cudaSuccess || cudaMalloc(&dQ, sizeof(double) * m * n) != cudaSuccess ||
        cudaMalloc(&dR, sizeof(double) * n * n) != cudaSuccess)
        return 2;
    cudaMemcpy(dA, A.data(), sizeof(double) * m * n, cudaMemcpyHostToDevice);
    CHECK(tn_qr(ctx, m, n, dA, m, dQ, m, dR, n));
    std::vector<double> Q(m * n), R(n * n);
    cudaMemcpy(Q.data(), dQ, sizeof(double) * m * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(R.data(), dR, sizeof(double) * n * n, cudaMemcpyDeviceToHost);
    double err = 0.0;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k <= j; ++k) s += Q[k * m + i] * R[j * n + k];
            err = std::fmax(err, std::fabs(s - A[j * m + i]));
        }
    std::printf("QR reconstruction error %.3e\n", err);
    cudaFree(dA);
    cudaFree(dQ);
    cudaFree(dR);
    CHECK(tn_mps_destroy(psi));
    CHECK(tn_hamiltonian_destroy(H));
    CHECK(tn_ctx_destroy(ctx));
    return (std::fabs(e - golden) <= 1e-11 && err < 1e-12) ? 0 : 1;
}
