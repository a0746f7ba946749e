/*
 * tn_oracle.h -- FP64 CPU oracle for the variational ground-state sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, in plain C++ on the CPU,
 * the algorithm of JanReimers/TensorNetworks for the single-site variational
 * (DMRG-style) ground-state search of open 1-D spin chains, together with the
 * linear algebra it relies on (SVD, QR, symmetric eigenproblems).  It is the
 * checker for the CUDA path: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product (libtn_cuda.so)
 * never links, loads or calls it.
 *
 * Conventions (shared with include/tn_cuda.h):
 *   - Site tensor A (d x D1 x D2): d consecutive column-major D1 x D2 blocks,
 *     element (n,i1,i2) at n*D1*D2 + i2*D1 + i1.  This is the memory order of
 *     MPSSite::itsMs[n](i1,i2) in the reference (oml matrices are
 *     column-major), with 0-based indices.
 *   - MPO tensor W (Dw1 x Dw2 x d x d): element (w1,w2,m,n) at
 *     ((w1*Dw2 + w2)*d + m)*d + n; it is <m| W(w1,w2) |n>.
 *   - Environment F (Dw x D x D): Dw consecutive column-major D x D blocks,
 *     element (w,i,j) at w*D*D + j*D + i; i is the bra index, j the ket index
 *     (the reference's Vector3 F(w,i,j), MPSSite_Contractions.C:292-400).
 *
 * Parity pins: the golden energies quoted in the reference's own tests
 * (VariationalGroundStateTests.C, ExactDiagTests.C, PyTensorNetworks/
 * test_Unittest1.py) are checked in tests/test_oracle_golden.py.
 */
#ifndef TN_ORACLE_H
#define TN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One line of an IterationSchedule (IterationSchedule.H:13-38) plus the
 * Epsilons fields the variational search reads (Epsilons.H:11-26). */
typedef struct {
    int    max_sweeps;       /* itsMaxGSSweepIterations                    */
    int    Dmax;             /* itsDmax                                    */
    int    deltaD;           /* itsDeltaD                                  */
    double eps_energy;       /* itsDelatEnergy1Epsilon                     */
    double eps_lambda;       /* itsDeltaLambdaEpsilon                      */
    double eps_eigen;        /* itsEigenSolverEpsilon                      */
} orc_sched_line;

/* Options of the oracle sweep that the reference does not expose. */
typedef struct {
    int eig_mode;      /* 0 = dense Heff + full symmetric eigensolve (the
                          reference's GetHeff -> zheevx path); 1 = matrix-free
                          restarted Lanczos (the algorithm of the CUDA path)  */
    int gauge;         /* 0 = SVD normalisation (MPSSite::SVDNormalize);
                          1 = Householder QR gauge + bond singular values of R
                          (the CUDA path's arithmetic)                        */
    int krylov;        /* Lanczos basis size per restart (eig_mode 1)        */
    int max_restarts;  /* Lanczos restarts per site (eig_mode 1)             */
    int nthreads;      /* OpenMP threads for the contractions (0 = default)  */
    int verbose;       /* 1 = print the reference's per-sweep log line        */
} orc_options;

/* Result summary of a ground-state search. */
typedef struct {
    double energy;        /* <H> after the last schedule line               */
    double energy2;       /* <H^2>                                           */
    double variance;      /* <H^2>-<H>^2 (the reference's return value)      */
    int    total_sweeps;  /* number of sweep pairs run over all lines        */
    long long matvecs;    /* Heff applications (eig_mode 1)                  */
    int    final_D;       /* GetMaxD() at the end                            */
    double last_dE;       /* GetMaxDeltaE() after the last sweep pair        */
    double last_dlambda;  /* GetMaxDeltal() after the last sweep pair        */
} orc_result;

/* ---- model ---------------------------------------------------------------- */
int  orc_mpo_dims(int L, double S, int site, int* Dw1, int* Dw2);
/* W of site `site` (1-based) of the 1-D nearest-neighbour Heisenberg/XXZ MPO.
 * form: 1 = RegularUpper, 2 = RegularLower (Enums.H MPOForm numbering). */
int  orc_mpo_site(int L, double S, int form, double Jxy, double Jz, double hz,
                  int site, double* W);
/* Two-site H12 (d^2 x d^2, row (ma,mb) = ma*d+mb, col (na,nb)); GetH(). */
int  orc_local_h12(double S, double Jxy, double Jz, double hz, double* H12);

/* ---- seeded initial state ----------------------------------------------- */
/* Fill `count` doubles with uniform(-1,1) from mt19937_64(seed) advanced by
 * `offset` draws; the generator every path of this project uses. */
void orc_uniform(unsigned long long seed, long long offset, long long count, double* out);

/* ---- contractions --------------------------------------------------------- */
int orc_env_left (int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                  const double* A, const double* F, double* Fout);
int orc_env_right(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                  const double* A, const double* G, double* Gout);
/* Literal nested-loop restatements of IterateLeft_F / IterateRightF
 * (MPSSite_Contractions.C:292-400), used to pin the staged versions. */
int orc_env_left_literal (int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                          const double* A, const double* F, double* Fout);
int orc_env_right_literal(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                          const double* A, const double* G, double* Gout);
int orc_heff_matvec(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                    const double* F, const double* G, const double* x, double* y);
/* Dense Heff (N x N column-major, N = d*D1*D2, site-tensor flattening). */
int orc_heff_dense(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                   const double* F, const double* G, double* H);
/* diag(Heff) */
int orc_heff_diag(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                  const double* F, const double* G, double* diag);

/* ---- dense linear algebra (column-major) ---------------------------------- */
/* Thin SVD A = U s Vt; U m x k, s k, Vt k x n, k = min(m,n); s descending;
 * zero singular values get orthonormal completion vectors in U/Vt. */
int orc_svd(int m, int n, const double* A, double* U, double* s, double* Vt);
/* Singular values only. */
int orc_svd_values(int m, int n, const double* A, double* s);
/* Thin Householder QR: Q m x k, R k x n, k = min(m,n). */
int orc_qr(int m, int n, const double* A, double* Q, double* R);
/* Thin LQ: L m x k, Q k x n. */
int orc_lq(int m, int n, const double* A, double* L, double* Q);
/* All eigenpairs of a symmetric N x N matrix, ascending. */
int orc_eigh(int N, const double* A, double* w, double* V);
/* Lowest k eigenpairs of the symmetric tridiagonal (alpha[0..n), beta[0..n-1)). */
int orc_tridiag_lowest(int n, const double* alpha, const double* beta, int k,
                       double* theta, double* Y);
/* Restarted Lanczos on Heff for the lowest eigenpair; x is the start vector
 * and receives the Ritz vector. Returns number of matvecs (<0 on error). */
int orc_lanczos_heff(int d, int Dw1, int Dw2, int D1, int D2, const double* W,
                     const double* F, const double* G, double* x, int krylov,
                     int max_restarts, double tol, double* theta_out, double* resid_out);

/* SVCompressorImp<T>::Compress(U,s,Vd) (SVCompressorImp.C:19-73).  In/out:
 * U (m x k, column-major), s (k), Vt (k x n, column-major with leading
 * dimension k on input); returns the new k in *k_out and the discarded
 * sum of s^2 as the function value.  Outputs are compacted in place. */
double orc_compress(int Dmax, double eps, int m, int n, int k, double* U,
                    double* s, double* Vt, int* k_out);

/* ---- full searches ------------------------------------------------------- */
int orc_find_ground_state(int L, double S, int form, double Jxy, double Jz, double hz,
                          int Dstart, unsigned long long seed,
                          const orc_sched_line* lines, int nlines,
                          const orc_options* opt, orc_result* res,
                          double* site_energies /* L, may be NULL */);
/* Timing sample of the sweep's site update on a given MPS (the CPU baseline):
 * sites are given as L tensors (dims D1s/D2s, concatenated in site order, shared
 * layout).  Sites 1..first-1 are left-normalised (QR), environments built, and
 * then nsites consecutive DLeft site updates (Lanczos + QR gauge + left
 * environment, the same work as one site of the CUDA sweep) are timed. */
int orc_sweep_sample(int L, double S, int form, double Jxy, double Jz, double hz,
                     const int* D1s, const int* D2s, const double* sites, int first, int nsites,
                     int krylov, int max_restarts, double tol, int nthreads,
                     double* seconds, long long* matvecs);
/* Exact diagonalisation (Lanczos on the d^L space). field_mode 0: the MPO's
 * +hz*Sz once per site; 1: the reference FullState's GetH convention
 * (hz*(Sz_a+Sz_b) on every bond). */
int orc_ed_ground(int L, double S, double Jxy, double Jz, double hz, int field_mode,
                  double tol, double* E);

/* iTEBD on the infinite chain, two-site unit cell, Vidal gauge, second-order
 * Trotter gates (iTEBDStateImp_iTime.C:25-135).  dts/nsteps give the
 * imaginary-time schedule; returns the energy per bond. */
int orc_itebd(double S, double Jxy, double Jz, double hz, int D,
              const double* dts, const int* nsteps, int nlines,
              unsigned long long seed, double eps_sv, double* E_bond);

#ifdef __cplusplus
}
#endif
#endif
