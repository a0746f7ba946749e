/*
 * tn_cuda.h -- C ABI of the B200 (sm_100a) variational ground-state sweep.
 *
 * This is the drop-in boundary for the LAPACK/ARPACK/PRIMME solver path of
 * JanReimers/TensorNetworks.  Every entry point names the reference interface
 * it replaces (file:line, paths relative to the reference project root).
 * Signatures use plain C types only: opaque handles, int status codes, raw
 * pointers and sizes.  Pointers documented as "device" are CUDA device
 * pointers; "host" pointers are ordinary CPU memory.
 *
 * Layout conventions (0-based indices, column-major matrices):
 *   site tensor A (d x D1 x D2): d consecutive column-major D1 x D2 blocks,
 *       element (n,i1,i2) at n*D1*D2 + i2*D1 + i1  (MPSSite::itsMs[n](i1,i2),
 *       TensorNetworksImp/MPS/MPSSite.H:175-177);
 *   MPO tensor W (Dw1 x Dw2 x d x d): element (w1,w2,m,n) at
 *       ((w1*Dw2 + w2)*d + m)*d + n, the value <m|W(w1,w2)|n>;
 *   environment F (Dw x D x D): Dw consecutive column-major D x D blocks,
 *       element (w,i,j) at w*D*D + j*D + i (bra index i, ket index j; the
 *       Vector3 caches of MPSSite_Contractions.C:292-400).
 *
 * Threading: a tn_ctx owns one CUDA stream and its scratch memory; calls on
 * one context must not overlap.  Distinct contexts are independent.
 */
#ifndef TN_CUDA_H
#define TN_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum {
    TN_OK             = 0,
    TN_NOT_CONVERGED  = 1,  /* iteration cap reached (result still usable)  */
    TN_BAD_SHAPE      = 2,  /* inconsistent dimensions                       */
    TN_NAN_DETECTED   = 3,  /* non-finite value in an input or result        */
    TN_CUDA_ERROR     = 4,  /* a CUDA runtime call failed                    */
    TN_BAD_ARG        = 5,  /* null handle/pointer or out-of-range argument  */
    TN_NO_DEVICE      = 6,  /* no sm_100 device visible                      */
    TN_OUT_OF_MEMORY  = 7
};

/* MPO forms, numbered as TensorNetworks/Enums.H:17 (enum MPOForm). */
enum { TN_FORM_REGULAR_UPPER = 1, TN_FORM_REGULAR_LOWER = 2 };
/* Directions, as TensorNetworks/Enums.H:10 (enum Direction). */
enum { TN_DLEFT = 0, TN_DRIGHT = 1 };
/* Arithmetic of the Heff / environment contractions. */
enum {
    TN_PREC_FP64     = 0,  /* FP64 throughout (the plain GPU sweep)          */
    TN_PREC_MIXED    = 1,  /* BF16x3 tcgen05 contractions (2 BF16 pieces per
                              operand, 3 products, FP32 accumulate); FP64
                              Lanczos coefficients, QR, SVD and energies     */
    TN_PREC_MIXED_HI = 2   /* BF16x6 (3 pieces, 6 products: ~FP32 operand
                              accuracy) on the same tcgen05 kernels         */
};
/* Eigensolvers for the site problem. */
enum {
    TN_EIG_LANCZOS  = 0,  /* restarted Lanczos, full reorthogonalisation    */
    TN_EIG_DAVIDSON = 1   /* Davidson with diagonal or learned preconditioner */
};

typedef struct tn_ctx_s*         tn_ctx;
typedef struct tn_hamiltonian_s* tn_hamiltonian;
typedef struct tn_mps_s*         tn_mps;

/* One IterationScheduleLine (TensorNetworks/IterationSchedule.H:13-38) with
 * the Epsilons fields the variational search reads (Epsilons.H:11-26). */
typedef struct {
    int    max_sweeps;   /* itsMaxGSSweepIterations (pairs of half-sweeps) */
    int    Dmax;         /* itsDmax                                        */
    int    deltaD;       /* itsDeltaD                                      */
    double eps_energy;   /* itsDelatEnergy1Epsilon                         */
    double eps_lambda;   /* itsDeltaLambdaEpsilon                          */
    double eps_eigen;    /* itsEigenSolverEpsilon                          */
} tn_sched_line;

/* Solver options (no counterpart in the reference, which hard-wires
 * LapackEigenSolver at MPSSite.C:29 and LapackSVDSolver at
 * MPSSite_Normalization.C:49). */
typedef struct {
    int precision;       /* TN_PREC_*                                      */
    int eigensolver;     /* TN_EIG_*                                       */
    int krylov;          /* Krylov/Davidson basis size per restart (20)    */
    int max_restarts;    /* restarts per site (10)                         */
    int use_learned;     /* 1: learned preconditioner (Davidson only)      */
    int verbose;         /* 1: print the reference's per-sweep log line     */
    double mixed_tol;    /* residual target of the split-precision Krylov
                            phase relative to the norm of its tridiagonal
                            matrix (0: 2e-6 for MIXED, 1e-9 for MIXED_HI);
                            the phase also stops when its residual no
                            longer falls (the operator's noise floor)       */
    double refine_tol;   /* FP64 residual above which an FP64 Lanczos
                            continuation follows the split-precision solve
                            (0: never; the FP64 Rayleigh quotient always
                            supplies the site energy)                       */
    double fp64_tol_rel; /* FP64 Lanczos: residual target relative to the
                            norm of its tridiagonal matrix, with the same
                            stop on a stalled residual as the split-precision
                            phase (0: the absolute eps_eigen only).  Lets the
                            FP64 sweep stop by the mixed path's rule.       */
    int phase_timing;    /* 1: CUDA events on the library stream around each
                            site's eigen-solve, gauge move and environment
                            update; their device times go to the refine_ms,
                            gauge_ms and env_ms statistics                  */
} tn_solver_options;

/* Per-run statistics, device-timed with CUDA events. */
typedef struct {
    double energy;          /* <H> after the last line (GetExpectation)    */
    double energy2;         /* <H^2>                                        */
    double variance;        /* <H^2>-<H>^2 (the reference's return value)  */
    int    total_sweeps;    /* sweep pairs over all lines                   */
    int    final_D;         /* GetMaxD()                                    */
    long long matvecs;      /* Heff applications                            */
    long long matvecs_fp64; /* of which FP64 (refinement steps, mixed path) */
    double heff_flop;       /* algorithmic flops of all Heff applications    */
    double heff_ms;         /* device time inside the Heff contractions      */
    double sweep_ms;        /* device time of all sweeps                     */
    double last_dE;         /* GetMaxDeltaE() after the last sweep pair      */
    double last_dlambda;    /* GetMaxDeltal() after the last sweep pair      */
    int    not_converged;   /* site solves that hit the iteration cap        */
    int    fallbacks;       /* learned-correction stalls (diagonal Davidson
                               took over) plus FP64 refinements of the mixed
                               path                                          */
    long long learned_steps; /* Davidson corrections the learned MLP made    */
    double refine_ms;       /* device time of the site eigen-solves, the     */
    double gauge_ms;        /* gauge moves (QR/LQ and the neighbour product) */
    double env_ms;          /* and the environment updates (phase_timing=1)  */
} tn_sweep_stats;

/* ---- context ------------------------------------------------------------- */
const char* tn_status_string(int status);
/* Last error message recorded on this thread (for diagnostics). */
const char* tn_last_error(void);
int tn_ctx_create(int device, tn_ctx* out);
int tn_ctx_destroy(tn_ctx ctx);
/* Use an external cudaStream_t (passed as void*); NULL restores the own stream. */
int tn_ctx_set_stream(tn_ctx ctx, void* stream);
int tn_ctx_synchronize(tn_ctx ctx);

/* ---- Factory / Hamiltonian / MPO ------------------------------------------
 * Factory::Make1D_NN_HeisenbergHamiltonian (TensorNetworks/Factory.H:16,
 * TensorNetworksImp/FactoryImp.C:21-26) -> HamiltonianImp (MPO of L sites,
 * Hamiltonian_1D_NN_Heisenberg.C:35-79, boundaries SiteOperatorImp.C:109-134). */
int tn_hamiltonian_create_heisenberg(tn_ctx ctx, int L, double S, int form, double Jxy,
                                     double Jz, double hz, tn_hamiltonian* out);
int tn_hamiltonian_destroy(tn_hamiltonian H);
/* SiteOperator::GetDws / Getd (TensorNetworks/SiteOperator.H:44-46). */
int tn_hamiltonian_site_dims(tn_hamiltonian H, int site, int* Dw1, int* Dw2, int* d);
/* Bond dimensions of site `site` of the H^2 MPO that <H^2> contracts
 * (Hamiltonian::CreateH2Operator, Hamiltonian.C:8-16: the product H*H with its
 * exactly dependent bond directions removed by SVD sweeps). */
int tn_hamiltonian_h2_dims(tn_hamiltonian H, int site, int* Dw1, int* Dw2);
/* SiteOperator::GetW (SiteOperator.H:52): copies W of a site into host memory. */
int tn_hamiltonian_get_w(tn_hamiltonian H, int site, double* W_host);

/* ---- MPS -------------------------------------------------------------------
 * Hamiltonian::CreateMPS (TensorNetworks/Hamiltonian.H:26, HamiltonianImp.C:41-44). */
int tn_mps_create(tn_hamiltonian H, int D, double normEps, double epsSV, tn_mps* out);
int tn_mps_destroy(tn_mps psi);
/* MPS::InitializeWith(Random) (MPS.H:17, MPSSite.C:119-127): uniform(-1,1)
 * from mt19937_64(seed), sites 1..L in order, each scaled 1/sqrt(d*D1*D2). */
int tn_mps_initialize_random(tn_mps psi, uint64_t seed);
/* Site tensor access (host buffers, site 1-based). */
int tn_mps_get_site_dims(tn_mps psi, int site, int* D1, int* D2);
int tn_mps_get_site(tn_mps psi, int site, double* A_host);
int tn_mps_set_site(tn_mps psi, int site, int D1, int D2, const double* A_host);
/* Bond singular values (Bond::GetSVs, Bond.H), normalised; bond b in 1..L-1. */
int tn_mps_get_bond(tn_mps psi, int bond, int* D, double* s_host);
/* MPS::Normalize (MPS.C:8) / MPS::NormalizeQR (MPSImp_Normalization.C:39-63). */
int tn_mps_normalize(tn_mps psi, int direction);
/* MPS::GetMaxD (MPS.H:70). */
int tn_mps_get_max_d(tn_mps psi, int* D);
/* MPS::GetExpectation(MPO*) (MPSImp_ExpectationsAndDMs.C:33-45), FP64 on device. */
int tn_mps_get_expectation(tn_mps psi, tn_hamiltonian H, double* E);
/* <H^2> with the product MPO of Hamiltonian::CreateH2Operator (Hamiltonian.C:8-16). */
int tn_mps_get_expectation_h2(tn_mps psi, tn_hamiltonian H, double* E2);
/* MPS::FindVariationalGroundState(H, IterationSchedule) (MPS.H:36,
 * MPSImp_Variational.C:16-62).  Returns <H^2>-<H>^2 in *variance. */
int tn_mps_find_variational_ground_state(tn_mps psi, tn_hamiltonian H,
                                         const tn_sched_line* lines, int nlines,
                                         const tn_solver_options* opt,
                                         tn_sweep_stats* stats, double* variance);
/* nsweeps pairs of MPSImp::Sweep(DLeft) + Sweep(DRight) (MPSImp_Variational.C:43-47,
 * 64-76) at the current bond dimension, without the <H>, <H^2> evaluation that
 * closes each D step of FindVariationalGroundState.  The MPS must be right-
 * normalised with its right environments loaded (true after
 * tn_mps_find_variational_ground_state or tn_mps_prepare_sweeps). */
int tn_mps_sweep(tn_mps psi, tn_hamiltonian H, int nsweeps, double eps_eigen,
                 const tn_solver_options* opt, tn_sweep_stats* stats);
/* MPS::Normalize(DRight) followed by MPSImp::LoadHeffCaches (MPSImp_Variational.C:18-19). */
int tn_mps_prepare_sweeps(tn_mps psi, tn_hamiltonian H);
/* One line of an imaginary-time schedule: the fields of IterationScheduleLine
 * (IterationSchedule.H:27-35) and Epsilons (Epsilons.H:11-26) that
 * MPSImp::FindiTimeGroundState reads. */
typedef struct {
    int    max_iter;         /* itsMaxGSSweepIterations                        */
    int    Dmax;             /* itsDmax (the MPS compressor's Dmax)             */
    int    max_opt_iter;     /* itsMaxOptimizeIterations                        */
    int    order;            /* itsTrotterOrder: 1 (first) or 2 (second)        */
    double dt;               /* itsdt                                           */
    double eps_energy;       /* itsDelatEnergy1Epsilon                          */
    double eps_lambda;       /* itsDeltaLambdaEpsilon                           */
    double eps_norm;         /* itsDelatNormEpsilon (Optimize's stop)           */
    double eps_mps_compress; /* itsMPSCompressEpsilon (0: Dmax only)            */
} tn_itime_line;
/* MPS::FindiTimeGroundState(H, schedule) (MPSImp_iTime.C:18-88): per line, the
 * Trotter operator of exp(-dt H) (first or second order, the exact product of
 * the gate layers), applied, SVD-compressed both ways and variationally
 * optimised towards the uncompressed product, until |dE| and the bond-value
 * change fall below the line's epsilons or the energy rises.  *variance:
 * <H^2> - <H>^2 at the end; iters_out[line] (may be null): iterations run. */
int tn_mps_find_itime_ground_state(tn_mps psi, tn_hamiltonian h, const tn_itime_line* lines, int nlines,
                                   double* variance, int* iters_out);
/* MPS::CalculateOneSiteDMs (MPS.H:63, MPSImp_ExpectationsAndDMs.C:59-71):
 * L blocks of d x d, rho_host[(ia-1) d^2 + m d + n].  Right-normalises the
 * state first and leaves it left-normalised, as the reference does. */
int tn_mps_one_site_dms(tn_mps psi, double* rho_host);
/* MPS::CalculateTwoSiteDMs (MPS.H:64, MPSImp_ExpectationsAndDMs.C:73-117): for
 * the L(L-1)/2 pairs ia < ib in order (ia outer), d^4 values each,
 * rho[((m d + m2) d + n) d + n2] with (m, n) on site ia and (m2, n2) on ib. */
int tn_mps_two_site_dms(tn_mps psi, double* rho_host);
/* Per-site Ritz energies of the last solves (MPSSite::itsEmin), L values. */
int tn_mps_get_site_energies(tn_mps psi, double* E_host);

/* Number of kernels this library has launched in this process (diagnostics;
 * no counterpart in the reference). */
unsigned long long tn_launch_count(void);

/* ---- solver interfaces (device pointers) --------------------------------
 * SparseEigenSolverClient::DoMatVecContraction (NumericalMethods/
 * SparseEigenSolver.H:17-24) for the site problem: y = Heff x, the
 * matrix-free form of MPSSite::GetHeff (MPSSite_Contractions.C:155-193). */
int tn_heff_matvec(tn_ctx ctx, int precision, int d, int Dw1, int Dw2, int D1, int D2,
                   const double* W_host, const double* F, const double* G,
                   const double* x, double* y);
/* tn_heff_matvec with precision TN_PREC_FP64, allocating no memory: the MPO
 * term list and both contraction stage buffers live in a fixed device array
 * of TN_HEFF_STATIC_MAX_DOUBLES doubles (8 MiB) per device.  No counterpart in
 * the reference.  Limits: 2*d*max(Dw1,Dw2)*max(D1,D2)^2 doubles plus the term
 * list must fit (d=2, Dw=5: D1, D2 <= 224; D = 256 is rejected with
 * TN_BAD_SHAPE and a message in tn_last_error).  The first call on a device
 * looks up the array's address (device current) and should precede any
 * stream capture.  All calls on one device share the array: calls that may
 * overlap (other threads, streams or contexts on the same device) race and
 * must be serialised by the caller.  Nothing in the array needs to start at
 * zero.  The call enqueues on the context stream and returns without
 * synchronising. */
#define TN_HEFF_STATIC_MAX_DOUBLES (1 << 20)
int tn_heff_matvec_static(tn_ctx ctx, int d, int Dw1, int Dw2, int D1, int D2,
                          const double* W_host, const double* F, const double* G,
                          const double* x, double* y);
/* Heff operator object: the device-side SparseEigenSolverClient
 * (SparseEigenSolver.H:17-24) of one site.  Creation uploads W and, for the
 * split-precision modes, splits F and G into BF16 pieces once; apply is then
 * the client's DoMatVecContraction(N, x, y) on device vectors.  F and G must
 * stay unchanged while the handle is in use. */
typedef struct tn_heff_s* tn_heff;
int tn_heff_create(tn_ctx ctx, int precision, int d, int Dw1, int Dw2, int D1, int D2,
                   const double* W_host, const double* F, const double* G, tn_heff* out);
/* GetSize(): d*D1*D2. */
long long tn_heff_size(tn_heff op);
int tn_heff_apply(tn_heff op, const double* x, double* y);
int tn_heff_destroy(tn_heff op);
/* diag(Heff) (feature of the Davidson preconditioner). */
int tn_heff_diag(tn_ctx ctx, int d, int Dw1, int Dw2, int D1, int D2, const double* W_host,
                 const double* F, const double* G, double* diag);
/* MPSSite::IterateLeft_F / IterateRightF (MPSSite_Contractions.C:292-400). */
int tn_env_left(tn_ctx ctx, int precision, int d, int Dw1, int Dw2, int D1, int D2,
                const double* W_host, const double* A, const double* F, double* Fout);
int tn_env_right(tn_ctx ctx, int precision, int d, int Dw1, int Dw2, int D1, int D2,
                 const double* W_host, const double* A, const double* G, double* Gout);
/* Lowest eigenpair of Heff: replaces LapackEigenSolver<T>::Solve(Heff,eps,2)
 * (NumericalMethods/LapackEigenSolver.C:62-109) as called by MPSSite::Refine
 * (MPSSite_Variational.C:18-33).  x: start vector in, Ritz vector out. */
int tn_eigensolve_heff(tn_ctx ctx, const tn_solver_options* opt, int d, int Dw1, int Dw2,
                       int D1, int D2, const double* W_host, const double* F,
                       const double* G, double* x, double tol, double* theta,
                       double* residual, int* matvecs);
/* Dense symmetric eigensolver, lowest k pairs in ascending order:
 * EigenSolver<T>::Solve (NumericalMethods/EigenSolver.H:31), the contract of
 * LapackEigenSolver::Solve (LapackEigenSolver.C:62-109, zheevx RANGE='I',
 * IL=1, IU=k).  A: N x N (lda) device, U: N x k (ldu) device, w_host: k
 * eigenvalues.  On the device: A is shifted above its Gershgorin bound to a
 * positive-definite matrix whose one-sided Jacobi SVD is its eigen-
 * decomposition (absolute eigenvalue accuracy ~ eps |A|, as abstol gives
 * LAPACK); tol >= 0 is the reference's abstol and is accepted, not needed.
 * N is limited by the single-CTA Jacobi kernel (N <= ~17000). */
int tn_eigensolve_dense(tn_ctx ctx, int N, const double* A, int lda, int k, double tol,
                        double* w_host, double* U, int ldu);
/* SVDSolver<T>::SolveAll (NumericalMethods/SVDSolver.H:22, LapackSVDSolver.C:42-90),
 * one-sided Jacobi: A (m x n) = U s Vt, k = min(m,n); U m x k, s k (device),
 * Vt k x n.  Zero singular values get orthonormal completion vectors. */
int tn_svd(tn_ctx ctx, int m, int n, const double* A, int lda, double* U, int ldu,
           double* s, double* Vt, int ldvt);
/* SVDSolver<T>::Solve(A, eps, k) (SVDSolver.H:21, LapackSVDSolver.C:42-90):
 * the k largest singular triplets, U m x k (ldu), s k (device), Vt k x n
 * (ldvt); eps < 1 as the reference asserts. */
int tn_svd_solve(tn_ctx ctx, int m, int n, const double* A, int lda, double eps, int k, double* U, int ldu,
                 double* s, double* Vt, int ldvt);
/* Singular values only (descending). */
int tn_svd_values(tn_ctx ctx, int m, int n, const double* A, int lda, double* s);
/* QRSolver<T>::SolveThinQR / SolveThinLQ (NumericalMethods/QRSolver.H:18-21,
 * LapackQRSolver.C:116-160,277-320), Householder: Q m x k, R k x n;
 * L m x k, Q k x n. */
int tn_qr(tn_ctx ctx, int m, int n, const double* A, int lda, double* Q, int ldq,
          double* R, int ldr);
int tn_lq(tn_ctx ctx, int m, int n, const double* A, int lda, double* L, int ldl,
          double* Q, int ldq);
/* QRSolver<T>::SolveThinRQ / SolveThinQL (QRSolver.H:18-21,
 * LapackQRSolver.C:163-274): A = R Q with R m x k (upper for m <= n), Q k x n
 * orthonormal rows; A = Q L with Q m x k orthonormal columns, L k x n (lower
 * for n <= m).  Householder QR of the index-reversed matrix. */
int tn_rq(tn_ctx ctx, int m, int n, const double* A, int lda, double* R, int ldr, double* Q, int ldq);
int tn_ql(tn_ctx ctx, int m, int n, const double* A, int lda, double* Q, int ldq, double* L, int ldl);
/* QRSolver<T>::SolveRankRevealingQR / LQ / RQ / QL (LapackQRSolver.C:324-399):
 * the thin factorisation, then the pivots with |T_ii| <= eps whose row (QR,
 * QL) or column (LQ, RQ) of the triangular factor sums to at most eps are
 * removed with the matching column / row of the orthonormal factor.  kind: 0
 * QR, 1 LQ, 2 RQ, 3 QL.  QR / QL: F1 = Q (m x rank, ld1 >= m), F2 = R / L
 * (rank x n, ld2 >= min(m, n)); LQ / RQ: F1 = L / R (m x rank), F2 = Q
 * (rank x n).  *rank = columns / rows kept. */
int tn_qr_rank_revealing(tn_ctx ctx, int kind, int m, int n, const double* A, int lda, double* F1, int ld1,
                         double* F2, int ld2, double eps, int* rank);
/* SVCompressor<T>::Compress (TensorNetworks/SVCompressor.H:20,
 * SVCompressorImp.C:19-73) on device data: s (k, descending) is truncated and
 * rescaled in place; U (m x k, ldu) and Vt (k x n, ldvt) keep their leading
 * D columns/rows.  Returns the kept D and the discarded sum of s^2. */
int tn_compress(tn_ctx ctx, int Dmax, double eps, int k, double* s, int* D_out,
                double* discarded);

/* ---- iTEBD gates path -------------------------------------------------------
 * iTEBDState (TensorNetworks/iTEBDState.H) on an infinite chain with a
 * two-site unit cell, Vidal form.  FindiTimeGroundState
 * (iTEBDStateImp_iTime.C:25-104) with second-order Trotter gates
 * (iTEBDGates::InitGates, iTEBDGates.C:21-54) applied as
 * iTEBDStateImp::Apply(MultigateType) (iTEBDStateImp_iTime.C:119-135):
 * contraction, reshape (ReshapeForSVD), Jacobi SVD, SVCompressor truncation
 * (eps 1e-7 before the last two gates, Dmax after), Unpack. */
typedef struct tn_itebd_s* tn_itebd;
/* Gammas uniform(-1,1) from mt19937_64(seed), bond values 1/sqrt(D). */
int tn_itebd_create(tn_ctx ctx, double S, double Jxy, double Jz, double hz, int D, uint64_t seed,
                    tn_itebd* out);
int tn_itebd_destroy(tn_itebd st);
/* Site s (0 or 1): Gamma (d, Dl, Dr), element (n, i, j) at n*Dl*Dr + j*Dl + i;
 * bond b joins site b to site 1-b.  Dims of a site follow its two bonds. */
int tn_itebd_get_site(tn_itebd st, int site, int* Dl, int* Dr, double* host);
int tn_itebd_set_site(tn_itebd st, int site, int Dl, int Dr, const double* host);
int tn_itebd_get_bond(tn_itebd st, int bond, int* D, double* host);
int tn_itebd_set_bond(tn_itebd st, int bond, int D, const double* host);
/* nsteps second-order Trotter steps at time step dt, truncation to Dmax. */
int tn_itebd_step(tn_itebd st, double dt, int Dmax, int nsteps);
/* iTEBDStateImp::FindiTimeGroundState(H, iH, schedule)
 * (iTEBDStateImp_iTime.C:25-104) over the time steps dts[0..ndt), one
 * schedule line each: OrthogonalizeI, then for D = current .. Dmax by deltaD
 * (IncreaseBondDimensions) steps until both bond vectors move by at most
 * eps_factor*dt or max_iter steps, then OrthogonalizeI again.  steps_out[i]
 * receives the Trotter steps of line i. */
int tn_itebd_find_ground_state(tn_itebd st, const double* dts, int ndt, int max_iter, int Dmax,
                               int deltaD, double eps_factor, int* steps_out);
/* iTEBDStateImp::OrthogonalizeI(comp, eps, niter) (iTEBDStateImp_OrthoNorm.C:
 * 110-128, 511-637) at centre 1 with the (Dmax, 1e-16) compressor: the
 * iterative re-orthogonalisation to canonical Vidal form.  *delta: last change
 * of the bond values, *iters: iterations run.  TN_NOT_CONVERGED when a norm
 * matrix was singular (the reference's bail-out; the state is still unpacked). */
int tn_itebd_orthogonalize(tn_itebd st, int Dmax, double eps, int max_iter, double* delta, int* iters);
/* Energy per bond (iTEBDState::GetExpectation): transfer-matrix fixed points by
 * power iteration (max_iters, tolerance tol on the normalised fixed point). */
int tn_itebd_energy(tn_itebd st, int max_iters, double tol, double* E);

/* ---- learned Davidson correction (no counterpart in the reference) -------
 * A per-element MLP (4 -> 64 -> 64 -> 1, tanh; BF16 weights for inference,
 * FP32 master copy for training) maps (diag(Heff) - theta)/sigma, r/rms(r),
 * u*sqrt(N) and the bond position to the normalised Davidson correction.  It
 * is trained on pairs that FP64 diagonal-Davidson sweeps record (target: the
 * exact correction x/(u.x) - u towards the converged eigenvector x).  Sweeps
 * use it with tn_solver_options.eigensolver = TN_EIG_DAVIDSON and
 * use_learned = 1; diagonal Davidson takes over whenever it stalls. */
typedef struct tn_mlp_s* tn_mlp;
typedef struct tn_dataset_s* tn_dataset;
int tn_mlp_create(tn_ctx ctx, uint64_t seed, tn_mlp* out);
int tn_mlp_destroy(tn_mlp m);
int tn_mlp_num_params(void);
/* FP32 master parameters (layout W1[4][64], b1[64], W2[64][64], b2[64],
 * W3[64], b3); setting them also refreshes the BF16 copy and resets Adam. */
int tn_mlp_get_params(tn_mlp m, float* host);
int tn_mlp_set_params(tn_mlp m, const float* host);
/* Y[i] = MLP(F[i, 0:4]) with the BF16 weights (device pointers). */
int tn_mlp_forward(tn_mlp m, const float* F, long long n, float* Y);
/* Gradient of mean((MLP(F) - T)^2) w.r.t. the FP32 parameters (host, n_params). */
int tn_mlp_gradient(tn_mlp m, const float* F, const float* T, long long n, float* grad_host,
                    double* loss);
/* Adam on minibatches of a seeded permutation of the n pairs. */
int tn_mlp_train(tn_mlp m, const float* F, const float* T, long long n, int steps, int batch,
                 double lr, uint64_t seed, double* final_loss);
/* Training pairs recorded by FP64 diagonal-Davidson sweeps. */
int tn_dataset_create(tn_ctx ctx, long long capacity, tn_dataset* out);
int tn_dataset_destroy(tn_dataset ds);
long long tn_dataset_size(tn_dataset ds);
/* Device pointers: features (size x 4 floats) and targets (size floats). */
int tn_dataset_data(tn_dataset ds, const float** F, const float** T);
/* Attach (or detach with NULL) the learned correction / the recorder. */
int tn_mps_set_learned_correction(tn_mps psi, tn_mlp m);
int tn_mps_set_recorder(tn_mps psi, tn_dataset ds);

/* ---- full state: exact diagonalisation on the device ------------------------
 * FullState (TensorNetworks/FullState.H:15-35, FullStateImp.C): all d^L
 * amplitudes of the open chain (site 1 the most significant digit,
 * StateIterator::GetIndex), at most 2^31 - 1 of them.  The field enters as
 * hz Sz once per site (the MPO's convention; the reference's local matrix
 * Hamiltonian_1D_NN_Heisenberg::GetH adds it on both sites of every bond). */
typedef struct tn_fullstate_s* tn_fullstate;
/* Hamiltonian::CreateFullState (Hamiltonian.H:28): random amplitudes from seed. */
int tn_fullstate_create(tn_hamiltonian h, uint64_t seed, tn_fullstate* out);
int tn_fullstate_destroy(tn_fullstate fs);
/* FullState::GetSize: d^L. */
long long tn_fullstate_get_size(tn_fullstate fs);
/* FullState::FindGroundState(H, epsE) (FullStateImp.C:190-205): device Lanczos
 * on the operator below, residual target epsE; amplitudes normalised with the
 * sign of the first one above 0.01 positive (FullStateImp::Normalize). */
int tn_fullstate_find_ground_state(tn_fullstate fs, tn_hamiltonian h, double epsE, double* E, int* matvecs);
/* FullState::PowerIterate(H, epsE, epsPsi, maxIter) (FullStateImp.C:155-188). */
int tn_fullstate_power_iterate(tn_fullstate fs, tn_hamiltonian h, double epsE, double epsPsi, int max_iter,
                               double* E, int* iters);
/* FullState::GetE. */
int tn_fullstate_get_e(tn_fullstate fs, double* E);
/* Amplitudes to the host (d^L doubles). */
int tn_fullstate_get_amplitudes(tn_fullstate fs, double* host);
/* FullStateImp::DoMatVecContraction (FullStateImp.C:207-217), the
 * SparseEigenSolverClient face: y = H x on device vectors of d^L. */
int tn_fullstate_matvec(tn_fullstate fs, tn_hamiltonian h, const double* x, double* y);

/* Measurement hook (no counterpart in the reference): device microseconds per
 * step of the library's Lanczos Krylov kernels (CGS2 projections, update,
 * next vector, tridiagonal decision), replayed from its CUDA graph on a
 * diagonal operator of size N with a basis of m vectors; *bytes_per_step: the
 * algorithmic HBM bytes of one step, (j + 4) N doubles averaged over the
 * steps j plus the operator's read and write of 2 N doubles. */
int tn_lanczos_probe(tn_ctx ctx, long long N, int m, double* us_per_step, double* bytes_per_step);

#ifdef __cplusplus
}
#endif
#endif /* TN_CUDA_H */
