// engine.h -- device-resident Hamiltonian (MPO) and MPS with the reference's
// variational sweep semantics (MPSImp_Variational.C:16-173).
#pragma once
#include <vector>

#include "contract.h"
#include "lanczos.h"
#include "mixed.h"
#include "davidson.h"
#include "mlp.h"
#include "qr.h"

namespace tnb {

struct SiteMPO {
    int Dw1 = 1, Dw2 = 1;
    std::vector<double> W;  // (w1,w2,m,n)
    size_t offLR = 0, offRL = 0, offW = 0;
    int nLR = 0, nRL = 0;
};

struct Hamiltonian {
    Ctx* ctx = nullptr;
    int L = 0, d = 2, form = 2;
    double S = 0.5, Jxy = 1, Jz = 1, hz = 0;
    std::vector<SiteMPO> ops;   // 1-based
    std::vector<SiteMPO> ops2;  // product MPO (H^2), 1-based
    DevBuf terms;               // all term lists (WTermDev)
    DevBuf Wdev;                // all W tensors (for diag(Heff))
    int build();
};

// Site tensors of a second MPS (the imaginary-time target |psi2>), 1-based.
struct SiteSet {
    std::vector<DevBuf*> A;
    std::vector<int> D1, D2;
};

struct MPSState {
    Ctx* ctx = nullptr;
    Hamiltonian* H = nullptr;
    int L = 0, d = 2;
    double normEps = 1e-12, epsSV = 1e-12;
    std::vector<int> D1, D2;                  // 1-based
    std::vector<DevBuf*> A;                   // site tensors
    std::vector<DevBuf*> Lenv, Renv;          // 0..L+1
    std::vector<int> LenvDw, LenvD, RenvDw, RenvD;
    std::vector<std::vector<double>> bond_s;  // 1..L-1, normalised
    std::vector<double> bond_maxDelta;
    // Triangular factor of the last gauge move of each bond, kept per direction
    // (0: left-to-right half-sweep, 1: right-to-left), with its dims.  The bond
    // singular values are the singular values of these factors and are computed
    // only when something reads them (the dlambda test of the sweep loop runs
    // only when dE is already below its epsilon; accessors).
    std::vector<DevBuf*> bondR[2];
    std::vector<int> bondRm[2], bondRn[2];
    std::vector<char> bondHave[2];
    std::vector<int> bondLatest;              // direction of the most recent gauge move
    std::vector<int> bondK;                   // current bond dimension (Bond::GetD)
    std::vector<char> bondDirty;              // bond_s lags behind the latest factor
    std::vector<double> Emin, iterDE, gapE;
    DevBuf tmp, Wqr, Qqr, svdw, envA, envB, yvec, diagbuf;
    // FP64 check of the split-precision eigenvector on the context's second side
    // stream (refine_tol = 0): contraction scratch, reduction state, and per site
    // (theta, -, resid, error flag) in pinned memory, applied by rq_collect().
    // With the device-driven Lanczos solve (lanczos_solve_async) its summary
    // goes to the same slot (doubles 4 ..) and is applied there too.
    static constexpr int RQ_SLOT = 12;  // doubles per site
    DevBuf rqP, rqQ, rqbuf;
    HostBuf rqhost;
    std::vector<char> rq_pending, rq_lz, rq_exact;  // rq_exact: an FP64 solve, no separate check
    std::vector<double> rq_dtheta, rq_flop;
    bool rq_inflight = false;
    MixedSite msite;
    long long matvecs = 0, matvecs_fp64 = 0;
    double heff_flop = 0;
    int not_converged = 0, fallbacks = 0;
    long long learned_steps = 0, learned_stalls = 0;  // Davidson with the learned correction
    MlpModel* mlp = nullptr;         // learned Davidson correction (not owned)
    DvRecorder* recorder = nullptr;  // training-pair recorder (not owned)
    tn_solver_options opt{};
    // phase timing (verbose >= 2): seconds in refine / gauge / environment / bond values
    double t_refine = 0, t_gauge = 0, t_env = 0, t_bond = 0;
    unsigned long long n_refine = 0, n_gauge = 0, n_env = 0;  // launches per phase (verbose >= 2)
    // device phase timing (opt.phase_timing): four events per site of a half-sweep,
    // read after the half-sweep; milliseconds in refine / gauge / environment
    std::vector<cudaEvent_t> phase_ev;
    double phase_ms[3] = {0, 0, 0};
    int phase_events_ensure(size_t n);

    ~MPSState();
    int init(Hamiltonian* h, int D);
    int initialize_random(unsigned long long seed);
    int max_D() const;
    int ensure_capacity(int D);
    int normalize_site(int ia, bool left);
    int normalize_all(bool left);
    int bond_values(const std::vector<std::pair<int, int>>& which, std::vector<std::vector<double>>& out);
    int ensure_bond_values();
    void set_bond_dim(int b, int nD);   // Bond::NewBondDimension           // bond_s from the latest factor of every dirty bond
    int sweep_pair_dlambda(double* dl); // Bond::GetMaxDelta over the last two half-sweeps
    int compute_left_env(int ia);
    int compute_right_env(int ia);
    int load_heff_caches();
    int refine_site(int ia, double epsEigen);
    int refine_site_mixed(int ia, double epsEigen);
    int refine_site_davidson(int ia, double epsEigen);
    int sweep(bool left, double epsEigen);
    int increase_bond_dims(int D);
    int expectation(const std::vector<SiteMPO>& ops, double* E);
    // reduced density matrices (dms.cu): L d x d blocks; for the pairs ia < ib in
    // order, d^4 values rho[((m d + m2) d + n) d + n2]
    int one_site_dms(double* out_host);
    int two_site_dms(double* out_host);
    int dm_scatter(const double* dots, double* rho);
    // imaginary-time evolution (itime.cu)
    int site_reserve(int ia, size_t n);
    int trotter_mpo(double dt, int order, std::vector<SiteMPO>& out) const;
    int apply_mpo_inplace(const std::vector<SiteMPO>& W);
    int svd_compress_sweep(bool left, int Dmax, double eps, std::vector<std::vector<double>>* svals);
    int overlap_left(int ia, const SiteSet& P2, std::vector<DevBuf*>& Lo);
    int overlap_right(int ia, const SiteSet& P2, std::vector<DevBuf*>& Ro);
    int overlap_site(int ia, const SiteSet& P2, std::vector<DevBuf*>& Lo, std::vector<DevBuf*>& Ro);
    int itime_ground_state(const tn_itime_line* lines, int nlines, double* variance, int* iters_out);
    int find_ground_state(const tn_sched_line* lines, int nlines, const tn_solver_options* opt,
                          tn_sweep_stats* stats);
    int sweep_pairs(int nsweeps, double epsEigen, const tn_solver_options* opt, tn_sweep_stats* stats);
    int prepare_sweeps();
    int site_resize(int ia, int nD1, int nD2);
    int gauge_qr(int m, int n, double* W, double* Q, double* R, int ldr);
    int rescale_site(int ia);
    int rq_slots();
    int rq_launch(int ia, const ContractShape& s, const WTermDev* t, int nLR, const double* F, const double* G,
                  long long N, double dtheta);
    void rq_order();   // the context stream waits for the in-flight check (before A[ia] changes)
    int rq_collect();  // wait for the checks and apply them to Emin / iterDE / gapE
};

}  // namespace tnb

struct tn_hamiltonian_s {
    tnb::Hamiltonian h;
};
struct tn_mps_s {
    tnb::MPSState m;
};
