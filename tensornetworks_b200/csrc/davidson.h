// davidson.h -- device Davidson eigensolver (lowest pair) with a diagonal or
// learned (per-element MLP) correction.
#pragma once
#include "lanczos.h"

namespace tnb {

constexpr int DV_MAXK = 32;  // largest subspace (projected matrix in shared memory)

struct DvState {
    int done;              // converged / cannot expand / iteration cap: later kernels skip
    int k;                 // current subspace size
    int matvecs;
    int converged;
    unsigned int counter;  // last-block reduction ticket
    int restart;           // subspace full: the next step restarts from the Ritz vector
    int stalled;           // learned correction stalled: the diagonal one from now on
    int iters;             // corrections taken
    int kmax, max_iters;
    int learned;           // 1: use the MLP correction while not stalled
    int learned_steps;     // corrections the MLP produced
    int recorded;          // steps written to the training recorder
    int pad;
    double tol, tol_rel, theta, resid;
    double rms_r, sigma;   // |r|/sqrt(N) and rms(diag - theta): feature scales
    double tnorm;          // norm of the orthogonalised correction
    double pos;            // bond position feature
    double S[DV_MAXK * DV_MAXK];  // projected matrix V^T H V (column-major, ld DV_MAXK)
    double h[DV_MAXK], h2[DV_MAXK];
    double s[DV_MAXK];     // Ritz coefficients of the lowest pair
    double rhist[256];     // residual after each step
};

struct DvResult {
    double theta, resid;
    int matvecs, iters, converged, learned_steps, stalled;
};

// Per-element MLP used as the Davidson correction (mlp.h).
struct MlpModel;
// Feature/target recorder for training (mlp.h).
struct DvRecorder;

// Lowest eigenpair of the operator mv (symmetric, N x N).  x: start vector in,
// normalised Ritz vector out.  diag: the operator's diagonal (device, N).
// mlp == nullptr: diagonal Davidson.  pos: bond position feature in [0, 1].
// rec: with the diagonal correction, every step's features and Ritz vector
// are recorded and turned into training pairs once x is known.
// tol_rel > 0 (split-precision operators): also stop at |r| <= tol_rel
// max(|theta|, sigma) or when the residual stops halving over two steps.
int davidson_solve(Ctx& c, long long N, double* x, int kmax, int max_iters, double tol, const MatvecFn& mv,
                   const double* diag, const MlpModel* mlp, double pos, DvResult* out, DvRecorder* rec = nullptr,
                   unsigned long long graph_key = 0, double tol_rel = 0.0);

}  // namespace tnb
