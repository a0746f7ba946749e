// lanczos.h -- device Lanczos state and host driver.
#pragma once
#include "split.cuh"
#include <functional>

#include "tn_internal.h"

namespace tnb {

constexpr int LZ_MAXK = 64;

struct LzState {
    int done;              // 1: converged or basis exhausted; later kernels skip
    int nb;                // basis size of the current restart
    int matvecs;           // Heff applications so far
    int converged;         // residual criterion met
    unsigned int counter;  // last-block reduction ticket
    int j;                 // step of the current restart (read by dots / update)
    int jn;                // index of the vector lz_next builds (set by update)
    int mmax;              // basis limit of the current restart
    double tol, theta, theta2, resid, xnorm;
    double tol_rel;        // additional residual target relative to |T| (split-precision operators)
    double alpha[LZ_MAXK], beta[LZ_MAXK];
    double h[LZ_MAXK], h2[LZ_MAXK];
    double y[LZ_MAXK];
    double rhist[LZ_MAXK];  // residual estimate after each step of the current restart
    // device-driven restarts: restarts done, Krylov steps over all restarts,
    // and the residual of the previous restart
    int restarts, steps;
    double prev_resid;
};

struct LzResult {
    double theta, theta2, resid;
    int matvecs, restarts, converged;
};

// What a device-driven solve leaves for the host (copied once it finishes).
struct LzSummary {
    double theta, theta2, resid;
    int matvecs, restarts, converged, steps;
    long long launches;  // kernels the solve ran
};

// mv(x, y, skip): enqueue y = Heff x on the context stream; the launches must
// do nothing when *skip != 0 (device flag).  The solver always passes the same
// x and y buffers, so the launches can be recorded once in a CUDA graph.
using MatvecFn = std::function<int(const double*, double*, const int*)>;

// theta = x.y/x.x and |y - theta x|/|x| (device vectors; synchronises).
int rayleigh_residual(Ctx& c, long long N, const double* x, const double* y, double* theta, double* resid);
// The same on stream st without waiting: dev (rayleigh_scratch_bytes) holds the
// reduction state; (theta, -, resid) land in host_out[0..2] (pinned) when the
// stream gets there.
size_t rayleigh_scratch_bytes(long long N, int sm_count);
int rayleigh_residual_async(cudaStream_t st, int sm_count, long long N, const double* x, const double* y, void* dev,
                            double* host_out);

// tol: absolute residual target; tol_rel (>= 0): residual target relative to
// the norm of the tridiagonal matrix (the operator's noise floor for the
// split-precision matvec).  With tol_rel > 0 the restarts also stop once the
// residual no longer drops by half between restarts.
// graph_key != 0 identifies the operator (every pointer and shape mv's launches
// depend on): the Lanczos steps of a restart then run as one CUDA graph with a
// device-driven WHILE loop, recorded on first use of the key and replayed.
// split (optional): the kernels that produce each Krylov vector also write its
// BF16 pieces there (for a split-precision mv that skips its own splitting).
int lanczos_solve(Ctx& c, long long N, double* x, int m, int maxRestarts, double tol, const MatvecFn& mv,
                  LzResult* out, double tol_rel = 0.0, unsigned long long graph_key = 0,
                  const VecSplit* split = nullptr);

// The same solve with the restart loop on the device too (a WHILE node around
// the WHILE node of the steps), so that nothing waits for the host: enqueues
// the whole solve and, after it, the copy of its summary to host_out (pinned).
// Returns LZ_ASYNC_UNAVAILABLE (nothing enqueued) when graphs are off or the
// nested graph cannot be built; the caller then uses lanczos_solve.
constexpr int LZ_ASYNC_UNAVAILABLE = -1;
int lanczos_solve_async(Ctx& c, long long N, double* x, int m, int maxRestarts, double tol, const MatvecFn& mv,
                        double tol_rel, unsigned long long graph_key, LzSummary* host_out,
                        const VecSplit* split = nullptr);

}  // namespace tnb
