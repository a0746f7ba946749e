// qr.h -- Householder QR and one-sided Jacobi SVD on the device.
#pragma once
#include "tn_internal.h"

namespace tnb {

// In-place blocked Householder QR of the dense column-major W (m x n, ld m).
// Writes Q (m x k, ld ldq) and R (k x n, ld ldr) when the pointers are non-null.
int qr_dense(Ctx& c, int m, int n, double* W, double* Qout, int ldq, double* Rout, int ldr);

// Reads (and clears) the context's sticky device error word, raised when a
// bounded wait between CTAs expired; waits for the device.
int check_device_error(Ctx& c);

// One job of the batched one-sided Jacobi SVD (one CTA per job).  W is the
// tall (m >= n) working copy, overwritten.  With vectors: U (m x n, ldu),
// Vt (n x n, ldvt) and a scratch V (n x n, ld n).  s (n) is always written.
struct SvdJob {
    double* W;
    int m, n;
    double* V;
    double* U;
    int ldu;
    double* Vt;
    int ldvt;
    double* s;
    int* sweeps;  // may be null
};

int svd_batched(Ctx& c, const std::vector<SvdJob>& jobs, bool vectors);

}  // namespace tnb
