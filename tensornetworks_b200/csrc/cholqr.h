// cholqr.h -- Cholesky-QR2 for the sweep's gauge move (Householder fallback in qr.h).
#pragma once
#include "tn_internal.h"

namespace tnb {

bool cholqr_supported(int m, int n);
// A (m x n, ld m, m >= n) = Q (ld ldq) R (n x n, ld ldr).  *ok = false when a
// Cholesky pivot fails its threshold (cond(A) too large or rank deficient); the
// outputs are then unspecified and A is untouched.  Synchronises the stream.
int cholqr2_dense(Ctx& c, int m, int n, const double* A, double* Q, int ldq, double* R, int ldr, bool* ok);

}  // namespace tnb
