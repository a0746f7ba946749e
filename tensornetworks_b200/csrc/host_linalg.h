// host_linalg.h -- small dense host linear algebra for operator set-up (gates
// of the Trotter MPO, compression of the H^2 MPO): matrices of at most a few
// hundred entries per side, built once per schedule line or Hamiltonian.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

namespace tnb {

// host one-sided Jacobi SVD of an m x n column-major matrix (m >= n): A = U diag(s) V^T
inline void host_svd(std::vector<double> A, int m, int n, std::vector<double>& U, std::vector<double>& s,
              std::vector<double>& V) {
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 80; ++sweep) {
        bool rot = false;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double a = 0, b = 0, g = 0;
                for (int i = 0; i < m; ++i) {
                    const double x = A[(size_t)p * m + i], y = A[(size_t)q * m + i];
                    a += x * x;
                    b += y * y;
                    g += x * y;
                }
                if (g == 0.0 || std::fabs(g) <= 1e-15 * std::sqrt(a * b)) continue;
                rot = true;
                const double zeta = (b - a) / (2 * g);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
                const double c = 1 / std::sqrt(1 + t * t), sn = c * t;
                for (int i = 0; i < m; ++i) {
                    const double x = A[(size_t)p * m + i], y = A[(size_t)q * m + i];
                    A[(size_t)p * m + i] = c * x - sn * y;
                    A[(size_t)q * m + i] = sn * x + c * y;
                }
                for (int i = 0; i < n; ++i) {
                    const double x = V[(size_t)p * n + i], y = V[(size_t)q * n + i];
                    V[(size_t)p * n + i] = c * x - sn * y;
                    V[(size_t)q * n + i] = sn * x + c * y;
                }
            }
        if (!rot) break;
    }
    s.assign(n, 0.0);
    U.assign((size_t)m * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double nr = 0;
        for (int i = 0; i < m; ++i) nr += A[(size_t)j * m + i] * A[(size_t)j * m + i];
        s[j] = std::sqrt(nr);
        for (int i = 0; i < m; ++i) U[(size_t)j * m + i] = s[j] > 0 ? A[(size_t)j * m + i] / s[j] : 0.0;
    }
}


// Thin SVD of any m x n column-major matrix: A = U diag(s) V^T with r = min(m, n)
// columns in U (m x r) and V (n x r), unsorted.
inline void host_svd_thin(const std::vector<double>& A, int m, int n, std::vector<double>& U, std::vector<double>& s,
                          std::vector<double>& V) {
    if (m >= n) {
        host_svd(A, m, n, U, s, V);
        return;
    }
    std::vector<double> At((size_t)n * m);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) At[(size_t)j + (size_t)i * n] = A[(size_t)i + (size_t)j * m];
    host_svd(At, n, m, V, s, U);  // A^T = V s U^T
}

}  // namespace tnb
