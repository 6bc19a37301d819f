// Eigenvalues and eigenvectors of a real symmetric tridiagonal matrix (host code).  The 4-wall duct's pressure solve
// diagonalises S = W^(1/2) Dzz W^(-1/2) once at context creation (src/initialization.f90:579-608, where the reference
// calls LAPACK dstev).  This is the implicit QL method with Wilkinson shifts (Bowdler, Martin, Reinsch and Wilkinson,
// "The QR and QL algorithms for symmetric matrices", Numer. Math. 11, 1968; the tql2 procedure), applied to the
// identity to accumulate the eigenvectors, and the pairs are sorted ascending as dstev returns them.
#pragma once
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace dfdm {

// d: diagonal (n), e: off-diagonal (n - 1; e[i] couples rows i and i + 1).  On success d holds the eigenvalues in
// ascending order and q (n x n, row-major) the orthonormal eigenvectors, q[k * n + m] = component k of vector m.
inline bool tridiag_eigen(std::vector<double> &d, std::vector<double> e, std::vector<double> &q) {
    const int n = (int)d.size();
    e.resize(std::max(n, 1), 0.0);
    if (n > 0) e[n - 1] = 0.0;
    std::vector<double> z((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) z[(size_t)i * n + i] = 1.0;
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < n; ++l) {
        for (int iter = 0;; ++iter) {
            int m = l;
            for (; m < n - 1; ++m)
                if (std::fabs(e[m]) <= eps * (std::fabs(d[m]) + std::fabs(d[m + 1]))) break;
            if (m == l) break;
            if (iter >= 60) return false;
            // Wilkinson shift from the leading 2 x 2 block, then one implicit QL sweep from m up to l
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            bool deflated = false;
            for (int i = m - 1; i >= l; --i) {
                double f = s * e[i];
                const double b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {   // the plane rotation vanished: the matrix split, restart on the smaller block
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; ++k) {
                    f = z[(size_t)k * n + i + 1];
                    z[(size_t)k * n + i + 1] = s * z[(size_t)k * n + i] + c * f;
                    z[(size_t)k * n + i] = c * z[(size_t)k * n + i] - s * f;
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
    std::vector<double> ds(n);
    q.assign((size_t)n * n, 0.0);
    for (int m = 0; m < n; ++m) {
        ds[m] = d[order[m]];
        for (int k = 0; k < n; ++k) q[(size_t)k * n + m] = z[(size_t)k * n + order[m]];
    }
    d = ds;
    return true;
}

}  // namespace dfdm
