// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle.  Nothing in the product
// (edus_2.0_b200/) may include, link or call this file.
//
// Dense Hermitian eigensolver standing in for LAPACKE_zheevd, shared by the
// oracle restatement (oracle/edus_oracle.cpp) and by the MKL stand-in that
// the reference's own sources are compiled against (oracle/refshim/).
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace oracle {

using cd = std::complex<double>;

// ---------------------------------------------------------------------------
// Hermitian eigensolver (stands in for LAPACKE_zheevd 'V','U',
// src/Geometry/Matrix.cpp:10-23): cyclic complex Jacobi on the matrix built
// from the upper triangle; eigenvalues ascending, eigenvectors in columns.
inline void eigh(int n, const cd* Ain, double* w, cd* V) {
    std::vector<cd> A((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            if (j >= i) A[i * n + j] = Ain[i * n + j];
            else A[i * n + j] = std::conj(Ain[j * n + i]);
        }
    for (int i = 0; i < n; ++i) A[i * n + i] = A[i * n + i].real();
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, diag = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                if (i != j) off += std::norm(A[i * n + j]);
                else diag += std::norm(A[i * n + j]);
            }
        if (off <= 1e-32 * (diag + 1e-300) || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                cd g = A[p * n + q];
                double ag = std::abs(g);
                if (ag == 0.0) continue;
                double app = A[p * n + p].real(), aqq = A[q * n + q].real();
                cd ph = g / ag;  // e^{i phi}
                double theta = (aqq - app) / (2.0 * ag);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                // R = [[c, s e^{i phi}], [-s e^{-i phi}, c]] on (p,q); A <- R^H A R
                for (int k = 0; k < n; ++k) {  // A R (columns)
                    cd akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * std::conj(ph) * akq;
                    A[k * n + q] = s * ph * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // R^H A (rows)
                    cd apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * ph * aqk;
                    A[q * n + k] = s * std::conj(ph) * apk + c * aqk;
                }
                A[p * n + q] = 0.0;
                A[q * n + p] = 0.0;
                A[p * n + p] = app - t * ag;
                A[q * n + q] = aqq + t * ag;
                for (int k = 0; k < n; ++k) {
                    cd vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * std::conj(ph) * vkq;
                    V[k * n + q] = s * ph * vkp + c * vkq;
                }
            }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::vector<double> ev(n);
    for (int i = 0; i < n; ++i) ev[i] = A[i * n + i].real();
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ev[a] < ev[b]; });
    std::vector<cd> Vs((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        w[j] = ev[order[j]];
        for (int i = 0; i < n; ++i) Vs[i * n + j] = V[i * n + order[j]];
    }
    std::copy(Vs.begin(), Vs.end(), V);
}

}  // namespace oracle
