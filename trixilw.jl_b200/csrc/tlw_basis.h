// tlw_basis.h -- Gauss-Lobatto-Legendre basis on the host (Trixi's LobattoLegendreBasis), restated from
// Kopriva, "Implementing Spectral Methods for PDEs": Legendre recursion (Alg. 22/24), nodes and weights
// (Alg. 25), barycentric weights (Alg. 30), derivative matrix with the negative-sum diagonal (Alg. 37);
// Dhat = -M^{-1} D^T M and the weak-form lift factors 1/w_1, 1/w_n.
#pragma once
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "tlw_device.cuh"

namespace tlw {

inline void host_legendre_q(int N, double x, double& q, double& dq, double& LN) {
    double a = 1.0, b = x, da = 0.0, db = 1.0;
    for (int k = 2; k <= N; ++k) {
        const double c = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / k;
        const double dc = da + (2.0 * k - 1.0) * b;
        a = b; b = c; da = db; db = dc;
    }
    const int k = N + 1;
    const double c = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / k;
    const double dc = da + (2.0 * k - 1.0) * b;
    q = c - a;
    dq = dc - da;
    LN = b;
}

inline void host_build_basis(int N, Basis& B, std::vector<double>* nodes_out = nullptr) {
    const int n = N + 1;
    std::vector<double> x(n), w(n), wb(n, 1.0);
    x[0] = -1.0; x[N] = 1.0;
    w[0] = w[N] = 2.0 / (N * (N + 1.0));
    const double pi = 3.14159265358979323846;
    for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
        double xj = -std::cos((j + 0.25) * pi / N - 3.0 / (8.0 * N * pi * (j + 0.25)));
        double q, dq, LN;
        for (int it = 0; it < 100; ++it) {
            host_legendre_q(N, xj, q, dq, LN);
            const double d = -q / dq;
            xj += d;
            if (std::fabs(d) <= 4.0 * 2.220446049250313e-16 * std::fabs(xj)) break;
        }
        host_legendre_q(N, xj, q, dq, LN);
        x[j] = xj; x[N - j] = -xj;
        w[j] = w[N - j] = 2.0 / (N * (N + 1.0) * LN * LN);
    }
    if (N >= 2 && N % 2 == 0) {
        double q, dq, LN;
        host_legendre_q(N, 0.0, q, dq, LN);
        x[N / 2] = 0.0;
        w[N / 2] = 2.0 / (N * (N + 1.0) * LN * LN);
    }
    for (int j = 0; j < n; ++j) {
        for (int k = 0; k < n; ++k)
            if (k != j) wb[j] *= (x[j] - x[k]);
        wb[j] = 1.0 / wb[j];
    }
    std::memset(&B, 0, sizeof(B));
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c)
            if (c != r) {
                B.D[r * n + c] = wb[c] / wb[r] / (x[r] - x[c]);
                B.D[r * n + r] -= B.D[r * n + c];
            }
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) B.Dhat[r * n + c] = -B.D[c * n + r] * w[c] / w[r];
    for (int k = 0; k < n; ++k) B.weights[k] = w[k];
    B.inv_w_first = 1.0 / w[0];
    B.inv_w_last = 1.0 / w[n - 1];
    // inverse of V[i][m] = sqrt(m + 1/2) P_m(x_i) (Trixi vandermonde_legendre), Gauss-Jordan with pivoting
    std::vector<double> A(n * n), I(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int m = 0; m < n; ++m) {
            double p = 1.0;
            if (m >= 1) {
                double a = 1.0, b = x[i];
                p = x[i];
                for (int k = 2; k <= m; ++k) {
                    p = ((2.0 * k - 1.0) * x[i] * b - (k - 1.0) * a) / k;
                    a = b; b = p;
                }
            }
            A[i * n + m] = p * std::sqrt(m + 0.5);
        }
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        for (int k = 0; k < n; ++k) {
            std::swap(A[c * n + k], A[piv * n + k]);
            std::swap(I[c * n + k], I[piv * n + k]);
        }
        const double d = A[c * n + c];
        for (int k = 0; k < n; ++k) { A[c * n + k] /= d; I[c * n + k] /= d; }
        for (int r = 0; r < n; ++r)
            if (r != c) {
                const double f = A[r * n + c];
                for (int k = 0; k < n; ++k) { A[r * n + k] -= f * A[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
            }
    }
    for (int k = 0; k < n * n; ++k) B.Vinv[k] = I[k];
    if (nodes_out) *nodes_out = x;
}

}  // namespace tlw
