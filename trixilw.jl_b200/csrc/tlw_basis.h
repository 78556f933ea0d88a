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

// Lagrange polynomials of `nodes` evaluated at t (barycentric; exact at a node)
inline std::vector<double> host_lagrange(const std::vector<double>& nodes, double t) {
    const int n = (int)nodes.size();
    std::vector<double> wb(n, 1.0), l(n, 0.0);
    for (int j = 0; j < n; ++j) {
        for (int k = 0; k < n; ++k)
            if (k != j) wb[j] *= nodes[j] - nodes[k];
        wb[j] = 1.0 / wb[j];
    }
    for (int j = 0; j < n; ++j)
        if (t == nodes[j]) { l[j] = 1.0; return l; }
    double s = 0.0;
    for (int j = 0; j < n; ++j) { l[j] = wb[j] / (t - nodes[j]); s += l[j]; }
    for (int j = 0; j < n; ++j) l[j] /= s;
    return l;
}

// Operators of the L2 mortar between one large face and its two halves (Trixi LobattoLegendreMortarL2,
// restated from the mathematics): out[0] forward_upper, [1] forward_lower (interpolation of the large face
// polynomial at the half's GLL nodes, t = (x +- 1) / 2), [2] reverse_upper, [3] reverse_lower (exact L2
// projection of the halves back onto the large face, computed through the N+1 point Gauss basis whose
// mass matrix is diagonal and exact for the degree-2N products). Row-major n x n in 64 slots.
inline void host_mortar_operators(int N, double out[4][64]) {
    const int n = N + 1;
    std::vector<double> x;
    Basis B;
    host_build_basis(N, B, &x);
    std::memset(out, 0, 4 * 64 * sizeof(double));
    for (int i = 0; i < n; ++i) {
        const auto lu = host_lagrange(x, 0.5 * (x[i] + 1.0));
        const auto ll = host_lagrange(x, 0.5 * (x[i] - 1.0));
        for (int j = 0; j < n; ++j) { out[0][i * n + j] = lu[j]; out[1][i * n + j] = ll[j]; }
    }
    // Gauss-Legendre nodes / weights (Newton on P_n from -cos((2j+1) pi / 2n))
    std::vector<double> g(n), wg(n);
    const double pi = 3.14159265358979323846;
    auto legendre = [&](double t, double& p, double& dp) {
        double p0 = 1.0, p1 = t, d0 = 0.0, d1 = 1.0;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
            const double d2 = d0 + (2.0 * k - 1.0) * p1;
            p0 = p1; p1 = p2; d0 = d1; d1 = d2;
        }
        p = p1;
        dp = d1;
    };
    for (int j = 0; j < n; ++j) {
        double t = -std::cos((2.0 * j + 1.0) * pi / (2.0 * n)), p, dp;
        for (int it = 0; it < 100; ++it) {
            legendre(t, p, dp);
            const double d = -p / dp;
            t += d;
            if (std::fabs(d) <= 4.0 * 2.220446049250313e-16 * std::fabs(t)) break;
        }
        legendre(t, p, dp);
        g[j] = t;
        wg[j] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
    std::vector<double> g2l(n * n), l2g(n * n);
    for (int i = 0; i < n; ++i) {
        const auto a = host_lagrange(g, x[i]);
        const auto c = host_lagrange(x, g[i]);
        for (int j = 0; j < n; ++j) { g2l[i * n + j] = a[j]; l2g[i * n + j] = c[j]; }
    }
    for (int half = 0; half < 2; ++half) {
        const double shift = half == 0 ? 1.0 : -1.0;
        std::vector<double> op(n * n), tmp(n * n, 0.0);
        for (int j = 0; j < n; ++j) {
            const auto lg = host_lagrange(g, 0.5 * (g[j] + shift));
            for (int i = 0; i < n; ++i) op[i * n + j] = 0.5 * lg[i] * wg[j] / wg[i];
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) tmp[i * n + j] += op[i * n + k] * l2g[k * n + j];
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double acc = 0.0;
                for (int k = 0; k < n; ++k) acc += g2l[i * n + k] * tmp[k * n + j];
                out[2 + half][i * n + j] = acc;
            }
    }
}

}  // namespace tlw
