// tlw_oracle.hpp -- CPU restatement of TrixiLW's Lax-Wendroff / MDRK right-hand side on TreeMesh{2}
// for the 2D compressible Euler equations.
//
// TEST INFRASTRUCTURE ONLY. This header is the oracle against which the CUDA library is checked. Only
// the test-suite, the smoke check and the CPU-baseline leg of the benchmark may call it; the product
// path never does.
//
// Parity status: UNPINNED against the reference itself. The reference is Julia + Trixi.jl, neither of
// which exists on this machine, and it ships no tests, golden vectors or rhs fixtures. The restatement is
// therefore pinned by properties the reference's scheme has by construction (exact free-stream
// preservation, discrete conservation on periodic meshes, design order of accuracy on the isentropic
// vortex, symmetry under mirroring) and by hand-checked known answers (GLL nodes/weights, the
// derivative matrix). Every function cites the reference file:line it restates (paths relative to the
// TrixiLW.jl repository root). Trixi.jl pieces that are not in the reference (basis, Euler flux,
// max_abs_speed, surface integral, apply_jacobian, max_dt) are restated from their mathematics.
//
// Array layout is the reference's (Julia column-major, leftmost index fastest):
//   u, du       [v, i, j, e]        -> u[v + NV*(i + n*(j + n*e))]
//   F (element) [v, d, i, j, e]     -> d = 0 x-flux, d = 1 y-flux
//   interfaces  [side, v, i, I]     -> side 0 = left, 1 = right
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

namespace tlwo {

constexpr int NV = 4;
constexpr int MAXN = 8;   // oracle supports polydeg <= 7

// fixed-size per-element scratch tile [v, i, j]
struct Tile {
    double a[NV * MAXN * MAXN];
    double& operator[](int k) { return a[k]; }
    const double& operator[](int k) const { return a[k]; }
    void zero(int m) { for (int k = 0; k < m; ++k) a[k] = 0.0; }
};

// ------------------------------------------------------------------------------------------------
// Lobatto-Legendre basis (Trixi.jl LobattoLegendreBasis; restated from Kopriva, "Implementing
// Spectral Methods for PDEs", Alg. 22/24/25 (Legendre recursion, GLL nodes/weights), Alg. 30
// (barycentric weights), Alg. 37 (derivative matrix with the negative-sum diagonal)).
// ------------------------------------------------------------------------------------------------
struct Basis {
    int n = 0;                      // nodes per direction, N + 1
    std::vector<double> nodes, weights, wbary;
    std::vector<double> D;          // D[a*n + b]    = l_b'(x_a)          (Trixi derivative_matrix[a, b])
    std::vector<double> Dhat;       // Dhat[a*n + b] = -D[b, a] w_b / w_a (Trixi derivative_dhat[a, b])
    double inv_w_first = 0, inv_w_last = 0;   // Trixi boundary_interpolation[1,1], [n,2]
    // LobattoLegendreMortarL2 (Trixi): forward_{upper,lower}[i*n + j] = l_j((x_i +- 1) / 2), reverse_* the L2
    // projections back onto the large face (computed in make_basis from their mathematics)
    std::vector<double> fwd_upper, fwd_lower, rev_upper, rev_lower;
};

// Lagrange basis polynomials of `nodes` at x (barycentric form, exact at the nodes)
inline std::vector<double> lagrange_at(const std::vector<double>& nodes, double x) {
    const int n = (int)nodes.size();
    std::vector<double> wb(n, 1.0), l(n, 0.0);
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k)
            if (k != j) wb[j] *= nodes[j] - nodes[k];
    for (int j = 0; j < n; ++j) {
        if (x == nodes[j]) { l[j] = 1.0; return l; }
        wb[j] = 1.0 / wb[j];
    }
    double den = 0.0;
    for (int j = 0; j < n; ++j) {
        l[j] = wb[j] / (x - nodes[j]);
        den += l[j];
    }
    for (int j = 0; j < n; ++j) l[j] /= den;
    return l;
}

// Gauss-Legendre nodes and weights with n points (Newton on P_n, Kopriva Alg. 23)
inline void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const double pi = 3.14159265358979323846;
    for (int j = 0; j < n; ++j) {
        double xj = -std::cos((2.0 * j + 1.0) * pi / (2.0 * n)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = xj;
            dp = 1.0;
            double d0 = 0.0;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * xj * p1 - (k - 1.0) * p0) / k;
                const double d2 = d0 + (2.0 * k - 1.0) * p1;
                p0 = p1; p1 = p2; d0 = dp; dp = d2;
            }
            if (n == 1) { p1 = xj; dp = 1.0; }
            const double delta = -p1 / dp;
            xj += delta;
            if (std::fabs(delta) <= 4.0 * std::numeric_limits<double>::epsilon() * std::fabs(xj)) break;
        }
        // derivative at the converged root
        double p0 = 1.0, p1 = xj, d0 = 0.0;
        dp = 1.0;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * xj * p1 - (k - 1.0) * p0) / k;
            const double d2 = d0 + (2.0 * k - 1.0) * p1;
            p0 = p1; p1 = p2; d0 = dp; dp = d2;
        }
        x[j] = xj;
        w[j] = 2.0 / ((1.0 - xj * xj) * dp * dp);
    }
}

// The L2 mortar operators: forward = interpolation of the large face onto the small halves; reverse = the
// L2 projection of the two halves back onto the large face, exact (done in the Gauss basis, whose mass
// matrix is diagonal and exact for these degree-2N products, then mapped to and from the Lobatto nodes).
inline void mortar_operators(Basis& b) {
    const int n = b.n;
    b.fwd_upper.assign(n * n, 0.0);
    b.fwd_lower.assign(n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        const auto lu = lagrange_at(b.nodes, 0.5 * (b.nodes[i] + 1.0));
        const auto ll = lagrange_at(b.nodes, 0.5 * (b.nodes[i] - 1.0));
        for (int j = 0; j < n; ++j) { b.fwd_upper[i * n + j] = lu[j]; b.fwd_lower[i * n + j] = ll[j]; }
    }
    std::vector<double> g, wg;
    gauss_legendre(n, g, wg);
    std::vector<double> g2l(n * n), l2g(n * n);   // g2l[i][j] = lg_j(x_i); l2g[i][j] = l_j(g_i)
    for (int i = 0; i < n; ++i) {
        const auto a = lagrange_at(g, b.nodes[i]);
        const auto c = lagrange_at(b.nodes, g[i]);
        for (int j = 0; j < n; ++j) { g2l[i * n + j] = a[j]; l2g[i * n + j] = c[j]; }
    }
    auto reverse = [&](double shift, std::vector<double>& out) {
        std::vector<double> op(n * n), tmp(n * n, 0.0);
        for (int j = 0; j < n; ++j) {
            const auto lg = lagrange_at(g, 0.5 * (g[j] + shift));
            for (int i = 0; i < n; ++i) op[i * n + j] = 0.5 * lg[i] * wg[j] / wg[i];
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) tmp[i * n + j] += op[i * n + k] * l2g[k * n + j];
        out.assign(n * n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) out[i * n + j] += g2l[i * n + k] * tmp[k * n + j];
    };
    reverse(1.0, b.rev_upper);
    reverse(-1.0, b.rev_lower);
}

inline void legendre_q_and_l(int N, double x, double& q, double& dq, double& LN) {
    // Kopriva Alg. 24 (qAndLEvaluation)
    double L_m2 = 1.0, L_m1 = x, dL_m2 = 0.0, dL_m1 = 1.0, L = 0, dL = 0;
    for (int k = 2; k <= N; ++k) {
        L = (2.0 * k - 1.0) / k * x * L_m1 - (k - 1.0) / k * L_m2;
        dL = dL_m2 + (2.0 * k - 1.0) * L_m1;
        L_m2 = L_m1; L_m1 = L; dL_m2 = dL_m1; dL_m1 = dL;
    }
    const int k = N + 1;
    const double L_p1 = (2.0 * k - 1.0) / k * x * L_m1 - (k - 1.0) / k * L_m2;
    const double dL_p1 = dL_m2 + (2.0 * k - 1.0) * L_m1;
    q = L_p1 - L_m2;
    dq = dL_p1 - dL_m2;
    LN = L_m1;
}

inline Basis make_basis(int N) {
    if (N < 1 || N + 1 > MAXN) throw std::invalid_argument("polydeg out of range");
    Basis b;
    b.n = N + 1;
    const int n = b.n;
    b.nodes.assign(n, 0.0);
    b.weights.assign(n, 0.0);
    // Kopriva Alg. 25 (LegendreGaussLobattoNodesAndWeights)
    if (N == 1) {
        b.nodes = {-1.0, 1.0};
        b.weights = {1.0, 1.0};
    } else {
        b.nodes[0] = -1.0; b.nodes[N] = 1.0;
        b.weights[0] = b.weights[N] = 2.0 / (N * (N + 1.0));
        const double pi = 3.14159265358979323846;
        for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
            double x = -std::cos((j + 0.25) * pi / N - 3.0 / (8.0 * N * pi * (j + 0.25)));
            double q, dq, LN;
            for (int it = 0; it < 100; ++it) {
                legendre_q_and_l(N, x, q, dq, LN);
                const double delta = -q / dq;
                x += delta;
                if (std::fabs(delta) <= 4.0 * std::numeric_limits<double>::epsilon() * std::fabs(x)) break;
            }
            legendre_q_and_l(N, x, q, dq, LN);
            b.nodes[j] = x;
            b.nodes[N - j] = -x;
            b.weights[j] = b.weights[N - j] = 2.0 / (N * (N + 1.0) * LN * LN);
        }
        if (N % 2 == 0) {
            double q, dq, LN;
            legendre_q_and_l(N, 0.0, q, dq, LN);
            b.nodes[N / 2] = 0.0;
            b.weights[N / 2] = 2.0 / (N * (N + 1.0) * LN * LN);
        }
    }
    // Kopriva Alg. 30 (BarycentricWeights)
    b.wbary.assign(n, 1.0);
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k)
            if (k != j) b.wbary[j] *= (b.nodes[j] - b.nodes[k]);
    for (int j = 0; j < n; ++j) b.wbary[j] = 1.0 / b.wbary[j];
    // Kopriva Alg. 37 (PolynomialDerivativeMatrix), the form Trixi's polynomial_derivative_matrix uses
    b.D.assign(n * n, 0.0);
    for (int a = 0; a < n; ++a)
        for (int c = 0; c < n; ++c)
            if (c != a) {
                b.D[a * n + c] = b.wbary[c] / b.wbary[a] / (b.nodes[a] - b.nodes[c]);
                b.D[a * n + a] -= b.D[a * n + c];
            }
    // Trixi calc_dhat: dhat = D^T, then dhat[j, m] *= -w[m] / w[j]
    b.Dhat.assign(n * n, 0.0);
    for (int a = 0; a < n; ++a)
        for (int c = 0; c < n; ++c) b.Dhat[a * n + c] = -b.D[c * n + a] * b.weights[c] / b.weights[a];
    b.inv_w_first = 1.0 / b.weights[0];
    b.inv_w_last = 1.0 / b.weights[n - 1];
    mortar_operators(b);
    return b;
}

// ------------------------------------------------------------------------------------------------
// Compressible Euler 2D pointwise functions (Trixi.jl CompressibleEulerEquations2D, restated).
// ------------------------------------------------------------------------------------------------
struct Euler {
    double gamma = 1.4;

    // Trixi flux(u, orientation, eq); the pair is TrixiLW `fluxes` (src/solvers/dgsem_tree/dg_2d.jl:368)
    inline void fluxes(const double* u, double* f, double* g) const {
        const double rho = u[0], m1 = u[1], m2 = u[2], e = u[3];
        const double v1 = m1 / rho, v2 = m2 / rho;
        const double p = (gamma - 1.0) * (e - 0.5 * (m1 * v1 + m2 * v2));
        f[0] = m1; f[1] = m1 * v1 + p; f[2] = m1 * v2; f[3] = (e + p) * v1;
        g[0] = m2; g[1] = m2 * v1; g[2] = m2 * v2 + p; g[3] = (e + p) * v2;
    }
    inline void flux(const double* u, int orientation, double* f) const {
        double fx[NV], gy[NV];
        fluxes(u, fx, gy);
        for (int v = 0; v < NV; ++v) f[v] = orientation == 1 ? fx[v] : gy[v];
    }
    // Trixi cons2prim
    inline void cons2prim(const double* u, double& rho, double& v1, double& v2, double& p) const {
        rho = u[0]; v1 = u[1] / rho; v2 = u[2] / rho;
        p = (gamma - 1.0) * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    }
    // Julia's sqrt throws DomainError for a negative argument; the oracle reports it through `bad`.
    inline double checked_sqrt(double x, bool& bad) const {
        if (!(x >= 0.0)) { bad = true; return std::numeric_limits<double>::quiet_NaN(); }
        return std::sqrt(x);
    }
    // Trixi max_abs_speed_naive (speed_kind 0) and max_abs_speed (speed_kind 1), orientation 1|2
    inline double max_abs_speed(const double* ul, const double* ur, int orientation, int speed_kind,
                                bool& bad) const {
        double rl, v1l, v2l, pl, rr, v1r, v2r, pr;
        cons2prim(ul, rl, v1l, v2l, pl);
        cons2prim(ur, rr, v1r, v2r, pr);
        const double vl = orientation == 1 ? v1l : v2l;
        const double vr = orientation == 1 ? v1r : v2r;
        const double cl = checked_sqrt(gamma * pl / rl, bad);
        const double cr = checked_sqrt(gamma * pr / rr, bad);
        if (speed_kind == 0) return std::max(std::fabs(vl), std::fabs(vr)) + std::max(cl, cr);
        return std::max(std::fabs(vl) + cl, std::fabs(vr) + cr);
    }
    // Trixi min_max_speed_naive (the FluxHLL default)
    inline void min_max_speed(const double* ul, const double* ur, int orientation, double& lmin, double& lmax,
                              bool& bad) const {
        double rl, v1l, v2l, pl, rr, v1r, v2r, pr;
        cons2prim(ul, rl, v1l, v2l, pl);
        cons2prim(ur, rr, v1r, v2r, pr);
        const double vl = orientation == 1 ? v1l : v2l;
        const double vr = orientation == 1 ? v1r : v2r;
        const double cl = checked_sqrt(gamma * pl / rl, bad);
        const double cr = checked_sqrt(gamma * pr / rr, bad);
        lmin = vl - cl;
        lmax = vr + cr;
    }
    // Trixi max_abs_speeds (used by max_dt)
    inline void max_abs_speeds(const double* u, double& l1, double& l2, bool& bad) const {
        double rho, v1, v2, p;
        cons2prim(u, rho, v1, v2, p);
        const double c = checked_sqrt(gamma * p / rho, bad);
        l1 = std::fabs(v1) + c;
        l2 = std::fabs(v2) + c;
    }
    // src/equations/compressible_euler_2d.jl:4-7
    inline bool is_admissible(const double* u) const {
        double rho, v1, v2, p;
        cons2prim(u, rho, v1, v2, p);
        return rho > 0.0 && p > 0.0;
    }
};

// 8-argument LW surface flux as called on TreeMesh: surface_flux(f_ll, f_rr, U_ll, U_rr, u_ll, u_rr, ...)
// (src/solvers/dgsem_tree/dg_2d.jl:1928). For FluxPlusDissipation (src/equations/numerical_fluxes.jl:14-22)
// the third/fourth arguments feed the speed estimate and the fifth/sixth the jump
// (DissipationLocalLaxFriedrichs, numerical_fluxes.jl:34-38), so on TreeMesh lambda comes from the
// time-averaged U and the jump is in the instantaneous u. flux_central is numerical_fluxes.jl:7-12.
// For FluxHLL (src/equations/compressible_euler_2d.jl:24-40) the argument names are (f, f, U, U, u, u):
// the speeds come from the fifth/sixth arguments and the jump from the third/fourth.
enum SurfaceFlux { RUSANOV = 0, HLL = 1 };

inline void lw_surface_flux(const Euler& eq, int flux_kind, int speed_kind, const double* f_ll, const double* f_rr,
                            const double* a3, const double* a4, const double* a5, const double* a6,
                            int orientation, double* out, bool& bad) {
    if (flux_kind == RUSANOV) {
        // FluxPlusDissipation(f_ll, f_rr, u_ll=a3, u_rr=a4, U_ll=a5, U_rr=a6)
        const double lambda = eq.max_abs_speed(a3, a4, orientation, speed_kind, bad);
        for (int v = 0; v < NV; ++v) out[v] = 0.5 * (f_ll[v] + f_rr[v]) + (-0.5 * lambda * (a6[v] - a5[v]));
    } else {
        // FluxHLL(f_ll, f_rr, U_ll=a3, U_rr=a4, u_ll=a5, u_rr=a6)
        double lmin, lmax;
        eq.min_max_speed(a5, a6, orientation, lmin, lmax, bad);
        if (lmin >= 0 && lmax >= 0) {
            for (int v = 0; v < NV; ++v) out[v] = f_ll[v];
        } else if (lmax <= 0 && lmin <= 0) {
            for (int v = 0; v < NV; ++v) out[v] = f_rr[v];
        } else {
            const double inv = 1.0 / (lmax - lmin);
            const double fll = lmax * inv, frr = lmin * inv, fd = lmin * lmax * inv;
            for (int v = 0; v < NV; ++v) out[v] = fll * f_ll[v] - frr * f_rr[v] + fd * (a4[v] - a3[v]);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// TreeMesh connectivity and LW caches (src/solvers/dgsem_tree/containers.jl:73-121, 216-237).
// ------------------------------------------------------------------------------------------------
struct TreeMesh {
    int n_elements = 0;
    std::vector<double> inverse_jacobian;      // [E]
    int n_interfaces = 0;
    std::vector<int32_t> interface_left, interface_right, interface_orientation;   // 0-based ids, 1|2
    // boundaries (src/solvers/dgsem_tree/dg_2d.jl:1328-1454); neighbor_side 1: element on the -side
    int n_boundaries = 0;
    std::vector<int32_t> boundary_element, boundary_orientation, boundary_side, boundary_direction;
    // condition per boundary (empty: all Dirichlet): BC_DIRICHLET, BC_SLIP_WALL_VERTICAL, BC_SLIP_WALL_HORIZONTAL
    std::vector<int32_t> boundary_kind;
    // L2 mortars (Trixi mortars container): lower / upper small element, large element (0-based),
    // large_sides 1: large element on the -side, 2: on the +side; orientation 1 (x) / 2 (y)
    int n_mortars = 0;
    std::vector<int32_t> mortar_lower, mortar_upper, mortar_large, mortar_large_side, mortar_orientation;
};

struct Options {
    int N = 4;
    int flux_kind = RUSANOV;
    int speed_kind = 0;            // 0 = max_abs_speed_naive
    bool temporal_errors = false;  // lw_volume_kernel_4! u_np1/u_np1_low tail (dg_2d.jl:1251-1265)
    double abstol = 0.0, reltol = 0.0;
    // VolumeIntegralFRShockCapturing(IndicatorHennemannGassner(...; variable = density_pressure),
    // volume_flux_fv = flux_lax_friedrichs, reconstruction = FirstOrderReconstruction())
    bool shock_capturing = false;
    double alpha_max = 0.5, alpha_min = 0.001;
    bool alpha_smooth = true;
    int reconstruction = 0;        // curvilinear meshes: 0 FirstOrderReconstruction, 1 MUSCLReconstruction
    // source terms (SemidiscretizationHyperbolic(...; source_terms)): 0 none, 1 Trixi's
    // source_terms_convergence_test; node coordinates [2, i, j, e] (Trixi's cache.elements.node_coordinates)
    int source = 0;
    const double* xnode = nullptr;
};

// Trixi's source_terms_convergence_test for CompressibleEulerEquations2D: the source that makes the manufactured
// solution rho = rho v1 = rho v2 = c + A sin(w (x + y - t)), rho e = rho^2 (c = 2, A = 0.1, L = 2, w = 2 pi / L,
// initial_condition_convergence_test) exact. With rho' = w A cos(w (x + y - t)) (d/dt rho = -d/dx rho = -d/dy rho)
// and p' = (gamma - 1)(2 rho - 1) rho': (rho', rho' (1 + tmp), rho' (1 + tmp), 2 rho' (rho + tmp)), tmp = (2 rho - 1)
// (gamma - 1). It does not depend on u.
inline void source_convergence_test(double gamma, double x1, double x2, double t, double* s) {
    const double c = 2.0, A = 0.1, L = 2.0, f = 1.0 / L, w = 2.0 * 3.14159265358979323846 * f;
    const double si = std::sin(w * (x1 + x2 - t)), co = std::cos(w * (x1 + x2 - t));
    const double rho = c + A * si;
    const double rho_x = w * A * co;
    const double tmp = (2.0 * rho - 1.0) * (gamma - 1.0);
    s[0] = rho_x;
    s[1] = rho_x * (1.0 + tmp);
    s[2] = s[1];
    s[3] = 2.0 * rho_x * (rho + tmp);
}
inline void source_eval(int kind, double gamma, const double* /*u*/, double x1, double x2, double t, double* s) {
    if (kind == 1) source_convergence_test(gamma, x1, x2, t, s);
    else s[0] = s[1] = s[2] = s[3] = 0.0;
}
// c * sum_k w[k] s(x, t + (k - 2) dt), k = 0..4: a stencil of a source that does not depend on u (the only kind
// built), for which the states of the reference's calls do not matter
inline void source_stencil_t(int kind, double gamma, double x1, double x2, double t, double dt, double c,
                             const double (&w)[5], double* o) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0}, sv[4];
    for (int k = 0; k < 5; ++k) {
        if (w[k] == 0.0) continue;
        source_eval(kind, gamma, nullptr, x1, x2, t + (k - 2) * dt, sv);
        for (int v = 0; v < 4; ++v) acc[v] += w[k] * sv[v];
    }
    for (int v = 0; v < 4; ++v) o[v] = c * acc[v];
}

struct Workspace {
    // element cache
    std::vector<double> U, F;            // [v,i,j,e], [v,d,i,j,e]
    std::vector<double> U2, F2, us;      // MDRK cache (containers.jl:83-98)
    std::vector<double> S2;              // MDRK stage 1's source S2 = s + st/6 [v,i,j,e] (source terms only)
    std::vector<double> temporal_errors; // [E]
    // interface cache [side, v, i, I]
    std::vector<double> iu, iU, iF;
    std::vector<double> surface_flux_values;  // [v, i, face, e], face 0..3 = -x, +x, -y, +y
    // boundary cache [side, v, i, B] and exterior time-averaged states supplied per call
    std::vector<double> bu, bU, bF;
    std::vector<double> alpha;           // blending factor per element (shock capturing)
    std::vector<double> fn_low;          // [v, l, face, e] first-order subcell flux next to each face
    // small-mortar nodes of the last curvilinear shock-capturing rhs at which zhang_shu_flux_fix changed the
    // blended flux: [0] the small element's side, [1] the large element's side
    std::vector<double> mortar_fixes = std::vector<double>(2, 0.0);
    bool bad = false;                    // a sqrt of a negative number happened (Julia DomainError)
};

inline size_t idx_u(int n, int v, int i, int j, int e) { return v + NV * (i + (size_t)n * (j + (size_t)n * e)); }
inline size_t idx_F(int n, int v, int d, int i, int j, int e) {
    return v + NV * (d + 2 * (i + (size_t)n * (j + (size_t)n * e)));
}

// ------------------------------------------------------------------------------------------------
// LW volume kernel for one element: lw_volume_kernel_{1,2,3,4}! (TreeMesh, no source terms).
//   depth 4: src/solvers/dgsem_tree/dg_2d.jl:918-1267 (every polydeg >= 4, dispatch :179-218)
//   depth 3: dg_2d.jl:674-916
//   depth 2: dg_2d.jl:495-672 (as written; the shipped dispatcher cannot call it, see the header)
//   depth 1: dg_2d.jl:370-493
// Every time derivative is carried pre-multiplied by dt^k, so the stencils are evaluated at unit step.
// du receives alpha * (Dhat F + Dhat G) (before surface integral and Jacobian); U/F are stored in ws.
// ------------------------------------------------------------------------------------------------
inline void lw_volume_element(const Basis& b, const Euler& eq, const Options& opt, int e, const double* u,
                              double* du, double dt, double inv_jac, double alpha, Workspace& ws, double t = 0.0) {
    const int n = b.n;
    const int nn = n * n;
    const int depth = std::min(opt.N, 4);
    Tile f, g, Fc, Gc, Uc, up, um, upp, umm, ut, utt, uttt, utttt, unp1, unp1_low, S;
    ut.zero(NV * nn); utt.zero(NV * nn); uttt.zero(NV * nn); utttt.zero(NV * nn); S.zero(NV * nn);
    auto L = [&](int i, int j) { return NV * (i + n * j); };
    const double* ue = u + idx_u(n, 0, 0, 0, e);
    // source terms: s(u_, dtau) = source_terms(u_, x, t + dtau) at node (i, j) (dg_2d.jl:89-175); the stencils
    // calc_source_t_N12 / _t_N34 / _tt_N23 / _ttt_N34 / _tttt_N4 as the reference defines them
    auto src = [&](const double* us, int i, int j, double dtau, double* o) {
        const double* xn = opt.xnode + 2 * ((size_t)e * nn + i + (size_t)n * j);
        source_eval(opt.source, eq.gamma, us, xn[0], xn[1], t + dtau, o);
    };
    auto st_N12 = [&](const double* up_, const double* um_, int i, int j, double* o) {
        double a[NV], c[NV];
        src(up_, i, j, dt, a);
        src(um_, i, j, -dt, c);
        for (int v = 0; v < NV; ++v) o[v] = 0.5 * (a[v] - c[v]);
    };
    auto st_N34 = [&](const double* up_, const double* upp_, const double* um_, const double* umm_, int i, int j,
                      double* o) {
        double a[NV], c[NV], d[NV], h[NV];
        src(upp_, i, j, 2.0 * dt, a);
        src(up_, i, j, dt, c);
        src(um_, i, j, -dt, d);
        src(umm_, i, j, -2.0 * dt, h);
        for (int v = 0; v < NV; ++v) o[v] = (1.0 / 12.0) * (-a[v] + 8.0 * c[v] - 8.0 * d[v] + h[v]);
    };
    auto stt_N23 = [&](const double* u_, const double* up_, const double* um_, int i, int j, double* o) {
        double a[NV], c[NV], d[NV];
        src(up_, i, j, dt, a);
        src(u_, i, j, 0.0, c);
        src(um_, i, j, -dt, d);
        for (int v = 0; v < NV; ++v) o[v] = a[v] - 2.0 * c[v] + d[v];
    };
    auto sttt_N34 = [&](const double* up_, const double* upp_, const double* um_, const double* umm_, int i, int j,
                        double* o) {
        double a[NV], c[NV], d[NV], h[NV];
        src(upp_, i, j, 2.0 * dt, a);
        src(up_, i, j, dt, c);
        src(um_, i, j, -dt, d);
        src(umm_, i, j, -2.0 * dt, h);
        for (int v = 0; v < NV; ++v) o[v] = 0.5 * (a[v] - 2.0 * c[v] + 2.0 * d[v] - h[v]);
    };
    auto stttt_N4 = [&](const double* u_, const double* up_, const double* upp_, const double* um_,
                        const double* umm_, int i, int j, double* o) {
        double a[NV], c[NV], d[NV], h[NV], k[NV];
        src(upp_, i, j, 2.0 * dt, a);
        src(up_, i, j, dt, c);
        src(u_, i, j, 0.0, d);
        src(um_, i, j, -dt, h);
        src(umm_, i, j, -2.0 * dt, k);
        for (int v = 0; v < NV; ++v) o[v] = a[v] - 4.0 * c[v] + 6.0 * d[v] - 4.0 * h[v] + k[v];
    };
    // add (factor S, factor of the derivative) * stencil at every node; states read before this stage's update
    auto add_source = [&](Tile& deriv, double cS, auto&& stencil) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double st[NV];
                stencil(o, i, j, st);
                for (int v = 0; v < NV; ++v) {
                    S[o + v] += cS * st[v];
                    deriv[o + v] += dt * st[v];
                }
            }
    };

    // contraction target += -dt * D (x: along i, y: along j), scatter form as in the reference loops
    auto contract = [&](const Tile& fx, const Tile& gy, Tile& tgt) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                for (int ii = 0; ii < n; ++ii) {
                    const double c = -dt * b.D[ii * n + i];
                    for (int v = 0; v < NV; ++v) tgt[L(ii, j) + v] += c * fx[L(i, j) + v];
                }
                for (int jj = 0; jj < n; ++jj) {
                    const double c = -dt * b.D[jj * n + j];
                    for (int v = 0; v < NV; ++v) tgt[L(i, jj) + v] += c * gy[L(i, j) + v];
                }
            }
        for (int k = 0; k < NV * nn; ++k) tgt[k] *= inv_jac;
    };
    auto fl = [&](const Tile& s, int i, int j, double* fo, double* go) { eq.fluxes(&s[L(i, j)], fo, go); };

    // stage 0: f, g at u; ut (dg_2d.jl:941-978)
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const double* un = ue + L(i, j);
            eq.fluxes(un, &f[L(i, j)], &g[L(i, j)]);
            for (int v = 0; v < NV; ++v) {
                Fc[L(i, j) + v] = f[L(i, j) + v];
                Gc[L(i, j) + v] = g[L(i, j) + v];
                up[L(i, j) + v] = um[L(i, j) + v] = upp[L(i, j) + v] = umm[L(i, j) + v] = un[v];
                Uc[L(i, j) + v] = un[v];
                unp1[L(i, j) + v] = unp1_low[L(i, j) + v] = un[v];
            }
        }
    if (depth == 2) {
        // kernel_2 scales after a plain D contraction (dg_2d.jl:526-549); same value as -dt*D then J
        Tile tmp;
        tmp.zero(NV * nn);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                for (int ii = 0; ii < n; ++ii)
                    for (int v = 0; v < NV; ++v) tmp[L(ii, j) + v] += b.D[ii * n + i] * f[L(i, j) + v];
                for (int jj = 0; jj < n; ++jj)
                    for (int v = 0; v < NV; ++v) tmp[L(i, jj) + v] += b.D[jj * n + j] * g[L(i, j) + v];
            }
        for (int k = 0; k < NV * nn; ++k) ut[k] = tmp[k] * (-dt * inv_jac);
    } else {
        contract(f, g, ut);
    }
    if (opt.source) {
        // S = s(u, x, t); ut += dt s (dg_2d.jl:979-987 and the same lines of kernels 1-3)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double s0[NV];
                src(ue + o, i, j, 0.0, s0);
                for (int v = 0; v < NV; ++v) {
                    S[o + v] = s0[v];
                    ut[o + v] += dt * s0[v];
                }
            }
    }

    double fp[NV], gp[NV], fm[NV], gm[NV], fpp[NV], gpp[NV], fmm[NV], gmm[NV];
    Tile ft, gt;

    // stage 1 (dg_2d.jl:990-1023 for depth 3/4; :435-456 / :561-595 for depth 1/2)
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            for (int v = 0; v < NV; ++v) {
                const double d = ut[o + v];
                Uc[o + v] += 0.5 * d;
                up[o + v] += d;
                um[o + v] += -d;
                if (depth >= 3) { umm[o + v] += -2.0 * d; upp[o + v] += 2.0 * d; }
            }
            fl(um, i, j, fm, gm);
            fl(up, i, j, fp, gp);
            if (depth >= 3) {
                fl(umm, i, j, fmm, gmm);
                fl(upp, i, j, fpp, gpp);
                for (int v = 0; v < NV; ++v) {
                    ft[o + v] = 1.0 / 12.0 * (-fpp[v] + 8.0 * fp[v] - 8.0 * fm[v] + fmm[v]);
                    gt[o + v] = 1.0 / 12.0 * (-gpp[v] + 8.0 * gp[v] - 8.0 * gm[v] + gmm[v]);
                }
            } else {
                for (int v = 0; v < NV; ++v) {
                    ft[o + v] = 0.5 * fp[v] - 0.5 * fm[v];
                    gt[o + v] = 0.5 * gp[v] - 0.5 * gm[v];
                }
            }
            for (int v = 0; v < NV; ++v) { Fc[o + v] += 0.5 * ft[o + v]; Gc[o + v] += 0.5 * gt[o + v]; }
        }
    if (depth >= 2) {
        contract(ft, gt, utt);
        if (opt.source) {
            // st from the states after ut: N34 at depths 3, 4 (dg_2d.jl:1027-1040, :785-799), N12 at depth 2 (:605-615)
            add_source(utt, 0.5, [&](int o, int i, int j, double* st) {
                if (depth >= 3) st_N34(&up[o], &upp[o], &um[o], &umm[o], i, j, st);
                else st_N12(&up[o], &um[o], i, j, st);
            });
        }
        // stage 2 (dg_2d.jl:1049-1083 depth 4; :801-831 depth 3; :617-634 depth 2)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                for (int v = 0; v < NV; ++v) {
                    const double d = utt[o + v];
                    Uc[o + v] += 1.0 / 6.0 * d;
                    up[o + v] += 0.5 * d;
                    um[o + v] += 0.5 * d;
                    if (depth >= 3) { upp[o + v] += 2.0 * d; umm[o + v] += 2.0 * d; }
                }
                if (depth == 4) {
                    fl(um, i, j, fm, gm);
                    fl(up, i, j, fp, gp);
                    fl(umm, i, j, fmm, gmm);
                    fl(upp, i, j, fpp, gpp);
                    for (int v = 0; v < NV; ++v) {
                        ft[o + v] = (1.0 / 12.0) * (-fpp[v] + 16.0 * fp[v] - 30.0 * f[o + v] + 16.0 * fm[v] - fmm[v]);
                        gt[o + v] = (1.0 / 12.0) * (-gpp[v] + 16.0 * gp[v] - 30.0 * g[o + v] + 16.0 * gm[v] - gmm[v]);
                    }
                } else {
                    fl(um, i, j, fm, gm);
                    fl(up, i, j, fp, gp);
                    for (int v = 0; v < NV; ++v) {
                        ft[o + v] = fp[v] - 2.0 * f[o + v] + fm[v];
                        gt[o + v] = gp[v] - 2.0 * g[o + v] + gm[v];
                    }
                }
                for (int v = 0; v < NV; ++v) {
                    Fc[o + v] += 1.0 / 6.0 * ft[o + v];
                    Gc[o + v] += 1.0 / 6.0 * gt[o + v];
                }
            }
    }
    if (depth >= 3) {
        contract(ft, gt, uttt);
        if (opt.source) {
            // stt = calc_source_tt_N23 from the states after utt, at depth 4 as well (dg_2d.jl:1093-1104, :841-852)
            add_source(uttt, 1.0 / 6.0, [&](int o, int i, int j, double* st) { stt_N23(ue + o, &up[o], &um[o], i, j, st); });
        }
        // stage 3 (dg_2d.jl:1106-1138 depth 4; :854-875 depth 3)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                for (int v = 0; v < NV; ++v) {
                    const double d = uttt[o + v];
                    Uc[o + v] += 1.0 / 24.0 * d;
                    um[o + v] += -1.0 / 6.0 * d;
                    up[o + v] += 1.0 / 6.0 * d;
                    umm[o + v] += -4.0 / 3.0 * d;
                    upp[o + v] += 4.0 / 3.0 * d;
                }
                fl(um, i, j, fm, gm);
                fl(up, i, j, fp, gp);
                fl(umm, i, j, fmm, gmm);
                fl(upp, i, j, fpp, gpp);
                for (int v = 0; v < NV; ++v) {
                    ft[o + v] = 0.5 * (fpp[v] - 2.0 * fp[v] + 2.0 * fm[v] - fmm[v]);
                    gt[o + v] = 0.5 * (gpp[v] - 2.0 * gp[v] + 2.0 * gm[v] - gmm[v]);
                    Fc[o + v] += 1.0 / 24.0 * ft[o + v];
                    Gc[o + v] += 1.0 / 24.0 * gt[o + v];
                }
            }
    }
    if (depth >= 4) {
        contract(ft, gt, utttt);
        if (opt.source) {
            // sttt from the states after uttt (dg_2d.jl:1148-1162)
            add_source(utttt, 1.0 / 24.0, [&](int o, int i, int j, double* st) {
                sttt_N34(&up[o], &upp[o], &um[o], &umm[o], i, j, st);
            });
        }
        // stage 4 (dg_2d.jl:1164-1226)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                for (int v = 0; v < NV; ++v) {
                    const double d = utttt[o + v];
                    Uc[o + v] += 1.0 / 120.0 * d;
                    um[o + v] += 1.0 / 24.0 * d;
                    up[o + v] += 1.0 / 24.0 * d;
                    umm[o + v] += 2.0 / 3.0 * d;
                    upp[o + v] += 2.0 / 3.0 * d;
                }
                fl(um, i, j, fm, gm);
                fl(up, i, j, fp, gp);
                fl(umm, i, j, fmm, gmm);
                fl(upp, i, j, fpp, gpp);
                if (opt.temporal_errors) {
                    // u_np1_low uses F, G before the fourth-derivative term (dg_2d.jl:1183-1199)
                    for (int ii = 0; ii < n; ++ii) {
                        const double c = -dt * inv_jac * b.D[ii * n + i];
                        for (int v = 0; v < NV; ++v) unp1_low[L(ii, j) + v] += c * Fc[o + v];
                    }
                    for (int jj = 0; jj < n; ++jj) {
                        const double c = -dt * inv_jac * b.D[jj * n + j];
                        for (int v = 0; v < NV; ++v) unp1_low[L(i, jj) + v] += c * Gc[o + v];
                    }
                }
                for (int v = 0; v < NV; ++v) {
                    const double ftttt = 0.5 * (fpp[v] - 4.0 * fp[v] + 6.0 * f[o + v] - 4.0 * fm[v] + fmm[v]);
                    const double gtttt = 0.5 * (gpp[v] - 4.0 * gp[v] + 6.0 * g[o + v] - 4.0 * gm[v] + gmm[v]);
                    Fc[o + v] += 1.0 / 120.0 * ftttt;
                    Gc[o + v] += 1.0 / 120.0 * gtttt;
                }
                if (opt.temporal_errors) {
                    for (int ii = 0; ii < n; ++ii) {
                        const double c = -dt * inv_jac * b.D[ii * n + i];
                        for (int v = 0; v < NV; ++v) unp1[L(ii, j) + v] += c * Fc[o + v];
                    }
                    for (int jj = 0; jj < n; ++jj) {
                        const double c = -dt * inv_jac * b.D[jj * n + j];
                        for (int v = 0; v < NV; ++v) unp1[L(i, jj) + v] += c * Gc[o + v];
                    }
                }
            }
    }
    if (opt.source) {
        // the last stencil, from the states after the last derivative (the reference's argument lists as written):
        //   depth 1: S += st_N12(up, um) / 2                         (dg_2d.jl:474-477)
        //   depth 2: S += stt_N23(u, up, um) / 6                      (:651-654)
        //   depth 3: S += sttt_N34(u, up, upp, upp, umm) / 24, i.e. upp in um's place (:891-897)
        //   depth 4: S += stttt_N4(u, up, um, upp, umm) / 120 into (u, up, upp, um, umm): um and upp swap (:1227-1233)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double st[NV];
                double c;
                if (depth == 1) { st_N12(&up[o], &um[o], i, j, st); c = 0.5; }
                else if (depth == 2) { stt_N23(ue + o, &up[o], &um[o], i, j, st); c = 1.0 / 6.0; }
                else if (depth == 3) { sttt_N34(&up[o], &upp[o], &upp[o], &umm[o], i, j, st); c = 1.0 / 24.0; }
                else { stttt_N4(ue + o, &up[o], &um[o], &upp[o], &umm[o], i, j, st); c = 1.0 / 120.0; }
                for (int v = 0; v < NV; ++v) S[o + v] += c * st[v];
            }
    }
    // final: du += alpha * Dhat (F, G); store U and F (dg_2d.jl:1208-1248, :876-912)
    double* due = du + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            for (int ii = 0; ii < n; ++ii) {
                const double c = alpha * b.Dhat[ii * n + i];
                for (int v = 0; v < NV; ++v) due[L(ii, j) + v] += c * Fc[o + v];
            }
            for (int jj = 0; jj < n; ++jj) {
                const double c = alpha * b.Dhat[jj * n + j];
                for (int v = 0; v < NV; ++v) due[L(i, jj) + v] += c * Gc[o + v];
            }
            for (int v = 0; v < NV; ++v) {
                ws.F[idx_F(n, v, 0, i, j, e)] = Fc[o + v];
                ws.F[idx_F(n, v, 1, i, j, e)] = Gc[o + v];
                ws.U[idx_u(n, v, i, j, e)] = Uc[o + v];
            }
            // du += -S / J^{-1} (apply_jacobian! multiplies by -J^{-1}: the source enters du unscaled)
            if (opt.source)
                for (int v = 0; v < NV; ++v) due[o + v] += (-1.0 / inv_jac) * S[o + v];
        }
    if (opt.temporal_errors && depth >= 4) {
        // dg_2d.jl:1251-1265
        double te = 0.0;
        for (int k = 0; k < NV * nn; ++k) {
            const double r = (unp1[k] - unp1_low[k]) /
                             (opt.abstol + opt.reltol * std::max(std::fabs(unp1[k]), std::fabs(unp1_low[k])));
            te += r * r;
        }
        ws.temporal_errors[e] = te;
    }
}

// ------------------------------------------------------------------------------------------------
// MDRK stage kernels on TreeMesh (src/solvers/dgsem_tree/multi_derivative_2d.jl:263-421, 423-555),
// no source terms. Stage 1 as shipped unpacks `u_low` from a cache that has no such field (:287); the
// value is write-only on this path (it never reaches du, U, F, U2 or F2), so it is not computed here.
// ------------------------------------------------------------------------------------------------
// On a curvilinear mesh (Jae = the element's contravariant vectors [4, i, j], ije = its inverse Jacobian per
// node; mdrk_kernel_1! / _2! of src/solvers/dgsem_structured/multi_derivative_2d.jl:82-445) the contractions
// take the contravariant fluxes and ut carries the node's J^{-1}; F, F2 stay physical.
inline void mdrk_contra(const double* Jae, int n, int i, int j, const double* f, const double* g, double* cf, double* cg) {
    if (!Jae) {
        for (int v = 0; v < NV; ++v) { cf[v] = f[v]; cg[v] = g[v]; }
        return;
    }
    const double* J = Jae + 4 * (i + n * j);
    for (int v = 0; v < NV; ++v) {
        cf[v] = J[0] * f[v] + J[1] * g[v];
        cg[v] = J[2] * f[v] + J[3] * g[v];
    }
}

// source terms of the MDRK stages (TreeMesh): kind, node coordinates, gamma and the rhs call's t
struct SourceArgs {
    int kind = 0;
    const double* xnode = nullptr;
    double gamma = 1.4, t = 0.0;
    bool stage2_at_t = false;   // curvilinear meshes: stage 2's source at t, not t + dt/2
    // s(u_, x, t0 + dtau) at node (i, j) of element e
    void at(int e, int n, int i, int j, const double* us, double t0, double dtau, double* o) const {
        const double* xn = xnode + 2 * ((size_t)e * n * n + i + (size_t)n * j);
        source_eval(kind, gamma, us, xn[0], xn[1], t0 + dtau, o);
    }
    // calc_source_t_N34 (dg_2d.jl:108-116) at time t0
    void t_N34(int e, int n, int i, int j, const double* up, const double* upp, const double* um, const double* umm,
               double t0, double dt, double* o) const {
        double a[NV], c[NV], d[NV], h[NV];
        at(e, n, i, j, upp, t0, 2.0 * dt, a);
        at(e, n, i, j, up, t0, dt, c);
        at(e, n, i, j, um, t0, -dt, d);
        at(e, n, i, j, umm, t0, -2.0 * dt, h);
        for (int v = 0; v < NV; ++v) o[v] = (1.0 / 12.0) * (-a[v] + 8.0 * c[v] - 8.0 * d[v] + h[v]);
    }
};

// Stage 1 with source terms (multi_derivative_2d.jl:321-400): S = s/2 + st/8 enters du, S2 = s + st/6 is kept
// for stage 2 (ws.S2); ut += dt s before the perturbed states.
inline void mdrk1_volume_element(const Basis& b, const Euler& eq, int e, const double* u, double* du, double dt,
                                 double inv_jac, double alpha, Workspace& ws, const double* Jae = nullptr,
                                 const double* ije = nullptr, const SourceArgs* src = nullptr) {
    const int n = b.n, nn = n * n;
    Tile Fh, Gh, F2, G2, Uh, U2, ut, f, g, Sh, S2;
    ut.zero(NV * nn);
    const bool with_src = src && src->kind;
    auto L = [&](int i, int j) { return NV * (i + n * j); };
    const double* ue = u + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            eq.fluxes(ue + o, &f[o], &g[o]);
            for (int v = 0; v < NV; ++v) {
                Fh[o + v] = 0.5 * f[o + v];
                F2[o + v] = f[o + v];
                Gh[o + v] = 0.5 * g[o + v];
                G2[o + v] = g[o + v];
                Uh[o + v] = 0.5 * ue[o + v];
                U2[o + v] = ue[o + v];
            }
            double cf[NV], cg[NV];
            mdrk_contra(Jae, n, i, j, &f[o], &g[o], cf, cg);
            for (int ii = 0; ii < n; ++ii) {
                const double c = -dt * b.D[ii * n + i];
                for (int v = 0; v < NV; ++v) ut[L(ii, j) + v] += c * cf[v];
            }
            for (int jj = 0; jj < n; ++jj) {
                const double c = -dt * b.D[jj * n + j];
                for (int v = 0; v < NV; ++v) ut[L(i, jj) + v] += c * cg[v];
            }
        }
    for (int k = 0; k < NV * nn; ++k) ut[k] *= Jae ? ije[k / NV] : inv_jac;
    if (with_src)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double s0[NV];
                src->at(e, n, i, j, ue + o, src->t, 0.0, s0);
                for (int v = 0; v < NV; ++v) {
                    Sh[o + v] = 0.5 * s0[v];
                    S2[o + v] = s0[v];
                    ut[o + v] += dt * s0[v];
                }
            }
    double* due = du + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            double um[NV], up[NV], umm[NV], upp[NV];
            for (int v = 0; v < NV; ++v) {
                um[v] = ue[o + v] - ut[o + v];
                up[v] = ue[o + v] + ut[o + v];
                umm[v] = ue[o + v] - 2 * ut[o + v];
                upp[v] = ue[o + v] + 2 * ut[o + v];
            }
            if (with_src) {
                double st[NV];
                src->t_N34(e, n, i, j, up, upp, um, umm, src->t, dt, st);
                const double ijn = Jae ? ije[i + n * j] : inv_jac;
                for (int v = 0; v < NV; ++v) {
                    Sh[o + v] += 0.125 * st[v];
                    S2[o + v] += 1.0 / 6.0 * st[v];
                    due[o + v] += (-1.0 / ijn) * Sh[o + v];
                    ws.S2[idx_u(n, v, i, j, e)] = S2[o + v];
                }
            }
            double fm[NV], gm[NV], fp[NV], gp[NV], fmm[NV], gmm[NV], fpp[NV], gpp[NV];
            eq.fluxes(um, fm, gm);
            eq.fluxes(up, fp, gp);
            eq.fluxes(umm, fmm, gmm);
            eq.fluxes(upp, fpp, gpp);
            double ft[NV], gt[NV];
            for (int v = 0; v < NV; ++v) {
                ft[v] = 1.0 / 12.0 * (-fpp[v] + 8.0 * fp[v] - 8.0 * fm[v] + fmm[v]);
                gt[v] = 1.0 / 12.0 * (-gpp[v] + 8.0 * gp[v] - 8.0 * gm[v] + gmm[v]);
                Fh[o + v] += 0.125 * ft[v];
                Gh[o + v] += 0.125 * gt[v];
                Uh[o + v] += 0.125 * ut[o + v];
                F2[o + v] += 1.0 / 6.0 * ft[v];
                G2[o + v] += 1.0 / 6.0 * gt[v];
                U2[o + v] += 1.0 / 6.0 * ut[o + v];
            }
            double cF[NV], cG[NV];
            mdrk_contra(Jae, n, i, j, &Fh[o], &Gh[o], cF, cG);
            for (int ii = 0; ii < n; ++ii) {
                const double c = alpha * b.Dhat[ii * n + i];
                for (int v = 0; v < NV; ++v) due[L(ii, j) + v] += c * cF[v];
            }
            for (int jj = 0; jj < n; ++jj) {
                const double c = alpha * b.Dhat[jj * n + j];
                for (int v = 0; v < NV; ++v) due[L(i, jj) + v] += c * cG[v];
            }
            for (int v = 0; v < NV; ++v) {
                ws.U[idx_u(n, v, i, j, e)] = Uh[o + v];
                ws.F[idx_F(n, v, 0, i, j, e)] = Fh[o + v];
                ws.F[idx_F(n, v, 1, i, j, e)] = Gh[o + v];
                ws.U2[idx_u(n, v, i, j, e)] = U2[o + v];
                ws.F2[idx_F(n, v, 0, i, j, e)] = F2[o + v];
                ws.F2[idx_F(n, v, 1, i, j, e)] = G2[o + v];
            }
        }
}

// Stage 2 with source terms (multi_derivative_2d.jl:484-550): S = S2 + st(u*)/3 at t + dt/2, ust += dt s(u*, t + dt/2).
inline void mdrk2_volume_element(const Basis& b, const Euler& eq, int e, const double* us, double* du, double dt,
                                 double inv_jac, double alpha, Workspace& ws, const double* Jae = nullptr,
                                 const double* ije = nullptr, const SourceArgs* src = nullptr) {
    const int n = b.n, nn = n * n;
    Tile Fc, Gc, Uc, ust;
    ust.zero(NV * nn);
    const bool with_src = src && src->kind;
    const double th = with_src ? (src->stage2_at_t ? src->t : src->t + 0.5 * dt) : 0.0;
    auto L = [&](int i, int j) { return NV * (i + n * j); };
    const double* ue = us + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int v = 0; v < NV; ++v) {
                Fc[L(i, j) + v] = ws.F2[idx_F(n, v, 0, i, j, e)];
                Gc[L(i, j) + v] = ws.F2[idx_F(n, v, 1, i, j, e)];
                Uc[L(i, j) + v] = ws.U2[idx_u(n, v, i, j, e)];
            }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double f[NV], g[NV], cf[NV], cg[NV];
            eq.fluxes(ue + L(i, j), f, g);
            mdrk_contra(Jae, n, i, j, f, g, cf, cg);
            for (int ii = 0; ii < n; ++ii) {
                const double c = -dt * b.D[ii * n + i];
                for (int v = 0; v < NV; ++v) ust[L(ii, j) + v] += c * cf[v];
            }
            for (int jj = 0; jj < n; ++jj) {
                const double c = -dt * b.D[jj * n + j];
                for (int v = 0; v < NV; ++v) ust[L(i, jj) + v] += c * cg[v];
            }
        }
    for (int k = 0; k < NV * nn; ++k) ust[k] *= Jae ? ije[k / NV] : inv_jac;
    if (with_src)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double s0[NV];
                src->at(e, n, i, j, ue + o, th, 0.0, s0);
                for (int v = 0; v < NV; ++v) ust[o + v] += dt * s0[v];
            }
    double* due = du + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            double um[NV], up[NV], umm[NV], upp[NV];
            for (int v = 0; v < NV; ++v) {
                um[v] = ue[o + v] - ust[o + v];
                up[v] = ue[o + v] + ust[o + v];
                umm[v] = ue[o + v] - 2 * ust[o + v];
                upp[v] = ue[o + v] + 2 * ust[o + v];
            }
            if (with_src) {
                double st[NV];
                src->t_N34(e, n, i, j, up, upp, um, umm, th, dt, st);
                const double ijn = Jae ? ije[i + n * j] : inv_jac;
                for (int v = 0; v < NV; ++v)
                    due[o + v] += (-1.0 / ijn) * (ws.S2[idx_u(n, v, i, j, e)] + 1.0 / 3.0 * st[v]);
            }
            double fm[NV], gm[NV], fp[NV], gp[NV], fmm[NV], gmm[NV], fpp[NV], gpp[NV];
            eq.fluxes(um, fm, gm);
            eq.fluxes(up, fp, gp);
            eq.fluxes(umm, fmm, gmm);
            eq.fluxes(upp, fpp, gpp);
            for (int v = 0; v < NV; ++v) {
                const double ft = 1.0 / 12.0 * (-fpp[v] + 8.0 * fp[v] - 8.0 * fm[v] + fmm[v]);
                const double gt = 1.0 / 12.0 * (-gpp[v] + 8.0 * gp[v] - 8.0 * gm[v] + gmm[v]);
                Fc[o + v] += 1.0 / 3.0 * ft;
                Gc[o + v] += 1.0 / 3.0 * gt;
                Uc[o + v] += 1.0 / 3.0 * ust[o + v];
            }
            double cF[NV], cG[NV];
            mdrk_contra(Jae, n, i, j, &Fc[o], &Gc[o], cF, cG);
            for (int ii = 0; ii < n; ++ii) {
                const double c = alpha * b.Dhat[ii * n + i];
                for (int v = 0; v < NV; ++v) due[L(ii, j) + v] += c * cF[v];
            }
            for (int jj = 0; jj < n; ++jj) {
                const double c = alpha * b.Dhat[jj * n + j];
                for (int v = 0; v < NV; ++v) due[L(i, jj) + v] += c * cG[v];
            }
            for (int v = 0; v < NV; ++v) {
                ws.U[idx_u(n, v, i, j, e)] = Uc[o + v];
                ws.F[idx_F(n, v, 0, i, j, e)] = Fc[o + v];
                ws.F[idx_F(n, v, 1, i, j, e)] = Gc[o + v];
            }
        }
}

// ------------------------------------------------------------------------------------------------
// Surface: prolong2interfaces! (dg_2d.jl:1269-1326), calc_interface_flux! (dg_2d.jl:1903-1946, plain FR
// so compute_alp = 0, :1873-1877), Trixi calc_surface_integral! (weak form, boundary_interpolation =
// lhat/w) and apply_jacobian! (du *= -inverse_jacobian).
// ------------------------------------------------------------------------------------------------
inline void prolong2interfaces(const Basis& b, const TreeMesh& m, const double* u, Workspace& ws, int nthreads = 1) {
    const int n = b.n;
    const size_t I = m.n_interfaces;
    ws.iu.assign(2 * NV * n * I, 0.0);
    ws.iU.assign(2 * NV * n * I, 0.0);
    ws.iF.assign(2 * NV * n * I, 0.0);
    auto ii = [&](int side, int v, int l, size_t k) { return side + 2 * (v + NV * (l + (size_t)n * k)); };
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (size_t k = 0; k < I; ++k) {
        const int le = m.interface_left[k], re = m.interface_right[k];
        for (int l = 0; l < n; ++l)
            for (int v = 0; v < NV; ++v) {
                if (m.interface_orientation[k] == 1) {
                    ws.iu[ii(0, v, l, k)] = u[idx_u(n, v, n - 1, l, le)];
                    ws.iu[ii(1, v, l, k)] = u[idx_u(n, v, 0, l, re)];
                    ws.iU[ii(0, v, l, k)] = ws.U[idx_u(n, v, n - 1, l, le)];
                    ws.iU[ii(1, v, l, k)] = ws.U[idx_u(n, v, 0, l, re)];
                    ws.iF[ii(0, v, l, k)] = ws.F[idx_F(n, v, 0, n - 1, l, le)];
                    ws.iF[ii(1, v, l, k)] = ws.F[idx_F(n, v, 0, 0, l, re)];
                } else {
                    ws.iu[ii(0, v, l, k)] = u[idx_u(n, v, l, n - 1, le)];
                    ws.iu[ii(1, v, l, k)] = u[idx_u(n, v, l, 0, re)];
                    ws.iU[ii(0, v, l, k)] = ws.U[idx_u(n, v, l, n - 1, le)];
                    ws.iU[ii(1, v, l, k)] = ws.U[idx_u(n, v, l, 0, re)];
                    ws.iF[ii(0, v, l, k)] = ws.F[idx_F(n, v, 1, l, n - 1, le)];
                    ws.iF[ii(1, v, l, k)] = ws.F[idx_F(n, v, 1, l, 0, re)];
                }
            }
    }
}

inline void calc_interface_flux(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m,
                                Workspace& ws, int nthreads = 1) {
    const int n = b.n;
    auto ii = [&](int side, int v, int l, size_t k) { return side + 2 * (v + NV * (l + (size_t)n * k)); };
    bool bad = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad)
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int le = m.interface_left[k], re = m.interface_right[k];
        const int o = m.interface_orientation[k];
        const int left_dir = 2 * o - 1, right_dir = 2 * o - 2;   // 0-based face of Trixi's 2o / 2o-1
        for (int l = 0; l < n; ++l) {
            double Ul[NV], Ur[NV], ul[NV], ur[NV], fl[NV], fr[NV], Fn[NV];
            for (int v = 0; v < NV; ++v) {
                Ul[v] = ws.iU[ii(0, v, l, k)]; Ur[v] = ws.iU[ii(1, v, l, k)];
                ul[v] = ws.iu[ii(0, v, l, k)]; ur[v] = ws.iu[ii(1, v, l, k)];
                fl[v] = ws.iF[ii(0, v, l, k)]; fr[v] = ws.iF[ii(1, v, l, k)];
            }
            lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, fl, fr, Ul, Ur, ul, ur, o, Fn, bad);
            for (int v = 0; v < NV; ++v) {
                ws.surface_flux_values[v + NV * (l + n * (left_dir + 4 * (size_t)le))] = Fn[v];
                ws.surface_flux_values[v + NV * (l + n * (right_dir + 4 * (size_t)re))] = Fn[v];
            }
        }
    }
    if (bad) ws.bad = true;
}

// Exterior data for time-averaged Dirichlet boundaries (src/equations/equations.jl:6-37): the caller
// supplies, per boundary node, the exterior state at the n Gauss-Lobatto time levels
// ts_k = t + 0.5 dt_scaled (x_k + 1) and at t.
struct BoundaryData {
    const double* u_levels = nullptr;   // [v, k, l, B]  state at time level k
    const double* u_now = nullptr;      // [v, l, B]     state at t
};

enum BoundaryKind { BC_DIRICHLET = 0, BC_SLIP_WALL_VERTICAL = 1, BC_SLIP_WALL_HORIZONTAL = 2 };

inline int boundary_kind(const TreeMesh& m, int k) { return m.boundary_kind.empty() ? BC_DIRICHLET : m.boundary_kind[k]; }

inline bool has_dirichlet_boundaries(const TreeMesh& m) {
    for (int k = 0; k < m.n_boundaries; ++k)
        if (boundary_kind(m, k) == BC_DIRICHLET) return true;
    return false;
}

// Slip walls (boundary_condition_slip_wall_vertical / _horizontal, src/equations/equations.jl:95-135): the
// exterior normal flux, U and u are the inner ones mirrored in the wall's normal momentum.
inline void slip_wall_exterior(int kind, const double* Fi, const double* Ui, const double* ui, double* Fo, double* Uo,
                               double* uo) {
    if (kind == BC_SLIP_WALL_VERTICAL) {
        Fo[0] = -Fi[0]; Fo[1] = Fi[1]; Fo[2] = -Fi[2]; Fo[3] = -Fi[3];
        Uo[0] = Ui[0]; Uo[1] = -Ui[1]; Uo[2] = Ui[2]; Uo[3] = Ui[3];
        uo[0] = ui[0]; uo[1] = -ui[1]; uo[2] = ui[2]; uo[3] = ui[3];
    } else {
        Fo[0] = -Fi[0]; Fo[1] = -Fi[1]; Fo[2] = Fi[2]; Fo[3] = -Fi[3];
        Uo[0] = Ui[0]; Uo[1] = Ui[1]; Uo[2] = -Ui[2]; Uo[3] = Ui[3];
        uo[0] = ui[0]; uo[1] = ui[1]; uo[2] = -ui[2]; uo[3] = ui[3];
    }
}

inline void calc_boundary_flux(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m,
                               const double* u, const BoundaryData& bd, double scaling_factor, Workspace& ws) {
    // prolong2boundaries! (dg_2d.jl:1328-1376) + calc_adv_boundary_flux_by_direction! (:1411-1454)
    const int n = b.n;
    for (int k = 0; k < m.n_boundaries; ++k) {
        const int e = m.boundary_element[k];
        const int o = m.boundary_orientation[k];
        const int side = m.boundary_side[k];
        const int dir = m.boundary_direction[k];   // 1..4 (Trixi direction)
        const int kind = boundary_kind(m, k);
        for (int l = 0; l < n; ++l) {
            double ui[NV], Ui[NV], Fi[NV];
            int i, j;
            if (o == 1) { i = side == 1 ? n - 1 : 0; j = l; } else { i = l; j = side == 1 ? n - 1 : 0; }
            for (int v = 0; v < NV; ++v) {
                ui[v] = u[idx_u(n, v, i, j, e)];
                Ui[v] = ws.U[idx_u(n, v, i, j, e)];
                Fi[v] = ws.F[idx_F(n, v, o - 1, i, j, e)];
            }
            double Uo[NV] = {0, 0, 0, 0}, Fo[NV] = {0, 0, 0, 0}, uo[NV];
            if (kind != BC_DIRICHLET) {
                slip_wall_exterior(kind, Fi, Ui, ui, Fo, Uo, uo);
                double Fn[NV];
                if (dir % 2 == 0)
                    lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, Fi, Fo, Ui, Uo, ui, uo, o, Fn, ws.bad);
                else
                    lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, Fo, Fi, Uo, Ui, uo, ui, o, Fn, ws.bad);
                for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * ((dir - 1) + 4 * (size_t)e))] = Fn[v];
                continue;
            }
            for (int q = 0; q < n; ++q) {
                const double* ub = bd.u_levels + NV * (q + (size_t)n * (l + (size_t)n * k));
                double fb[NV];
                eq.flux(ub, o, fb);
                for (int v = 0; v < NV; ++v) {
                    Uo[v] += 0.5 * scaling_factor * ub[v] * b.weights[q];
                    Fo[v] += 0.5 * scaling_factor * fb[v] * b.weights[q];
                }
            }
            for (int v = 0; v < NV; ++v) uo[v] = bd.u_now[v + NV * (l + (size_t)n * k)];
            double Fn[NV];
            if (dir % 2 == 0)
                lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, Fi, Fo, Ui, Uo, ui, uo, o, Fn, ws.bad);
            else
                lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, Fo, Fi, Uo, Ui, uo, ui, o, Fn, ws.bad);
            for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * ((dir - 1) + 4 * (size_t)e))] = Fn[v];
        }
    }
}

inline void surface_integral_and_jacobian(const Basis& b, const TreeMesh& m, double* du, const Workspace& ws,
                                          int nthreads = 1) {
    const int n = b.n;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e) {
        for (int l = 0; l < n; ++l)
            for (int v = 0; v < NV; ++v) {
                auto sfv = [&](int face) { return ws.surface_flux_values[v + NV * (l + n * (face + 4 * (size_t)e))]; };
                du[idx_u(n, v, 0, l, e)] = du[idx_u(n, v, 0, l, e)] - sfv(0) * b.inv_w_first;
                du[idx_u(n, v, n - 1, l, e)] = du[idx_u(n, v, n - 1, l, e)] + sfv(1) * b.inv_w_last;
                du[idx_u(n, v, l, 0, e)] = du[idx_u(n, v, l, 0, e)] - sfv(2) * b.inv_w_first;
                du[idx_u(n, v, l, n - 1, e)] = du[idx_u(n, v, l, n - 1, e)] + sfv(3) * b.inv_w_last;
            }
        const double factor = -m.inverse_jacobian[e];
        for (int k = 0; k < NV * n * n; ++k) du[idx_u(n, 0, 0, 0, e) + k] *= factor;
    }
}

// L2 mortars on TreeMesh{2} with the LW traces (src/solvers/dgsem_tree/dg_2d.jl:1456-1646):
// prolong2mortars! copies the small elements' u, U, F face traces and interpolates the large element's
// (element_solutions_to_mortars!), calc_fstar! evaluates the surface flux in the TreeMesh argument order on
// both halves, and mortar_fluxes_to_elements! (Trixi) hands fstar to the small faces and its L2 projection
// to the large face.
inline void calc_mortar_flux(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m,
                             const double* u, Workspace& ws, int nthreads = 1) {
    const int n = b.n;
    bool bad = false;
    auto face_node = [&](int f, int l, int& i, int& j) {
        i = f == 0 ? 0 : f == 1 ? n - 1 : l;
        j = f == 2 ? 0 : f == 3 ? n - 1 : l;
    };
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad)
    for (int k = 0; k < m.n_mortars; ++k) {
        const int o = m.mortar_orientation[k];
        const bool large_left = m.mortar_large_side[k] == 1;
        const int small_face = large_left ? (o == 1 ? 0 : 2) : (o == 1 ? 1 : 3);
        const int large_face = large_left ? (o == 1 ? 1 : 3) : (o == 1 ? 0 : 2);
        const int d = o - 1;   // normal flux component
        const int le = m.mortar_large[k];
        std::vector<double> fstar(2 * n * NV);
        for (int h = 0; h < 2; ++h) {
            const int se = h ? m.mortar_upper[k] : m.mortar_lower[k];
            const std::vector<double>& fwd = h ? b.fwd_upper : b.fwd_lower;
            for (int l = 0; l < n; ++l) {
                int is, js;
                face_node(small_face, l, is, js);
                double us[NV], Us[NV], Fs[NV], ul[NV] = {0, 0, 0, 0}, Ul[NV] = {0, 0, 0, 0}, Fl[NV] = {0, 0, 0, 0};
                for (int v = 0; v < NV; ++v) {
                    us[v] = u[idx_u(n, v, is, js, se)];
                    Us[v] = ws.U[idx_u(n, v, is, js, se)];
                    Fs[v] = ws.F[idx_F(n, v, d, is, js, se)];
                }
                for (int jj = 0; jj < n; ++jj) {
                    int il, jl;
                    face_node(large_face, jj, il, jl);
                    const double c = fwd[l * n + jj];
                    for (int v = 0; v < NV; ++v) {
                        ul[v] += c * u[idx_u(n, v, il, jl, le)];
                        Ul[v] += c * ws.U[idx_u(n, v, il, jl, le)];
                        Fl[v] += c * ws.F[idx_F(n, v, d, il, jl, le)];
                    }
                }
                bool b_ = false;
                double* out = &fstar[(h * n + l) * NV];
                if (large_left) lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, Fl, Fs, Ul, Us, ul, us, o, out, b_);
                else lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, Fs, Fl, Us, Ul, us, ul, o, out, b_);
                bad = bad || b_;
                for (int v = 0; v < NV; ++v)
                    ws.surface_flux_values[v + NV * (l + n * (small_face + 4 * (size_t)se))] = out[v];
            }
        }
        for (int mm = 0; mm < n; ++mm)
            for (int v = 0; v < NV; ++v) {
                double acc = 0.0;
                for (int l = 0; l < n; ++l)
                    acc += b.rev_upper[mm * n + l] * fstar[(n + l) * NV + v] + b.rev_lower[mm * n + l] * fstar[l * NV + v];
                ws.surface_flux_values[v + NV * (mm + n * (large_face + 4 * (size_t)le))] = acc;
            }
    }
    if (bad) ws.bad = true;
}

inline void ensure_workspace(const Basis& b, const TreeMesh& m, Workspace& ws, bool mdrk) {
    const size_t nodes = (size_t)b.n * b.n * m.n_elements;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (ws.U.size() != NV * nodes) ws.U.assign(NV * nodes, nan);
    if (ws.F.size() != 2 * NV * nodes) ws.F.assign(2 * NV * nodes, nan);
    if (mdrk) {
        if (ws.U2.size() != NV * nodes) ws.U2.assign(NV * nodes, nan);
        if (ws.F2.size() != 2 * NV * nodes) ws.F2.assign(2 * NV * nodes, nan);
        if (ws.S2.size() != NV * nodes) ws.S2.assign(NV * nodes, nan);
    }
    ws.surface_flux_values.assign((size_t)NV * b.n * 4 * m.n_elements, nan);
    if (ws.temporal_errors.size() != (size_t)m.n_elements) ws.temporal_errors.assign(m.n_elements, nan);
}

// ------------------------------------------------------------------------------------------------
// Shock capturing (VolumeIntegralFRShockCapturing, src/solvers/dgsem_tree/dg_2d.jl:1648-1804).
// ------------------------------------------------------------------------------------------------
// Trixi legendre_polynomial_and_derivative, normalised by sqrt(m + 1/2)
inline double legendre_normalized(int m, double x) {
    double p;
    if (m == 0) p = 1.0;
    else if (m == 1) p = x;
    else {
        double a = 1.0, b = x;
        p = 0.0;
        for (int k = 2; k <= m; ++k) {
            p = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / k;
            a = b; b = p;
        }
    }
    return p * std::sqrt(m + 0.5);
}

// inverse of the Legendre Vandermonde matrix V[i][m] = P~_m(x_i) (Trixi vandermonde_legendre), by
// Gauss-Jordan elimination with partial pivoting; row-major n x n.
inline std::vector<double> inverse_vandermonde_legendre(const Basis& b) {
    const int n = b.n;
    std::vector<double> A(n * n), I(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int m = 0; m < n; ++m) A[i * n + m] = legendre_normalized(m, b.nodes[i]);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
        for (int k = 0; k < n; ++k) { std::swap(A[c * n + k], A[piv * n + k]); std::swap(I[c * n + k], I[piv * n + k]); }
        const double d = A[c * n + c];
        for (int k = 0; k < n; ++k) { A[c * n + k] /= d; I[c * n + k] /= d; }
        for (int r = 0; r < n; ++r)
            if (r != c) {
                const double f = A[r * n + c];
                for (int k = 0; k < n; ++k) { A[r * n + k] -= f * A[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
            }
    }
    return I;
}

// Trixi IndicatorHennemannGassner (Hennemann, Rueda-Ramirez, Hindenlang, Gassner, J. Comput. Phys. 426
// (2021)), indicator variable density_pressure = (gamma-1)(rho rho_e - |rho v|^2 / 2), followed by the
// interface smoothing alpha_e = max(alpha_e, alpha_nb / 2) (Trixi apply_smoothing!).
inline void indicator_hennemann_gassner(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m,
                                        const double* u, std::vector<double>& alpha) {
    const int n = b.n;
    const std::vector<double> Vinv = inverse_vandermonde_legendre(b);
    const double threshold = 0.5 * std::pow(10.0, -1.8 * std::pow((double)n, 0.25));
    const double parameter_s = std::log((1.0 - 0.0001) / 0.0001);
    alpha.assign(m.n_elements, 0.0);
    for (int e = 0; e < m.n_elements; ++e) {
        double ind[MAXN * MAXN], tmp[MAXN * MAXN], modal[MAXN * MAXN];
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const double* x = u + idx_u(n, 0, i, j, e);
                ind[i + n * j] = (eq.gamma - 1.0) * (x[0] * x[3] - 0.5 * (x[1] * x[1] + x[2] * x[2]));
            }
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double r = 0.0;
                for (int a = 0; a < n; ++a) r += Vinv[i * n + a] * ind[a + n * j];
                tmp[i + n * j] = r;
            }
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double r = 0.0;
                for (int c = 0; c < n; ++c) r += Vinv[j * n + c] * tmp[i + n * c];
                modal[i + n * j] = r;
            }
        double total = 0.0, clip1 = 0.0, clip2 = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) total += modal[i + n * j] * modal[i + n * j];
        for (int j = 0; j < n - 1; ++j)
            for (int i = 0; i < n - 1; ++i) clip1 += modal[i + n * j] * modal[i + n * j];
        for (int j = 0; j < n - 2; ++j)
            for (int i = 0; i < n - 2; ++i) clip2 += modal[i + n * j] * modal[i + n * j];
        const double f1 = total != 0.0 ? (total - clip1) / total : 0.0;
        const double f2 = clip1 != 0.0 ? (clip1 - clip2) / clip1 : 0.0;
        const double energy = std::max(f1, f2);
        double a = 1.0 / (1.0 + std::exp(-parameter_s / threshold * (energy - threshold)));
        if (a < opt.alpha_min) a = 0.0;
        if (a > 1.0 - opt.alpha_min) a = 1.0;
        alpha[e] = std::min(opt.alpha_max, a);
    }
    if (opt.alpha_smooth) {
        const std::vector<double> tmp = alpha;
        for (int k = 0; k < m.n_interfaces; ++k) {
            const int l = m.interface_left[k], r = m.interface_right[k];
            alpha[l] = std::max(std::max(tmp[l], 0.5 * tmp[r]), alpha[l]);
            alpha[r] = std::max(std::max(tmp[r], 0.5 * tmp[l]), alpha[r]);
        }
        // and over the L2 mortars: each small element with the large one
        for (int k = 0; k < m.n_mortars; ++k) {
            const int lo = m.mortar_lower[k], up = m.mortar_upper[k], lg = m.mortar_large[k];
            alpha[lo] = std::max(std::max(tmp[lo], 0.5 * tmp[lg]), alpha[lo]);
            alpha[up] = std::max(std::max(tmp[up], 0.5 * tmp[lg]), alpha[up]);
            alpha[lg] = std::max(std::max(tmp[lg], 0.5 * tmp[lo]), alpha[lg]);
            alpha[lg] = std::max(std::max(tmp[lg], 0.5 * tmp[up]), alpha[lg]);
        }
    }
}

// Trixi 4-argument flux_lax_friedrichs (FluxPlusDissipation(flux_central, DissipationLocalLaxFriedrichs))
inline void rusanov(const Euler& eq, int speed_kind, const double* ul, const double* ur, int orientation, double* out,
                    bool& bad) {
    double fl[NV], fr[NV];
    eq.flux(ul, orientation, fl);
    eq.flux(ur, orientation, fr);
    const double lambda = eq.max_abs_speed(ul, ur, orientation, speed_kind, bad);
    for (int v = 0; v < NV; ++v) out[v] = 0.5 * (fl[v] + fr[v]) + (-0.5 * lambda * (ur[v] - ul[v]));
}

// First-order subcell FV on one element: Trixi calcflux_fv! (TreeMesh{2}) with volume_flux_fv; if
// `blended`, du += alpha * (w_i^-1 (f*_{i+1} - f*_i) + w_j^-1 (g*_{j+1} - g*_j)) (fv_kernel!,
// dg_2d.jl:251-282); always the subcell fluxes next to the faces into fn_low (load_fn_low!, :220-234;
// for pure DG elements calc_fn_low!, :1948-1991, computes exactly these).
inline void first_order_subcells(const Basis& b, const Euler& eq, const Options& opt, int e, const double* u,
                                 double* du, double alpha, bool blended, Workspace& ws, bool& bad) {
    const int n = b.n;
    double fx[(MAXN + 1) * MAXN * NV], fy[MAXN * (MAXN + 1) * NV];
    auto FX = [&](int f, int j) { return fx + NV * (f + (n + 1) * j); };   // face f in 0..n along x, row j
    auto FY = [&](int i, int f) { return fy + NV * (i + n * f); };         // face f in 0..n along y, column i
    for (int j = 0; j < n; ++j) {
        for (int v = 0; v < NV; ++v) { FX(0, j)[v] = 0.0; FX(n, j)[v] = 0.0; }
        for (int f = 1; f < n; ++f) rusanov(eq, opt.speed_kind, u + idx_u(n, 0, f - 1, j, e), u + idx_u(n, 0, f, j, e), 1, FX(f, j), bad);
    }
    for (int i = 0; i < n; ++i) {
        for (int v = 0; v < NV; ++v) { FY(i, 0)[v] = 0.0; FY(i, n)[v] = 0.0; }
        for (int f = 1; f < n; ++f) rusanov(eq, opt.speed_kind, u + idx_u(n, 0, i, f - 1, e), u + idx_u(n, 0, i, f, e), 2, FY(i, f), bad);
    }
    if (blended) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v)
                    du[idx_u(n, v, i, j, e)] += alpha * (1.0 / b.weights[i] * (FX(i + 1, j)[v] - FX(i, j)[v]) +
                                                         1.0 / b.weights[j] * (FY(i, j + 1)[v] - FY(i, j)[v]));
    }
    for (int l = 0; l < n; ++l)
        for (int v = 0; v < NV; ++v) {
            ws.fn_low[v + NV * (l + n * (0 + 4 * (size_t)e))] = FX(1, l)[v];
            ws.fn_low[v + NV * (l + n * (1 + 4 * (size_t)e))] = FX(n - 1, l)[v];
            ws.fn_low[v + NV * (l + n * (2 + 4 * (size_t)e))] = FY(l, 1)[v];
            ws.fn_low[v + NV * (l + n * (3 + 4 * (size_t)e))] = FY(l, n - 1)[v];
        }
}

// calc_interface_flux! with compute_alp for VolumeIntegralFRShockCapturing (dg_2d.jl:1879-1946): the LW
// flux Fn_ is blended with the first-order flux fn at the instantaneous u by alp = (alpha_L + alpha_R)/2,
// and alp = 1 where the low-order update of either face subcell (lambda = 1/2 weights) would not be
// admissible. J^{-1} at TreeMesh interfaces is element 1's (containers_2d.jl:29-31).
inline void calc_interface_flux_blended(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m,
                                        double dt, Workspace& ws, int nthreads = 1) {
    const int n = b.n;
    auto ii = [&](int side, int v, int l, size_t k) { return side + 2 * (v + NV * (l + (size_t)n * k)); };
    const double J = m.inverse_jacobian[0];
    bool bad = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad)
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int le = m.interface_left[k], re = m.interface_right[k];
        const int o = m.interface_orientation[k];
        const int left_dir = 2 * o - 1, right_dir = 2 * o - 2;
        for (int l = 0; l < n; ++l) {
            double Ul[NV], Ur[NV], ul[NV], ur[NV], fl[NV], fr[NV], Fn_[NV], fn[NV], fil[NV], fir[NV], Fn[NV];
            for (int v = 0; v < NV; ++v) {
                Ul[v] = ws.iU[ii(0, v, l, k)]; Ur[v] = ws.iU[ii(1, v, l, k)];
                ul[v] = ws.iu[ii(0, v, l, k)]; ur[v] = ws.iu[ii(1, v, l, k)];
                fl[v] = ws.iF[ii(0, v, l, k)]; fr[v] = ws.iF[ii(1, v, l, k)];
                fil[v] = ws.fn_low[v + NV * (l + n * (left_dir + 4 * (size_t)le))];
                fir[v] = ws.fn_low[v + NV * (l + n * (right_dir + 4 * (size_t)re))];
            }
            lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, fl, fr, Ul, Ur, ul, ur, o, Fn_, bad);
            rusanov(eq, opt.speed_kind, ul, ur, o, fn, bad);
            // compute_alp (dg_2d.jl:1879-1901)
            double alp = 0.5 * (ws.alpha[le] + ws.alpha[re]);
            double Fb[NV], low[NV];
            for (int v = 0; v < NV; ++v) Fb[v] = (1.0 - alp) * Fn_[v] + alp * fn[v];
            const double lam = 0.5;
            for (int v = 0; v < NV; ++v) low[v] = ul[v] - dt * J / (b.weights[n - 1] * lam) * (Fb[v] - fil[v]);
            if (!eq.is_admissible(low)) alp = 1.0;
            else {
                for (int v = 0; v < NV; ++v) low[v] = ur[v] - dt * J / (b.weights[0] * lam) * (fir[v] - Fb[v]);
                if (!eq.is_admissible(low)) alp = 1.0;
            }
            for (int v = 0; v < NV; ++v) Fn[v] = alp * fn[v] + (1.0 - alp) * Fn_[v];
            for (int v = 0; v < NV; ++v) {
                ws.surface_flux_values[v + NV * (l + n * (left_dir + 4 * (size_t)le))] = Fn[v];
                ws.surface_flux_values[v + NV * (l + n * (right_dir + 4 * (size_t)re))] = Fn[v];
            }
        }
    }
    if (bad) ws.bad = true;
}

// rhs!(du, u, t, dt, mesh::TreeMesh{2}, ..., ::LW, ...) (src/solvers/dgsem_tree/dg_2d.jl:28-83)
// kind 0 = LW, 1 = MDRK stage 1 (multi_derivative_2d.jl:1-57), 2 = MDRK stage 2 (:59-116; `u2` = u*).
inline void rhs(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m, const double* u,
                const double* u2, double* du, double t, double dt, const BoundaryData* bd, int kind, Workspace& ws,
                int nthreads = 1) {
    ensure_workspace(b, m, ws, kind != 0);
    ws.bad = false;
    const size_t ndof = (size_t)NV * b.n * b.n * m.n_elements;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (long long k = 0; k < (long long)ndof; ++k) du[k] = 0.0;   // reset_du!
    if (opt.shock_capturing) {
        // the indicator and the FV subcells use the instantaneous u in every stage
        // (dg_2d.jl:1665; multi_derivative_2d.jl:166, 222, 205, 257)
        indicator_hennemann_gassner(b, eq, opt, m, u, ws.alpha);
        ws.fn_low.assign((size_t)NV * b.n * 4 * m.n_elements, 0.0);
    }
    bool bad_fv = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad_fv)
    for (int e = 0; e < m.n_elements; ++e) {
        const double a = opt.shock_capturing ? 1.0 - ws.alpha[e] : 1.0;
        const SourceArgs sa{opt.source, opt.xnode, eq.gamma, t};
        if (kind == 0)
            lw_volume_element(b, eq, opt, e, u, du, dt, m.inverse_jacobian[e], a, ws, t);
        else if (kind == 1)
            mdrk1_volume_element(b, eq, e, u, du, dt, m.inverse_jacobian[e], a, ws, nullptr, nullptr, &sa);
        else
            mdrk2_volume_element(b, eq, e, u2, du, dt, m.inverse_jacobian[e], a, ws, nullptr, nullptr, &sa);
        if (opt.shock_capturing) {
            // pure_and_blended_element_ids!: DG only where isapprox(alpha, 0, atol = 1e-12)
            const bool blended = !(std::fabs(ws.alpha[e]) <= 1e-12);
            first_order_subcells(b, eq, opt, e, u, du, ws.alpha[e], blended, ws, bad_fv);
        }
    }
    if (bad_fv) ws.bad = true;
    prolong2interfaces(b, m, u, ws, nthreads);
    if (opt.shock_capturing)
        calc_interface_flux_blended(b, eq, opt, m, dt, ws, nthreads);
    else
        calc_interface_flux(b, eq, opt, m, ws, nthreads);
    if (m.n_boundaries > 0) {
        if (has_dirichlet_boundaries(m) && (!bd || !bd->u_levels || !bd->u_now))
            throw std::invalid_argument("boundary data missing");
        calc_boundary_flux(b, eq, opt, m, u, bd ? *bd : BoundaryData{}, kind == 1 ? 0.5 : 1.0, ws);
    }
    // (with shock capturing the mortars keep the plain LW flux: calc_mortar_flux!, dg_2d.jl:1596-1646, has no
    // blending)
    if (m.n_mortars > 0) calc_mortar_flux(b, eq, opt, m, u, ws, nthreads);
    surface_integral_and_jacobian(b, m, du, ws, nthreads);
}

// Trixi max_dt(u, t, mesh::TreeMesh{2}, constant_speed::False, ...) * cfl (src/solvers/lwfr.jl:176-190)
inline double max_dt(const Basis& b, const Euler& eq, const TreeMesh& m, const double* u, double cfl, bool& bad,
                     int nthreads = 1) {
    const int n = b.n;
    double max_scaled_speed = std::nextafter(0.0, 1.0);
    bool bad_any = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(max : max_scaled_speed) reduction(|| : bad_any)
    for (int e = 0; e < m.n_elements; ++e) {
        double ml1 = 0.0, ml2 = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double l1, l2;
                eq.max_abs_speeds(u + idx_u(n, 0, i, j, e), l1, l2, bad_any);
                ml1 = std::max(ml1, l1);
                ml2 = std::max(ml2, l2);
            }
        max_scaled_speed = std::max(max_scaled_speed, m.inverse_jacobian[e] * (ml1 + ml2));
    }
    if (bad_any) bad = true;
    return cfl * (2.0 / (n * max_scaled_speed));
}

}  // namespace tlwo
