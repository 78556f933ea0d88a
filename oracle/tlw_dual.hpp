// tlw_dual.hpp -- test infrastructure only: a scalar-templated restatement of one Lax-Wendroff step, and of one
// two-stage MDRK step, on a periodic TreeMesh{2}, instantiated with double and with a forward-mode dual number (value
// and one directional derivative). The dual instantiation differentiates the step map at a fixed dt along a direction, which is
// the check ForwardDiff gives for the reference's Julia code: directional derivatives of the discrete solution map
// that the discrete adjoint's dot products must reproduce.
//
// What is restated (the same forward map as tlw_oracle.hpp and tlw_adjoint.hpp):
//   volume: lw_volume_kernel_3! (N = 3) / lw_volume_kernel_4! (N >= 4), src/solvers/dgsem_tree/dg_2d.jl:674-1267:
//     d_1 = C(f(u), g(u)) with C(x, y) = -dt J^{-1} (D x + D y); per stage the perturbed states u +- d's, the
//     centred finite differences of the fluxes, d_{s+1} = C(ft_s, gt_s); F = f(u) + sum tw_s ft_s,
//     U = u + sum tw_s d_s (tw = 1/2, 1/6, 1/24, 1/120), and the volume term Dhat F + Dhat G;
//   interfaces: Rusanov in the TreeMesh order (dg_2d.jl:1903-1946): Fn = (F_L + F_R)/2 - lambda(U_L, U_R)/2 (u_R -
//     u_L), lambda = max_abs_speed_naive (or max_abs_speed) of the time-averaged U;
//   Trixi's weak-form surface integral and apply_jacobian (du *= -J^{-1}).
// Branches (max, |.|) follow the value, so the derivative is that of the branch the value takes.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "tlw_oracle.hpp"

namespace tlwo {

struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double a) : v(a) {}
    Dual(double a, double b) : v(a), d(b) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
inline Dual sqrt(Dual a) {
    const double s = std::sqrt(a.v);
    return {s, a.d / (2.0 * s)};
}
inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
inline Dual dmax(Dual a, Dual b) { return a.v < b.v ? b : a; }   // std::max's choice, with its derivative
inline double dmax(double a, double b) { return std::max(a, b); }
inline double value(double a) { return a; }
inline double value(Dual a) { return a.v; }

// Euler flux pair (Trixi flux(u, 1|2, eq))
template <class T>
inline void dual_fluxes(double gamma, const T* u, T* f, T* g) {
    const T rho = u[0], m1 = u[1], m2 = u[2], e = u[3];
    const T v1 = m1 / rho, v2 = m2 / rho;
    const T p = (gamma - 1.0) * (e - 0.5 * (m1 * v1 + m2 * v2));
    f[0] = m1; f[1] = m1 * v1 + p; f[2] = m1 * v2; f[3] = (e + p) * v1;
    g[0] = m2; g[1] = m2 * v1; g[2] = m2 * v2 + p; g[3] = (e + p) * v2;
}

// Rusanov interfaces in the TreeMesh order (lambda from the time-averaged U, jump in uj) and the weak-form lift
// into du [v, i, j, e]
template <class T>
inline void dual_interfaces(const Basis& b, double gamma, int speed_kind, const TreeMesh& m, const std::vector<T>& Ug,
                            const std::vector<T>& Fg, const std::vector<T>& Gg, const T* uj, std::vector<T>& du) {
    using std::fabs;
    using std::sqrt;
    const int n = b.n, nn = n * n;
    auto at = [&](int v, int i, int j) { return v + NV * (i + n * j); };
    for (int q = 0; q < m.n_interfaces; ++q) {
        const int le = m.interface_left[q], re = m.interface_right[q], o = m.interface_orientation[q];
        for (int l = 0; l < n; ++l) {
            const int iL = o == 1 ? n - 1 : l, jL = o == 1 ? l : n - 1, iR = o == 1 ? 0 : l, jR = o == 1 ? l : 0;
            const size_t pL = (size_t)NV * nn * le + at(0, iL, jL), pR = (size_t)NV * nn * re + at(0, iR, jR);
            const std::vector<T>& Fx = o == 1 ? Fg : Gg;
            const T rl = Ug[pL], rr = Ug[pR];
            const T vl = Ug[pL + o] / rl, vr = Ug[pR + o] / rr;
            const T v1l = Ug[pL + 1] / rl, v2l = Ug[pL + 2] / rl, v1r = Ug[pR + 1] / rr, v2r = Ug[pR + 2] / rr;
            const T pl = (gamma - 1.0) * (Ug[pL + 3] - 0.5 * (Ug[pL + 1] * v1l + Ug[pL + 2] * v2l));
            const T pr = (gamma - 1.0) * (Ug[pR + 3] - 0.5 * (Ug[pR + 1] * v1r + Ug[pR + 2] * v2r));
            const T cl = sqrt(gamma * pl / rl), cr = sqrt(gamma * pr / rr);
            const T lambda = speed_kind == 0 ? dmax(fabs(vl), fabs(vr)) + dmax(cl, cr) : dmax(fabs(vl) + cl, fabs(vr) + cr);
            for (int v = 0; v < NV; ++v) {
                const T Fn = 0.5 * (Fx[pL + v] + Fx[pR + v]) + (-0.5 * lambda * (uj[pR + v] - uj[pL + v]));
                du[pL + v] += Fn * b.inv_w_last;
                du[pR + v] -= Fn * b.inv_w_first;
            }
        }
    }
}

// One MDRK step (mdrk.jl:1-29 with rhs_mdrk1! / rhs_mdrk2!, src/solvers/dgsem_tree/multi_derivative_2d.jl:1-116 and
// the TreeMesh mdrk kernels :263-555) on a periodic TreeMesh at a fixed dt: stage 1 at u with d = C(f(u)) and the
// 4-point f_t from u +- d, u +- 2d: the time averages F = f/2 + f_t/8, U = u/2 + d/8 for the surface and F2 = f +
// f_t/6, U2 = u + d/6 kept for stage 2; u* = u + dt rhs_1. Stage 2 at u*: F = F2 + f*_t/3, U = U2 + d*/3, the
// interfaces with the jump in u^n; out = u + dt rhs_2.
template <class T>
inline void mdrk_step_templated(const Basis& b, double gamma, int speed_kind, const TreeMesh& m, const T* u,
                                double dt, T* out) {
    const int n = b.n, nn = n * n, E = m.n_elements;
    const size_t nd = (size_t)NV * nn * E;
    std::vector<T> Ug(nd), Fg(nd), Gg(nd), U2(nd), F2(nd), G2(nd), du(nd), us(nd);
    auto at = [&](int v, int i, int j) { return v + NV * (i + n * j); };
    for (int stage = 1; stage <= 2; ++stage) {
        const T* x = stage == 1 ? u : us.data();
        for (size_t k = 0; k < nd; ++k) du[k] = 0.0;
        for (int e = 0; e < E; ++e) {
            const double ij = m.inverse_jacobian[e];
            const T* xe = x + (size_t)NV * nn * e;
            const size_t o = (size_t)NV * nn * e;
            std::vector<T> f0(NV * nn), g0(NV * nn), d(NV * nn), F(NV * nn), G(NV * nn);
            for (int k = 0; k < nn; ++k) dual_fluxes(gamma, xe + NV * k, &f0[NV * k], &g0[NV * k]);
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    for (int v = 0; v < NV; ++v) {
                        T s = 0.0;
                        for (int k = 0; k < n; ++k) s += b.D[i * n + k] * f0[at(v, k, j)] + b.D[j * n + k] * g0[at(v, i, k)];
                        d[at(v, i, j)] = (-dt * ij) * s;
                    }
            for (int k = 0; k < nn; ++k) {
                T pm[NV], pp[NV], pmm[NV], ppp[NV];
                for (int v = 0; v < NV; ++v) {
                    const T dd = d[NV * k + v];
                    pm[v] = xe[NV * k + v] - dd;
                    pp[v] = xe[NV * k + v] + dd;
                    pmm[v] = xe[NV * k + v] - 2.0 * dd;
                    ppp[v] = xe[NV * k + v] + 2.0 * dd;
                }
                T fm[NV], gm[NV], fp[NV], gp[NV], fmm[NV], gmm[NV], fpp[NV], gpp[NV];
                dual_fluxes(gamma, pm, fm, gm);
                dual_fluxes(gamma, pp, fp, gp);
                dual_fluxes(gamma, pmm, fmm, gmm);
                dual_fluxes(gamma, ppp, fpp, gpp);
                for (int v = 0; v < NV; ++v) {
                    const int q = NV * k + v;
                    const T ft = (1.0 / 12.0) * (-fpp[v] + 8.0 * fp[v] - 8.0 * fm[v] + fmm[v]);
                    const T gt = (1.0 / 12.0) * (-gpp[v] + 8.0 * gp[v] - 8.0 * gm[v] + gmm[v]);
                    if (stage == 1) {
                        F[q] = 0.5 * f0[q] + 0.125 * ft;
                        G[q] = 0.5 * g0[q] + 0.125 * gt;
                        Ug[o + q] = 0.5 * xe[q] + 0.125 * d[q];
                        F2[o + q] = f0[q] + (1.0 / 6.0) * ft;
                        G2[o + q] = g0[q] + (1.0 / 6.0) * gt;
                        U2[o + q] = xe[q] + (1.0 / 6.0) * d[q];
                    } else {
                        F[q] = F2[o + q] + (1.0 / 3.0) * ft;
                        G[q] = G2[o + q] + (1.0 / 3.0) * gt;
                        Ug[o + q] = U2[o + q] + (1.0 / 3.0) * d[q];
                    }
                    Fg[o + q] = F[q];
                    Gg[o + q] = G[q];
                }
            }
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    for (int v = 0; v < NV; ++v) {
                        T s = 0.0;
                        for (int k = 0; k < n; ++k) s += b.Dhat[i * n + k] * F[at(v, k, j)] + b.Dhat[j * n + k] * G[at(v, i, k)];
                        du[o + at(v, i, j)] = s;
                    }
        }
        dual_interfaces(b, gamma, speed_kind, m, Ug, Fg, Gg, u, du);   // the jump in u^n in both stages
        T* tgt = stage == 1 ? us.data() : out;
        for (int e = 0; e < E; ++e)
            for (int k = 0; k < NV * nn; ++k) {
                const size_t p = (size_t)NV * nn * e + k;
                tgt[p] = u[p] + dt * ((-m.inverse_jacobian[e]) * du[p]);
            }
    }
}

// one step out = u + dt rhs(u) on a periodic TreeMesh (FR volume integral, Rusanov, N >= 3)
template <class T>
inline void lw_step_templated(const Basis& b, double gamma, int speed_kind, const TreeMesh& m, int N, const T* u,
                              double dt, T* out) {
    using std::fabs;
    using std::sqrt;
    const int n = b.n, nn = n * n, E = m.n_elements;
    const int depth = std::min(N, 4);
    std::vector<T> Ug((size_t)NV * nn * E), Fg((size_t)NV * nn * E), Gg((size_t)NV * nn * E), du((size_t)NV * nn * E);
    auto at = [&](int v, int i, int j) { return v + NV * (i + n * j); };
    for (int e = 0; e < E; ++e) {
        const double ij = m.inverse_jacobian[e];
        const T* ue = u + (size_t)NV * nn * e;
        std::vector<T> f0(NV * nn), g0(NV * nn), up(NV * nn), um(NV * nn), upp(NV * nn), umm(NV * nn);
        std::vector<T> F(NV * nn), G(NV * nn), U(NV * nn), dcur(NV * nn), ft(NV * nn), gt(NV * nn);
        // C(x, y) = -dt J^{-1} (D x + D y)
        auto contract = [&](const std::vector<T>& x, const std::vector<T>& y, std::vector<T>& d) {
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    for (int v = 0; v < NV; ++v) {
                        T s = 0.0;
                        for (int k = 0; k < n; ++k) s += b.D[i * n + k] * x[at(v, k, j)] + b.D[j * n + k] * y[at(v, i, k)];
                        d[at(v, i, j)] = (-dt * ij) * s;
                    }
        };
        for (int k = 0; k < nn; ++k) dual_fluxes(gamma, ue + NV * k, &f0[NV * k], &g0[NV * k]);
        for (int k = 0; k < NV * nn; ++k) {
            F[k] = f0[k]; G[k] = g0[k]; U[k] = ue[k];
            up[k] = um[k] = upp[k] = umm[k] = ue[k];
        }
        contract(f0, g0, dcur);
        const double tw[5] = {0.0, 0.5, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0};
        for (int s = 1; s <= depth; ++s) {
            // perturbed states after adding d_s (the kernels' update coefficients per stage)
            const double cp[5] = {0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0};
            const double cm[5] = {0, -1.0, 0.5, -1.0 / 6.0, 1.0 / 24.0};
            const double cpp[5] = {0, 2.0, 2.0, 4.0 / 3.0, 2.0 / 3.0};
            const double cmm[5] = {0, -2.0, 2.0, -4.0 / 3.0, 2.0 / 3.0};
            for (int k = 0; k < NV * nn; ++k) {
                const T d = dcur[k];
                U[k] += tw[s] * d;
                up[k] += cp[s] * d;
                um[k] += cm[s] * d;
                upp[k] += cpp[s] * d;
                umm[k] += cmm[s] * d;
            }
            for (int k = 0; k < nn; ++k) {
                T fp[NV], gp[NV], fm[NV], gm[NV], fpp[NV], gpp[NV], fmm[NV], gmm[NV];
                dual_fluxes(gamma, &up[NV * k], fp, gp);
                dual_fluxes(gamma, &um[NV * k], fm, gm);
                if (depth >= 3 || s == 1) {
                    dual_fluxes(gamma, &upp[NV * k], fpp, gpp);
                    dual_fluxes(gamma, &umm[NV * k], fmm, gmm);
                }
                for (int v = 0; v < NV; ++v) {
                    const int o = NV * k + v;
                    const T f = f0[o], g = g0[o];
                    if (s == 1) {            // f_t: 4-point centred difference
                        ft[o] = (1.0 / 12.0) * (-fpp[v] + 8.0 * fp[v] - 8.0 * fm[v] + fmm[v]);
                        gt[o] = (1.0 / 12.0) * (-gpp[v] + 8.0 * gp[v] - 8.0 * gm[v] + gmm[v]);
                    } else if (s == 2 && depth == 4) {   // f_tt: 5-point
                        ft[o] = (1.0 / 12.0) * (-fpp[v] + 16.0 * fp[v] - 30.0 * f + 16.0 * fm[v] - fmm[v]);
                        gt[o] = (1.0 / 12.0) * (-gpp[v] + 16.0 * gp[v] - 30.0 * g + 16.0 * gm[v] - gmm[v]);
                    } else if (s == 2) {     // f_tt: 3-point (depth 3)
                        ft[o] = fp[v] - 2.0 * f + fm[v];
                        gt[o] = gp[v] - 2.0 * g + gm[v];
                    } else if (s == 3) {     // f_ttt
                        ft[o] = 0.5 * (fpp[v] - 2.0 * fp[v] + 2.0 * fm[v] - fmm[v]);
                        gt[o] = 0.5 * (gpp[v] - 2.0 * gp[v] + 2.0 * gm[v] - gmm[v]);
                    } else {                 // f_tttt, with the reference's factor 1/2 (dg_2d.jl:1203)
                        ft[o] = 0.5 * (fpp[v] - 4.0 * fp[v] + 6.0 * f - 4.0 * fm[v] + fmm[v]);
                        gt[o] = 0.5 * (gpp[v] - 4.0 * gp[v] + 6.0 * g - 4.0 * gm[v] + gmm[v]);
                    }
                }
            }
            for (int k = 0; k < NV * nn; ++k) {
                F[k] += tw[s] * ft[k];
                G[k] += tw[s] * gt[k];
            }
            if (s < depth) contract(ft, gt, dcur);
        }
        // volume term Dhat F + Dhat G; element caches for the interfaces
        T* de = &du[(size_t)NV * nn * e];
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    T s = 0.0;
                    for (int k = 0; k < n; ++k) s += b.Dhat[i * n + k] * F[at(v, k, j)] + b.Dhat[j * n + k] * G[at(v, i, k)];
                    de[at(v, i, j)] = s;
                }
        for (int k = 0; k < NV * nn; ++k) {
            Ug[(size_t)NV * nn * e + k] = U[k];
            Fg[(size_t)NV * nn * e + k] = F[k];
            Gg[(size_t)NV * nn * e + k] = G[k];
        }
    }
    // interfaces: Rusanov in the TreeMesh argument order, lambda from U, jump in u; the weak-form lift
    for (int q = 0; q < m.n_interfaces; ++q) {
        const int le = m.interface_left[q], re = m.interface_right[q], o = m.interface_orientation[q];
        for (int l = 0; l < n; ++l) {
            const int iL = o == 1 ? n - 1 : l, jL = o == 1 ? l : n - 1, iR = o == 1 ? 0 : l, jR = o == 1 ? l : 0;
            const size_t pL = (size_t)NV * nn * le + at(0, iL, jL), pR = (size_t)NV * nn * re + at(0, iR, jR);
            const std::vector<T>& Fx = o == 1 ? Fg : Gg;
            const T rl = Ug[pL], rr = Ug[pR];
            const T vl = Ug[pL + o] / rl, vr = Ug[pR + o] / rr;
            const T v1l = Ug[pL + 1] / rl, v2l = Ug[pL + 2] / rl, v1r = Ug[pR + 1] / rr, v2r = Ug[pR + 2] / rr;
            const T pl = (gamma - 1.0) * (Ug[pL + 3] - 0.5 * (Ug[pL + 1] * v1l + Ug[pL + 2] * v2l));
            const T pr = (gamma - 1.0) * (Ug[pR + 3] - 0.5 * (Ug[pR + 1] * v1r + Ug[pR + 2] * v2r));
            const T cl = sqrt(gamma * pl / rl), cr = sqrt(gamma * pr / rr);
            const T lambda = speed_kind == 0 ? dmax(fabs(vl), fabs(vr)) + dmax(cl, cr) : dmax(fabs(vl) + cl, fabs(vr) + cr);
            for (int v = 0; v < NV; ++v) {
                const T Fn = 0.5 * (Fx[pL + v] + Fx[pR + v]) + (-0.5 * lambda * (u[pR + v] - u[pL + v]));
                du[pL + v] += Fn * b.inv_w_last;
                du[pR + v] -= Fn * b.inv_w_first;
            }
        }
    }
    for (int e = 0; e < E; ++e)
        for (int k = 0; k < NV * nn; ++k) {
            const size_t p = (size_t)NV * nn * e + k;
            out[p] = u[p] + dt * ((-m.inverse_jacobian[e]) * du[p]);
        }
}

}  // namespace tlwo
