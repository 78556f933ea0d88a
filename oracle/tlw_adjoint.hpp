// tlw_adjoint.hpp -- test infrastructure only: CPU restatement of the discrete adjoint (vector-Jacobian
// product) of one Lax-Wendroff step on a periodic TreeMesh{2}, used to check the CUDA adjoint kernels.
//
// The reference has no adjoint; what is differentiated is the reference's forward map
//   u_new = u + dt * rhs(u),  rhs = LW volume (src/solvers/dgsem_tree/dg_2d.jl:674-1267, depth 3 for N = 3,
//   depth 4 for N >= 4) + Rusanov interface flux with the TreeMesh argument order (dg_2d.jl:1903-1946:
//   speed from the time-averaged U, jump in the instantaneous u) + weak-form surface lift + apply_jacobian,
// at a fixed dt (the step sizes of the forward run are held constant, as the gradient of the discrete
// solution map at the recorded dt sequence). Plain FR volume integral, no boundaries, no shock capturing.
//
// Notation (matching the forward restatement in tlw_oracle.hpp): d_1 = ut, d_2 = utt, ... are the
// dt-scaled time derivatives, C(x, y) = -dt J^{-1} (D x + D y) the contraction that produces the next one,
// and the perturbed states of stage s are P_q = u + sum_{m <= s} a[q][m] d_m for q in {-, +, --, ++}.
// The forward map of one element is
//   d_1 = C(f(u), g(u));  ft_s = sum_q w_s[q] f(P_q^s) + w_s[0] f(u);  d_{s+1} = C(ft_s, gt_s)
//   F = f(u) + sum_s tw_s ft_s,   U = u + sum_s tw_s d_s,   tw = (1/2, 1/6, 1/24, 1/120)
// and its reverse runs s = depth .. 1 with the flux Jacobians transposed at each P_q^s.
#pragma once
#include "tlw_oracle.hpp"

namespace tlwo {

// out += Jf(u)^T wf + Jg(u)^T wg  (Euler flux Jacobians, conservative variables)
inline void euler_flux_vjp(const Euler& eq, const double* u, const double* wf, const double* wg, double* out) {
    const double g = eq.gamma, gm1 = g - 1.0;
    const double rho = u[0], v1 = u[1] / rho, v2 = u[2] / rho;
    const double q = 0.5 * (v1 * v1 + v2 * v2);
    const double p = gm1 * (u[3] - rho * q);
    const double H = (u[3] + p) / rho;
    out[0] += wf[1] * (gm1 * q - v1 * v1) + wf[2] * (-v1 * v2) + wf[3] * v1 * (gm1 * q - H)
            + wg[1] * (-v1 * v2) + wg[2] * (gm1 * q - v2 * v2) + wg[3] * v2 * (gm1 * q - H);
    out[1] += wf[0] + wf[1] * (2.0 - gm1) * v1 + wf[2] * v2 + wf[3] * (H - gm1 * v1 * v1)
            + wg[1] * v2 + wg[2] * (-gm1 * v1) + wg[3] * (-gm1 * v1 * v2);
    out[2] += wf[1] * (-gm1 * v2) + wf[2] * v1 + wf[3] * (-gm1 * v1 * v2)
            + wg[0] + wg[1] * v1 + wg[2] * (2.0 - gm1) * v2 + wg[3] * (H - gm1 * v2 * v2);
    out[3] += wf[1] * gm1 + wf[3] * g * v1 + wg[2] * gm1 + wg[3] * g * v2;
}

// gradients of |v_d| and of c = sqrt(gamma p / rho) with respect to the conservative state
inline void speed_partials(const Euler& eq, const double* u, int orientation, double* dv, double* dc) {
    const double g = eq.gamma, gm1 = g - 1.0;
    const double rho = u[0], v1 = u[1] / rho, v2 = u[2] / rho;
    const double q = 0.5 * (v1 * v1 + v2 * v2);
    const double p = gm1 * (u[3] - rho * q);
    const double c = std::sqrt(g * p / rho);
    const double vd = orientation == 1 ? v1 : v2;
    const double sg = (vd > 0.0) - (vd < 0.0);
    dv[0] = -sg * vd / rho;
    dv[1] = orientation == 1 ? sg / rho : 0.0;
    dv[2] = orientation == 2 ? sg / rho : 0.0;
    dv[3] = 0.0;
    const double k = g / (2.0 * c * rho);
    dc[0] = k * (gm1 * q - p / rho);
    dc[1] = -k * gm1 * v1;
    dc[2] = -k * gm1 * v2;
    dc[3] = k * gm1;
}

struct LWStencils {
    int depth;
    double tw[5];          // Taylor weights of stage s (index 1..4)
    double a[4][5];        // perturbation coefficients a[q][m], q = -, +, --, ++; m = 1..4
    double w[5][5];        // w[s][0] weight of f(u), w[s][1 + q] weight of f(P_q^s)
};

inline LWStencils lw_stencils(int N) {
    LWStencils S{};
    S.depth = N >= 4 ? 4 : 3;
    const double tw[5] = {0.0, 0.5, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0};
    for (int s = 0; s < 5; ++s) S.tw[s] = tw[s];
    const double a[4][5] = {{0.0, -1.0, 0.5, -1.0 / 6.0, 1.0 / 24.0},
                            {0.0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0},
                            {0.0, -2.0, 2.0, -4.0 / 3.0, 2.0 / 3.0},
                            {0.0, 2.0, 2.0, 4.0 / 3.0, 2.0 / 3.0}};
    std::memcpy(S.a, a, sizeof(a));
    // stage 1: (-fpp + 8 fp - 8 fm + fmm) / 12
    S.w[1][0] = 0.0; S.w[1][1] = -8.0 / 12.0; S.w[1][2] = 8.0 / 12.0; S.w[1][3] = 1.0 / 12.0; S.w[1][4] = -1.0 / 12.0;
    if (S.depth == 4) {
        // stage 2: (-fpp + 16 fp - 30 f + 16 fm - fmm) / 12
        S.w[2][0] = -30.0 / 12.0; S.w[2][1] = 16.0 / 12.0; S.w[2][2] = 16.0 / 12.0; S.w[2][3] = -1.0 / 12.0;
        S.w[2][4] = -1.0 / 12.0;
    } else {
        // stage 2 of the depth-3 procedure: fp - 2 f + fm
        S.w[2][0] = -2.0; S.w[2][1] = 1.0; S.w[2][2] = 1.0; S.w[2][3] = 0.0; S.w[2][4] = 0.0;
    }
    // stage 3: (fpp - 2 fp + 2 fm - fmm) / 2
    S.w[3][0] = 0.0; S.w[3][1] = 1.0; S.w[3][2] = -1.0; S.w[3][3] = -0.5; S.w[3][4] = 0.5;
    // stage 4: (fpp - 4 fp + 6 f - 4 fm + fmm) / 2
    S.w[4][0] = 3.0; S.w[4][1] = -2.0; S.w[4][2] = -2.0; S.w[4][3] = 0.5; S.w[4][4] = 0.5;
    return S;
}

// Reverse of the LW procedure of one element: given bar_F, bar_G, bar_U ([v, i, j] of the element),
// adds d(F, G, U)/du ^T (bar_F, bar_G, bar_U) to bar_u.
inline void lw_volume_element_vjp(const Basis& b, const Euler& eq, int N, const double* ue, double dt,
                                  double inv_jac, const double* bar_F, const double* bar_G, const double* bar_U,
                                  double* bar_u) {
    const int n = b.n, nn = n * n;
    const LWStencils S = lw_stencils(N);
    const int depth = S.depth;
    auto L = [&](int i, int j) { return NV * (i + n * j); };
    std::vector<double> d(5 * NV * nn, 0.0), bd(5 * NV * nn, 0.0);
    std::vector<double> fx(NV * nn), gy(NV * nn), bfx(NV * nn), bgy(NV * nn);
    auto D_ = [&](int m) { return d.data() + (size_t)m * NV * nn; };
    auto BD = [&](int m) { return bd.data() + (size_t)m * NV * nn; };
    // C(x, y) into t
    auto contract = [&](const std::vector<double>& x, const std::vector<double>& y, double* t) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    double s = 0.0;
                    for (int k = 0; k < n; ++k) s += b.D[i * n + k] * x[L(k, j) + v] + b.D[j * n + k] * y[L(i, k) + v];
                    t[L(i, j) + v] = -dt * inv_jac * s;
                }
    };
    // C^T(w): bx[k, j] += -dt J^-1 sum_i D[i, k] w[i, j];  by[i, k] += -dt J^-1 sum_j D[j, k] w[i, j]
    auto contract_t = [&](const double* w, std::vector<double>& bx, std::vector<double>& by) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    const double c = -dt * inv_jac * w[L(i, j) + v];
                    for (int k = 0; k < n; ++k) {
                        bx[L(k, j) + v] += b.D[i * n + k] * c;
                        by[L(i, k) + v] += b.D[j * n + k] * c;
                    }
                }
    };
    auto state = [&](int s, int q, int i, int j, double* P) {
        for (int v = 0; v < NV; ++v) {
            double x = ue[L(i, j) + v];
            for (int m = 1; m <= s; ++m) x += S.a[q][m] * D_(m)[L(i, j) + v];
            P[v] = x;
        }
    };
    // forward: d_1 .. d_depth
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) eq.fluxes(ue + L(i, j), &fx[L(i, j)], &gy[L(i, j)]);
    contract(fx, gy, D_(1));
    for (int s = 1; s < depth; ++s) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double f0[NV], g0[NV], P[NV], fq[NV], gq[NV];
                eq.fluxes(ue + L(i, j), f0, g0);
                for (int v = 0; v < NV; ++v) { fx[L(i, j) + v] = S.w[s][0] * f0[v]; gy[L(i, j) + v] = S.w[s][0] * g0[v]; }
                for (int q = 0; q < 4; ++q) {
                    if (S.w[s][1 + q] == 0.0) continue;
                    state(s, q, i, j, P);
                    eq.fluxes(P, fq, gq);
                    for (int v = 0; v < NV; ++v) {
                        fx[L(i, j) + v] += S.w[s][1 + q] * fq[v];
                        gy[L(i, j) + v] += S.w[s][1 + q] * gq[v];
                    }
                }
            }
        contract(fx, gy, D_(s + 1));
    }
    // reverse
    for (int m = 1; m <= depth; ++m)
        for (int k = 0; k < NV * nn; ++k) BD(m)[k] = S.tw[m] * bar_U[k];
    std::vector<double> bf0(bar_F, bar_F + NV * nn), bg0(bar_G, bar_G + NV * nn);
    for (int k = 0; k < NV * nn; ++k) bar_u[k] += bar_U[k];
    for (int s = depth; s >= 1; --s) {
        for (int k = 0; k < NV * nn; ++k) { bfx[k] = S.tw[s] * bar_F[k]; bgy[k] = S.tw[s] * bar_G[k]; }
        if (s < depth) contract_t(BD(s + 1), bfx, bgy);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                for (int v = 0; v < NV; ++v) {
                    bf0[o + v] += S.w[s][0] * bfx[o + v];
                    bg0[o + v] += S.w[s][0] * bgy[o + v];
                }
                for (int q = 0; q < 4; ++q) {
                    const double wq = S.w[s][1 + q];
                    if (wq == 0.0) continue;
                    double P[NV], wf[NV], wg[NV], bP[NV] = {0, 0, 0, 0};
                    state(s, q, i, j, P);
                    for (int v = 0; v < NV; ++v) { wf[v] = wq * bfx[o + v]; wg[v] = wq * bgy[o + v]; }
                    euler_flux_vjp(eq, P, wf, wg, bP);
                    for (int v = 0; v < NV; ++v) {
                        bar_u[o + v] += bP[v];
                        for (int m = 1; m <= s; ++m) BD(m)[o + v] += S.a[q][m] * bP[v];
                    }
                }
            }
    }
    contract_t(BD(1), bf0, bg0);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) euler_flux_vjp(eq, ue + L(i, j), &bf0[L(i, j)], &bg0[L(i, j)], bar_u + L(i, j));
}

// lam_out = (d u_new / d u)^T lam_in for u_new = u + dt * rhs(u) on a periodic TreeMesh{2}: LW volume
// integral (FR), Rusanov surface flux (speed_kind 0 = max_abs_speed_naive, 1 = max_abs_speed), weak-form
// lift, apply_jacobian. ws.U (the time-averaged U) is recomputed by a forward rhs.
inline void adjoint_step(const Basis& b, const Euler& eq, const Options& opt, const TreeMesh& m, const double* u,
                         double dt, const double* lam_in, double* lam_out, Workspace& ws, int nthreads = 1) {
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    std::vector<double> du(ndof);
    rhs(b, eq, opt, m, u, nullptr, du.data(), 0.0, dt, nullptr, 0, ws, nthreads);
    std::vector<double> bF(ndof, 0.0), bG(ndof, 0.0), bU(ndof, 0.0);
    for (size_t k = 0; k < ndof; ++k) lam_out[k] = lam_in[k];
    // volume: u_new += -dt J^-1 (Dhat F + Dhat G)
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e) {
        const double s = -dt * m.inverse_jacobian[e];
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    const double a = s * lam_in[idx_u(n, v, i, j, e)];
                    for (int k = 0; k < n; ++k) {
                        bF[idx_u(n, v, k, j, e)] += b.Dhat[i * n + k] * a;
                        bG[idx_u(n, v, i, k, e)] += b.Dhat[j * n + k] * a;
                    }
                }
    }
    // interfaces (serial: each element face belongs to one interface, but corners are shared by x and y)
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int le = m.interface_left[k], re = m.interface_right[k], o = m.interface_orientation[k];
        const double sL = -dt * m.inverse_jacobian[le] * b.inv_w_last;
        const double sR = dt * m.inverse_jacobian[re] * b.inv_w_first;
        for (int l = 0; l < n; ++l) {
            const int iL = o == 1 ? n - 1 : l, jL = o == 1 ? l : n - 1;
            const int iR = o == 1 ? 0 : l, jR = o == 1 ? l : 0;
            double uL[NV], uR[NV], UL[NV], UR[NV], bFn[NV];
            for (int v = 0; v < NV; ++v) {
                uL[v] = u[idx_u(n, v, iL, jL, le)];
                uR[v] = u[idx_u(n, v, iR, jR, re)];
                UL[v] = ws.U[idx_u(n, v, iL, jL, le)];
                UR[v] = ws.U[idx_u(n, v, iR, jR, re)];
                bFn[v] = sL * lam_in[idx_u(n, v, iL, jL, le)] + sR * lam_in[idx_u(n, v, iR, jR, re)];
            }
            bool bad = false;
            const double lam = eq.max_abs_speed(UL, UR, o, opt.speed_kind, bad);
            // Fn = (F_L + F_R)/2 - lam/2 (u_R - u_L)
            double* bFL = o == 1 ? &bF[idx_u(n, 0, iL, jL, le)] : &bG[idx_u(n, 0, iL, jL, le)];
            double* bFR = o == 1 ? &bF[idx_u(n, 0, iR, jR, re)] : &bG[idx_u(n, 0, iR, jR, re)];
            double blam = 0.0;
            for (int v = 0; v < NV; ++v) {
                bFL[v] += 0.5 * bFn[v];
                bFR[v] += 0.5 * bFn[v];
                lam_out[idx_u(n, v, iL, jL, le)] += 0.5 * lam * bFn[v];
                lam_out[idx_u(n, v, iR, jR, re)] -= 0.5 * lam * bFn[v];
                blam += -0.5 * bFn[v] * (uR[v] - uL[v]);
            }
            double dvL[NV], dcL[NV], dvR[NV], dcR[NV];
            speed_partials(eq, UL, o, dvL, dcL);
            speed_partials(eq, UR, o, dvR, dcR);
            double rl, v1l, v2l, pl, rr, v1r, v2r, pr;
            eq.cons2prim(UL, rl, v1l, v2l, pl);
            eq.cons2prim(UR, rr, v1r, v2r, pr);
            const double vl = std::fabs(o == 1 ? v1l : v2l), vr = std::fabs(o == 1 ? v1r : v2r);
            const double cl = std::sqrt(eq.gamma * pl / rl), cr = std::sqrt(eq.gamma * pr / rr);
            double* bUL = &bU[idx_u(n, 0, iL, jL, le)];
            double* bUR = &bU[idx_u(n, 0, iR, jR, re)];
            if (opt.speed_kind == 0) {
                // max(|v_L|, |v_R|) + max(c_L, c_R); std::max returns the first argument on ties
                double* bv = vl >= vr ? bUL : bUR;
                const double* dv = vl >= vr ? dvL : dvR;
                double* bc = cl >= cr ? bUL : bUR;
                const double* dc = cl >= cr ? dcL : dcR;
                for (int v = 0; v < NV; ++v) { bv[v] += blam * dv[v]; bc[v] += blam * dc[v]; }
            } else {
                const bool left = vl + cl >= vr + cr;
                double* bs = left ? bUL : bUR;
                const double* dv = left ? dvL : dvR;
                const double* dc = left ? dcL : dcR;
                for (int v = 0; v < NV; ++v) bs[v] += blam * (dv[v] + dc[v]);
            }
        }
    }
    // elements: reverse of the LW procedure
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e) {
        const size_t o = idx_u(n, 0, 0, 0, e);
        lw_volume_element_vjp(b, eq, opt.N, u + o, dt, m.inverse_jacobian[e], &bF[o], &bG[o], &bU[o], lam_out + o);
    }
}

}  // namespace tlwo
