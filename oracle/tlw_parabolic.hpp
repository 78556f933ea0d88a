// tlw_parabolic.hpp -- test infrastructure only: CPU restatement of the LW right-hand side of the compressible
// Navier-Stokes equations on a periodic TreeMesh{2}, used to check the CUDA parabolic kernels.
//
// rhs! for SemidiscretizationHyperbolicParabolic (src/solvers/dgsem_tree/dg_2d_parabolic.jl:15-99):
//   gradients of the conservative variables by BR1 (Trixi calc_gradient!: weak-form volume term Dhat u, the
//   interface average (u_L + u_R) / 2 lifted with 1 / w, times +J^{-1}) -> gradient variables are the
//   conservative ones (GradientVariablesConservative, src/equations/compressible_navier_stokes_2d.jl:14-57);
//   viscous fluxes at t^n (Trixi calc_viscous_fluxes!); the LW volume kernels lw_volume_kernel_3! / _4!
//   (dg_2d_parabolic.jl:725-1189, 1191-1860): the procedure of the hyperbolic kernels with the flux
//   f - f_v(u, grad u), the perturbed states u +- ut ... carried together with their gradients
//   grad u +- grad ut ... (grad ut = J^{-1} D ut), time averages Fa (advective) and Fv (viscous) kept apart,
//   du = Dhat (Fa - Fv) + Dhat (Ga - Gv);
//   interface flux = LW surface flux of the advective traces (TreeMesh order) - (Fv_L + Fv_R) / 2
//   (calc_interface_flux_hyperbolic_parabolic!, dg_2d_parabolic.jl:1911-1949); surface integral, Jacobian.
//   Viscous flux (Trixi CompressibleNavierStokesDiffusion2D, T = p / rho): the primitive derivatives of the
//   conservative gradients (convert_derivative_to_primitive, compressible_navier_stokes_2d.jl:36-57),
//   tau_11 = 4/3 v1_x - 2/3 v2_y, tau_12 = v1_y + v2_x, tau_22 = 4/3 v2_y - 2/3 v1_x, q = kappa grad T with
//   kappa = gamma / ((gamma - 1) Pr), f_v = mu (0, tau_11, tau_12, v1 tau_11 + v2 tau_12 + q_1), g_v alike.
//   dt = min(cfl max_dt(hyperbolic), cfl max_dt(parabolic)) (compute_dt, src/solvers/lwfr.jl:192-210; the
//   parabolic max_dt, compressible_navier_stokes_2d.jl:204-261).
#pragma once
#include "tlw_adjoint.hpp"
#include "tlw_oracle.hpp"

namespace tlwo {

// Wall conditions of the parabolic part per boundary: BoundaryConditionNavierStokesWall(NoSlip(v), Adiabatic(q))
// or (NoSlip(v), Isothermal(T)), src/equations/compressible_navier_stokes_2d.jl:81-124; wall data per
// boundary node [3, l, B] = (v1, v2, q or T) at the boundary's node coordinates.
enum WallKind { WALL_NONE = 0, WALL_ADIABATIC = 1, WALL_ISOTHERMAL = 2 };

struct NavierStokes {
    double gamma = 1.4, mu = 0.0, Pr = 0.72;
    std::vector<int32_t> wall_kind;   // [B]
    std::vector<double> wall;         // [3, l, B]
    double kappa() const { return gamma / ((gamma - 1.0) * Pr); }
};

// the face node (i, j) of boundary k's element, face index l
inline void boundary_node(const TreeMesh& m, int n, int k, int l, int& i, int& j) {
    const int o = m.boundary_orientation[k], side = m.boundary_side[k];
    if (o == 1) { i = side == 1 ? n - 1 : 0; j = l; } else { i = l; j = side == 1 ? n - 1 : 0; }
}

// the gradient's boundary value (operator Gradient): prim2cons(rho_inner, v_wall, p) with p the inner
// pressure (Adiabatic, :113-124) or rho_inner T_wall (Isothermal, :92-100)
inline void wall_gradient_value(const NavierStokes& ns, int kind, const double* w, const double* ui, double* uo) {
    const double rho = ui[0];
    const double p = kind == WALL_ADIABATIC
                         ? (ns.gamma - 1.0) * (ui[3] - 0.5 * (ui[1] * ui[1] + ui[2] * ui[2]) / rho)
                         : rho * w[2];
    uo[0] = rho;
    uo[1] = rho * w[0];
    uo[2] = rho * w[1];
    uo[3] = p / (ns.gamma - 1.0) + 0.5 * rho * (w[0] * w[0] + w[1] * w[1]);
}

// the viscous boundary flux (operator Divergence) from the inner normal viscous flux trace: Adiabatic keeps
// its momentum components and sets the energy flux to v_wall . tau_n + q (:81-90); Isothermal keeps it (:102-108)
inline void wall_viscous_flux(int kind, const double* w, const double* fi, double* fo) {
    for (int v = 0; v < NV; ++v) fo[v] = fi[v];
    if (kind == WALL_ADIABATIC) fo[3] = w[0] * fi[1] + w[1] * fi[2] + w[2];
}

// viscous flux pair of state u with conservative gradients gx, gy
inline void viscous_fluxes(const NavierStokes& ns, const double* u, const double* gx, const double* gy, double* fv,
                           double* gv) {
    const double rho = u[0], v1 = u[1] / rho, v2 = u[2] / rho;
    const double p = (ns.gamma - 1.0) * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    const double T = p / rho;
    auto prim = [&](const double* W, double& v1d, double& v2d, double& Td) {
        const double rd = W[0];
        v1d = (W[1] - rd * v1) / rho;
        v2d = (W[2] - rd * v2) / rho;
        const double pd = (W[3] - 0.5 * rd * (v1 * v1 + v2 * v2) - rho * (v1 * v1d + v2 * v2d)) * (ns.gamma - 1.0);
        Td = (pd - rd * T) / rho;
    };
    double v1x, v2x, Tx, v1y, v2y, Ty;
    prim(gx, v1x, v2x, Tx);
    prim(gy, v1y, v2y, Ty);
    const double t11 = 4.0 / 3.0 * v1x - 2.0 / 3.0 * v2y;
    const double t12 = v1y + v2x;
    const double t22 = 4.0 / 3.0 * v2y - 2.0 / 3.0 * v1x;
    const double k = ns.kappa();
    fv[0] = 0.0; fv[1] = t11 * ns.mu; fv[2] = t12 * ns.mu; fv[3] = (v1 * t11 + v2 * t12 + k * Tx) * ns.mu;
    gv[0] = 0.0; gv[1] = t12 * ns.mu; gv[2] = t22 * ns.mu; gv[3] = (v1 * t12 + v2 * t22 + k * Ty) * ns.mu;
}

// BR1 gradients of the conservative variables: g_d = J^{-1} (Dhat u + lifted interface averages)
inline void gradients_br1(const Basis& b, const TreeMesh& m, const NavierStokes& ns, const double* u,
                          std::vector<double>& gx, std::vector<double>& gy, int nthreads = 1) {
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    gx.assign(ndof, 0.0);
    gy.assign(ndof, 0.0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    double sx = 0.0, sy = 0.0;
                    for (int k = 0; k < n; ++k) {
                        sx += b.Dhat[i * n + k] * u[idx_u(n, v, k, j, e)];
                        sy += b.Dhat[j * n + k] * u[idx_u(n, v, i, k, e)];
                    }
                    gx[idx_u(n, v, i, j, e)] = sx;
                    gy[idx_u(n, v, i, j, e)] = sy;
                }
    // interfaces: BR1 flux (u_L + u_R) / 2; x-interfaces touch gx only, y-interfaces gy only
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int le = m.interface_left[k], re = m.interface_right[k], o = m.interface_orientation[k];
        std::vector<double>& g = o == 1 ? gx : gy;
        for (int l = 0; l < n; ++l) {
            const int iL = o == 1 ? n - 1 : l, jL = o == 1 ? l : n - 1;
            const int iR = o == 1 ? 0 : l, jR = o == 1 ? l : 0;
            for (int v = 0; v < NV; ++v) {
                const double us = 0.5 * (u[idx_u(n, v, iL, jL, le)] + u[idx_u(n, v, iR, jR, re)]);
                g[idx_u(n, v, iL, jL, le)] += us * b.inv_w_last;
                g[idx_u(n, v, iR, jR, re)] -= us * b.inv_w_first;
            }
        }
    }
    // boundaries (Trixi calc_boundary_flux_by_direction_gradient!): the wall value itself is the flux
    for (int k = 0; k < m.n_boundaries; ++k) {
        const int e = m.boundary_element[k], o = m.boundary_orientation[k], side = m.boundary_side[k];
        std::vector<double>& g = o == 1 ? gx : gy;
        for (int l = 0; l < n; ++l) {
            int i, j;
            boundary_node(m, n, k, l, i, j);
            double ui[NV], uo[NV];
            for (int v = 0; v < NV; ++v) ui[v] = u[idx_u(n, v, i, j, e)];
            wall_gradient_value(ns, ns.wall_kind[k], &ns.wall[3 * (l + (size_t)n * k)], ui, uo);
            for (int v = 0; v < NV; ++v) {
                if (side == 1) g[idx_u(n, v, i, j, e)] += uo[v] * b.inv_w_last;    // the boundary at the +face
                else g[idx_u(n, v, i, j, e)] -= uo[v] * b.inv_w_first;             // at the -face
            }
        }
    }
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e)
        for (int k = 0; k < NV * nn; ++k) {
            gx[(size_t)NV * nn * e + k] *= m.inverse_jacobian[e];
            gy[(size_t)NV * nn * e + k] *= m.inverse_jacobian[e];
        }
}

// one element of the parabolic LW volume kernel (depth 3 for N = 3, 4 for N >= 4); du += Dhat (F, G);
// Ua = time-averaged U, Fa = advective [v, d, i, j], Fv = viscous time averages
// On a curvilinear mesh (Jae = the element's contravariant vectors [4, i, j], ije = its inverse Jacobian per
// node; src/solvers/dgsem_p4est/dg_2d_parabolic.jl:1190-1787): the stage fluxes are the contravariant ones
// Ja^1 . (f_a - f_v, g_a - g_v), Ja^2 . (...), d_m carries the per-node J^{-1}, and its gradient is
// J^{-1} (Ja^1_d D_xi d_m + Ja^2_d D_eta d_m) (compute_local_grad_u!, :51-104); Fao / Fvo stay physical.
inline void lw_volume_element_parabolic(const Basis& b, const Euler& eq, const NavierStokes& ns, int N, int e,
                                        const double* u, const double* gx, const double* gy, double* du, double dt,
                                        double ij, double* Uo, double* Fao, double* Fvo,
                                        const double* Jae = nullptr, const double* ije = nullptr) {
    const int n = b.n, nn = n * n;
    const LWStencils S = lw_stencils(N);
    const int depth = S.depth;
    auto L = [&](int i, int j) { return NV * (i + n * j); };
    const double* ue = u + idx_u(n, 0, 0, 0, e);
    const double* gxe = gx + idx_u(n, 0, 0, 0, e);
    const double* gye = gy + idx_u(n, 0, 0, 0, e);
    // d[m], its gradients dx[m], dy[m] (m = 1..depth)
    std::vector<double> d(5 * NV * nn, 0.0), dx(5 * NV * nn, 0.0), dy(5 * NV * nn, 0.0);
    std::vector<double> ft(NV * nn), gt(NV * nn), Fa(NV * nn), Ga(NV * nn), Fv(NV * nn), Gv(NV * nn), U(NV * nn);
    auto at = [&](std::vector<double>& a, int m) { return a.data() + (size_t)m * NV * nn; };
    // all fluxes of a state with gradients
    auto all_fluxes = [&](const double* s, const double* sx, const double* sy, double* fa, double* ga, double* fv,
                          double* gv) {
        eq.fluxes(s, fa, ga);
        viscous_fluxes(ns, s, sx, sy, fv, gv);
    };
    auto ijn = [&](int i, int j) { return Jae ? ije[i + n * j] : ij; };
    // the stage flux pair along the reference coordinates: contravariant on a curvilinear mesh
    auto contra = [&](int i, int j, double f, double g, double& cf, double& cg) {
        if (!Jae) { cf = f; cg = g; return; }
        const double* J = Jae + 4 * (i + n * j);
        cf = J[0] * f + J[1] * g;
        cg = J[2] * f + J[3] * g;
    };
    auto next = [&](int m) {
        // d_m = -dt J^{-1} (D ft + D gt); grad d_m = J^{-1} (D d_m along i, along j), mixed by the metrics
        double* dm = at(d, m);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    double s = 0.0;
                    for (int k = 0; k < n; ++k) s += b.D[i * n + k] * ft[L(k, j) + v] + b.D[j * n + k] * gt[L(i, k) + v];
                    dm[L(i, j) + v] = -dt * ijn(i, j) * s;
                }
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    double sx = 0.0, sy = 0.0;
                    for (int k = 0; k < n; ++k) {
                        sx += b.D[i * n + k] * dm[L(k, j) + v];
                        sy += b.D[j * n + k] * dm[L(i, k) + v];
                    }
                    if (Jae) {
                        const double* J = Jae + 4 * (i + n * j);
                        at(dx, m)[L(i, j) + v] = ijn(i, j) * (J[0] * sx + J[2] * sy);
                        at(dy, m)[L(i, j) + v] = ijn(i, j) * (J[1] * sx + J[3] * sy);
                    } else {
                        at(dx, m)[L(i, j) + v] = ij * sx;
                        at(dy, m)[L(i, j) + v] = ij * sy;
                    }
                }
    };
    auto state = [&](int s, int q, int o, double* P, double* Px, double* Py) {
        for (int v = 0; v < NV; ++v) {
            double x = ue[o + v], y = gxe[o + v], z = gye[o + v];
            for (int m = 1; m <= s; ++m) {
                x += S.a[q][m] * at(d, m)[o + v];
                y += S.a[q][m] * at(dx, m)[o + v];
                z += S.a[q][m] * at(dy, m)[o + v];
            }
            P[v] = x; Px[v] = y; Py[v] = z;
        }
    };
    // stage 0
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            double fa[NV], ga[NV], fv[NV], gv[NV];
            all_fluxes(ue + o, gxe + o, gye + o, fa, ga, fv, gv);
            for (int v = 0; v < NV; ++v) {
                Fa[o + v] = fa[v]; Ga[o + v] = ga[v]; Fv[o + v] = fv[v]; Gv[o + v] = gv[v];
                contra(i, j, fa[v] - fv[v], ga[v] - gv[v], ft[o + v], gt[o + v]);
                U[o + v] = ue[o + v];
            }
        }
    next(1);
    for (int s = 1; s <= depth; ++s) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double fa[NV], ga[NV], fv[NV], gv[NV];
                double sfa[NV] = {0, 0, 0, 0}, sga[NV] = {0, 0, 0, 0}, sfv[NV] = {0, 0, 0, 0}, sgv[NV] = {0, 0, 0, 0};
                if (S.w[s][0] != 0.0) {
                    all_fluxes(ue + o, gxe + o, gye + o, fa, ga, fv, gv);
                    for (int v = 0; v < NV; ++v) {
                        sfa[v] = S.w[s][0] * fa[v]; sga[v] = S.w[s][0] * ga[v];
                        sfv[v] = S.w[s][0] * fv[v]; sgv[v] = S.w[s][0] * gv[v];
                    }
                }
                for (int q = 0; q < 4; ++q) {
                    if (S.w[s][1 + q] == 0.0) continue;
                    double P[NV], Px[NV], Py[NV];
                    state(s, q, o, P, Px, Py);
                    all_fluxes(P, Px, Py, fa, ga, fv, gv);
                    for (int v = 0; v < NV; ++v) {
                        sfa[v] += S.w[s][1 + q] * fa[v]; sga[v] += S.w[s][1 + q] * ga[v];
                        sfv[v] += S.w[s][1 + q] * fv[v]; sgv[v] += S.w[s][1 + q] * gv[v];
                    }
                }
                for (int v = 0; v < NV; ++v) {
                    Fa[o + v] += S.tw[s] * sfa[v]; Ga[o + v] += S.tw[s] * sga[v];
                    Fv[o + v] += S.tw[s] * sfv[v]; Gv[o + v] += S.tw[s] * sgv[v];
                    U[o + v] += S.tw[s] * at(d, s)[o + v];
                    contra(i, j, sfa[v] - sfv[v], sga[v] - sgv[v], ft[o + v], gt[o + v]);
                }
            }
        if (s < depth) next(s + 1);
    }
    double* due = du + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            double cf[NV], cg[NV];
            for (int v = 0; v < NV; ++v) contra(i, j, Fa[o + v] - Fv[o + v], Ga[o + v] - Gv[o + v], cf[v], cg[v]);
            for (int ii = 0; ii < n; ++ii)
                for (int v = 0; v < NV; ++v) due[L(ii, j) + v] += b.Dhat[ii * n + i] * cf[v];
            for (int jj = 0; jj < n; ++jj)
                for (int v = 0; v < NV; ++v) due[L(i, jj) + v] += b.Dhat[jj * n + j] * cg[v];
            for (int v = 0; v < NV; ++v) {
                Uo[idx_u(n, v, i, j, e)] = U[o + v];
                Fao[idx_F(n, v, 0, i, j, e)] = Fa[o + v];
                Fao[idx_F(n, v, 1, i, j, e)] = Ga[o + v];
                Fvo[idx_F(n, v, 0, i, j, e)] = Fv[o + v];
                Fvo[idx_F(n, v, 1, i, j, e)] = Gv[o + v];
            }
        }
}

// du = rhs(u) for compressible Navier-Stokes on a periodic TreeMesh{2} (LW)
inline void rhs_parabolic(const Basis& b, const Euler& eq, const NavierStokes& ns, const Options& opt,
                          const TreeMesh& m, const double* u, double* du, double dt, Workspace& ws, int nthreads = 1,
                          const BoundaryData* bd = nullptr) {
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    if (m.n_mortars > 0) throw std::invalid_argument("parabolic oracle: conforming mesh");
    if (m.n_boundaries > 0 && ns.wall_kind.size() != (size_t)m.n_boundaries)
        throw std::invalid_argument("parabolic oracle: boundaries need wall conditions");
    std::vector<double> gx, gy, Fv(2 * ndof);
    gradients_br1(b, m, ns, u, gx, gy, nthreads);
    ws.U.assign(ndof, 0.0);
    ws.F.assign(2 * ndof, 0.0);
    ws.surface_flux_values.assign((size_t)NV * n * 4 * m.n_elements, 0.0);
    ws.bad = false;
    for (size_t k = 0; k < ndof; ++k) du[k] = 0.0;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e)
        lw_volume_element_parabolic(b, eq, ns, opt.N, e, u, gx.data(), gy.data(), du, dt, m.inverse_jacobian[e],
                                    ws.U.data(), ws.F.data(), Fv.data());
    bool bad = false;
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int le = m.interface_left[k], re = m.interface_right[k], o = m.interface_orientation[k];
        const int d = o - 1;
        for (int l = 0; l < n; ++l) {
            const int iL = o == 1 ? n - 1 : l, jL = o == 1 ? l : n - 1;
            const int iR = o == 1 ? 0 : l, jR = o == 1 ? l : 0;
            double Ul[NV], Ur[NV], ul[NV], ur[NV], fl[NV], fr[NV], Fn[NV];
            for (int v = 0; v < NV; ++v) {
                Ul[v] = ws.U[idx_u(n, v, iL, jL, le)]; Ur[v] = ws.U[idx_u(n, v, iR, jR, re)];
                ul[v] = u[idx_u(n, v, iL, jL, le)]; ur[v] = u[idx_u(n, v, iR, jR, re)];
                fl[v] = ws.F[idx_F(n, v, d, iL, jL, le)]; fr[v] = ws.F[idx_F(n, v, d, iR, jR, re)];
            }
            bool b_ = false;
            lw_surface_flux(eq, opt.flux_kind, opt.speed_kind, fl, fr, Ul, Ur, ul, ur, o, Fn, b_);
            bad = bad || b_;
            for (int v = 0; v < NV; ++v) {
                const double visc = 0.5 * (Fv[idx_F(n, v, d, iL, jL, le)] + Fv[idx_F(n, v, d, iR, jR, re)]);
                const double f = Fn[v] - visc;
                ws.surface_flux_values[v + NV * (l + n * ((2 * o - 1) + 4 * (size_t)le))] = f;
                ws.surface_flux_values[v + NV * (l + n * ((2 * o - 2) + 4 * (size_t)re))] = f;
            }
        }
    }
    ws.bad = bad;
    if (m.n_boundaries > 0) {
        // the advective boundary flux (calc_boundary_flux!), then minus the wall's viscous flux
        // (prolong2boundaries_visc_lw! + calc_boundary_flux_divergence_lw!, dg_2d_parabolic.jl:1951-2084)
        if (has_dirichlet_boundaries(m) && (!bd || !bd->u_levels || !bd->u_now))
            throw std::invalid_argument("boundary data missing");
        calc_boundary_flux(b, eq, opt, m, u, bd ? *bd : BoundaryData{}, 1.0, ws);
        for (int k = 0; k < m.n_boundaries; ++k) {
            const int e = m.boundary_element[k], o = m.boundary_orientation[k], dir = m.boundary_direction[k];
            for (int l = 0; l < n; ++l) {
                int i, j;
                boundary_node(m, n, k, l, i, j);
                double fi[NV], fo[NV];
                for (int v = 0; v < NV; ++v) fi[v] = Fv[idx_F(n, v, o - 1, i, j, e)];
                wall_viscous_flux(ns.wall_kind[k], &ns.wall[3 * (l + (size_t)n * k)], fi, fo);
                for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * ((dir - 1) + 4 * (size_t)e))] -= fo[v];
            }
        }
    }
    surface_integral_and_jacobian(b, m, du, ws, nthreads);
}

// dt = min(cfl max_dt(hyperbolic), cfl max_dt(parabolic))
inline double max_dt_parabolic(const Basis& b, const Euler& eq, const NavierStokes& ns, const TreeMesh& m,
                               const double* u, double cfl, bool& bad, int nthreads = 1) {
    const int n = b.n, N = n - 1;
    double lam_a = std::nextafter(0.0, 1.0), lam_v = std::nextafter(0.0, 1.0);
    bool bad_any = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(max : lam_a, lam_v) reduction(|| : bad_any)
    for (int e = 0; e < m.n_elements; ++e) {
        double m1 = 0.0, m2 = 0.0;
        bool b_ = false;
        const double ij = m.inverse_jacobian[e];
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double l1, l2;
                eq.max_abs_speeds(u + idx_u(n, 0, i, j, e), l1, l2, b_);
                m1 = std::max(m1, l1);
                m2 = std::max(m2, l2);
                const double rho = u[idx_u(n, 0, i, j, e)];
                lam_v = std::max(lam_v, ij * ij * std::max(4.0 * ns.mu / (3.0 * rho), ns.mu * ns.kappa() / (rho * ns.Pr)));
            }
        lam_a = std::max(lam_a, ij * (m1 + m2));
        bad_any = bad_any || b_;
    }
    bad = bad_any;
    const double dt_adv = cfl * 2.0 / (n * lam_a);
    const double dt_visc = cfl / ((lam_a + lam_v * 2.0 * (2.0 * N + 1.0)) * (2.0 * (2.0 * N + 1.0)));
    return std::min(dt_adv, dt_visc);
}

}  // namespace tlwo
