// tlw_curved_parabolic.hpp -- TEST INFRASTRUCTURE ONLY (the oracle): the LW right-hand side of the compressible
// Navier-Stokes equations on a conforming curvilinear mesh (P4estMesh{2}; the reference has no StructuredMesh
// parabolic path), with slip walls for the advective part and no-slip walls for the parabolic part, restated
// on the CPU to check the CUDA kernels.
//
// rhs! for SemidiscretizationHyperbolicParabolic on P4estMesh{2} (src/solvers/dgsem_tree/dg_2d_parabolic.jl:15-99,
// the P4est methods of src/solvers/dgsem_p4est/dg_2d_parabolic.jl):
//   BR1 gradients of the conservative variables (Trixi calc_gradient! for P4estMesh{2}): the weak-form volume
//   term Dhat u along xi and eta mixed by the transposed contravariant vectors (grad_x = Ja^1_1 r_xi + Ja^2_1
//   r_eta, grad_y = Ja^1_2 r_xi + Ja^2_2 r_eta), the face value u* (interface: (u_P + u_S) / 2; boundary: the
//   wall's value, compressible_navier_stokes_2d.jl:92-124) times the element's own outward normal component and
//   1 / w of the face, all times J^{-1} per node;
//   the parabolic LW volume procedure on contravariant fluxes (lw_volume_kernel_3! / _4!, :641-1787);
//   interfaces: the advective LW surface flux in the curvilinear argument order minus the average of the two
//   sides' viscous normal fluxes (prolong2interfaces_lw_parabolic! + calc_interface_flux_hyperbolic_parabolic!,
//   :1788-1958); boundaries: the slip-wall flux minus the wall's viscous flux (prolong2boundaries_visc_lw! +
//   calc_boundary_flux_lw!, :1961-2127);
//   dt = min(cfl max_dt(curvilinear advective), cfl max_dt(parabolic)) (compute_dt, src/solvers/lwfr.jl:192-210).
// The parabolic max_dt (compressible_navier_stokes_2d.jl:204-247) is the TreeMesh formula with
// cache.elements.inverse_jacobian[element]: on a P4estMesh that array is [i, j, element], so Julia's linear
// indexing reads its element-th entry (node i = (e-1) % n + 1, j = ((e-1) / n) % n + 1 of element (e-1) / n^2 + 1),
// not a value of the element itself. The restatement keeps that reading.
#pragma once
#include "tlw_curved.hpp"
#include "tlw_parabolic.hpp"

namespace tlwo {

inline double face_inv_w(const Basis& b, int f) { return (f == 1 || f == 3) ? b.inv_w_last : b.inv_w_first; }

inline void gradients_br1_curved(const Basis& b, const CurvedMesh& m, const NavierStokes& ns, const double* u,
                                 std::vector<double>& gx, std::vector<double>& gy, int nthreads = 1) {
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    gx.assign(ndof, 0.0);
    gy.assign(ndof, 0.0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const double* J = &m.Ja[4 * (i + (size_t)n * (j + (size_t)n * e))];
                for (int v = 0; v < NV; ++v) {
                    double r1 = 0.0, r2 = 0.0;
                    for (int k = 0; k < n; ++k) {
                        r1 += b.Dhat[i * n + k] * u[idx_u(n, v, k, j, e)];
                        r2 += b.Dhat[j * n + k] * u[idx_u(n, v, i, k, e)];
                    }
                    gx[idx_u(n, v, i, j, e)] = J[0] * r1 + J[2] * r2;
                    gy[idx_u(n, v, i, j, e)] = J[1] * r1 + J[3] * r2;
                }
            }
    auto lift = [&](int e, int f, int l, const double* us) {
        int i, j;
        face_node(n, f, l, i, j);
        double nrm[2];
        outward_normal(m, n, f, i, j, e, nrm);
        const double iw = face_inv_w(b, f);
        for (int v = 0; v < NV; ++v) {
            gx[idx_u(n, v, i, j, e)] += us[v] * iw * nrm[0];
            gy[idx_u(n, v, i, j, e)] += us[v] * iw * nrm[1];
        }
    };
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int pe = m.p_elem[k], pf = m.p_face[k], se = m.s_elem[k], sf = m.s_face[k];
        for (int l = 0; l < n; ++l) {
            const int ls = m.s_rev[k] ? n - 1 - l : l;
            int ip, jp, is, js;
            face_node(n, pf, l, ip, jp);
            face_node(n, sf, ls, is, js);
            double us[NV];
            for (int v = 0; v < NV; ++v) us[v] = 0.5 * (u[idx_u(n, v, ip, jp, pe)] + u[idx_u(n, v, is, js, se)]);
            lift(pe, pf, l, us);
            lift(se, sf, ls, us);
        }
    }
    for (int k = 0; k < m.n_boundaries; ++k) {
        const int e = m.b_elem[k], f = m.b_face[k];
        for (int l = 0; l < n; ++l) {
            int i, j;
            face_node(n, f, l, i, j);
            double ui[NV], uo[NV];
            for (int v = 0; v < NV; ++v) ui[v] = u[idx_u(n, v, i, j, e)];
            wall_gradient_value(ns, ns.wall_kind[k], &ns.wall[3 * (l + (size_t)n * k)], ui, uo);
            lift(e, f, l, uo);
        }
    }
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e)
        for (int node = 0; node < nn; ++node) {
            const double ij = m.inv_jac[node + (size_t)nn * e];
            for (int v = 0; v < NV; ++v) {
                gx[(size_t)NV * (node + (size_t)nn * e) + v] *= ij;
                gy[(size_t)NV * (node + (size_t)nn * e) + v] *= ij;
            }
        }
}

inline void rhs_parabolic_curved(const Basis& b, const Euler& eq, const NavierStokes& ns, const Options& opt,
                                 const CurvedMesh& m, const double* u, double* du, double dt, Workspace& ws,
                                 int nthreads = 1) {
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    if (m.n_boundaries > 0 && ns.wall_kind.size() != (size_t)m.n_boundaries)
        throw std::invalid_argument("parabolic oracle: boundaries need wall conditions");
    std::vector<double> gx, gy, Fv(2 * ndof);
    gradients_br1_curved(b, m, ns, u, gx, gy, nthreads);
    ws.U.assign(ndof, 0.0);
    ws.F.assign(2 * ndof, 0.0);
    ws.surface_flux_values.assign((size_t)NV * n * 4 * m.n_elements, 0.0);
    ws.bad = false;
    for (size_t k = 0; k < ndof; ++k) du[k] = 0.0;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e)
        lw_volume_element_parabolic(b, eq, ns, opt.N, e, u, gx.data(), gy.data(), du, dt, 0.0, ws.U.data(),
                                    ws.F.data(), Fv.data(), &m.Ja[4 * (size_t)nn * e], &m.inv_jac[(size_t)nn * e]);
    auto normal_flux = [&](const std::vector<double>& F, int v, int i, int j, int e, const double* nrm) {
        return F[idx_F(n, v, 0, i, j, e)] * nrm[0] + F[idx_F(n, v, 1, i, j, e)] * nrm[1];
    };
    bool bad = false;
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int pe = m.p_elem[k], pf = m.p_face[k], se = m.s_elem[k], sf = m.s_face[k];
        for (int l = 0; l < n; ++l) {
            const int ls = m.s_rev[k] ? n - 1 - l : l;
            int ip, jp, is, js;
            face_node(n, pf, l, ip, jp);
            face_node(n, sf, ls, is, js);
            double nP[2], nS[2], f_ll[NV], f_rr[NV], u_ll[NV], u_rr[NV], U_ll[NV], U_rr[NV], Fn[NV];
            outward_normal(m, n, pf, ip, jp, pe, nP);
            outward_normal(m, n, sf, is, js, se, nS);
            double mS[2] = {-nS[0], -nS[1]};
            for (int v = 0; v < NV; ++v) {
                f_ll[v] = normal_flux(ws.F, v, ip, jp, pe, nP);
                f_rr[v] = normal_flux(ws.F, v, is, js, se, mS);
                u_ll[v] = u[idx_u(n, v, ip, jp, pe)];
                u_rr[v] = u[idx_u(n, v, is, js, se)];
                U_ll[v] = ws.U[idx_u(n, v, ip, jp, pe)];
                U_rr[v] = ws.U[idx_u(n, v, is, js, se)];
            }
            bool b_ = false;
            lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, nP, Fn, b_);
            bad = bad || b_;
            for (int v = 0; v < NV; ++v) {
                const double visc = 0.5 * (normal_flux(Fv, v, ip, jp, pe, nP) + normal_flux(Fv, v, is, js, se, mS));
                const double f = Fn[v] - visc;
                ws.surface_flux_values[v + NV * (l + n * (pf + 4 * (size_t)pe))] = f;
                ws.surface_flux_values[v + NV * (ls + n * (sf + 4 * (size_t)se))] = -f;
            }
        }
    }
    ws.bad = bad;
    calc_boundary_flux_curved(b, eq, opt, m, u, ws);
    for (int k = 0; k < m.n_boundaries; ++k) {
        const int e = m.b_elem[k], f = m.b_face[k];
        for (int l = 0; l < n; ++l) {
            int i, j;
            face_node(n, f, l, i, j);
            double nrm[2], fi[NV], fo[NV];
            outward_normal(m, n, f, i, j, e, nrm);
            for (int v = 0; v < NV; ++v) fi[v] = normal_flux(Fv, v, i, j, e, nrm);
            wall_viscous_flux(ns.wall_kind[k], &ns.wall[3 * (l + (size_t)n * k)], fi, fo);
            for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * (f + 4 * (size_t)e))] -= fo[v];
        }
    }
    surface_integral_and_jacobian_curved(b, m, du, ws, nthreads);
}

inline double max_dt_parabolic_curved(const Basis& b, const Euler& eq, const NavierStokes& ns, const CurvedMesh& m,
                                      const double* u, double cfl, bool& bad, int nthreads = 1) {
    const int n = b.n, N = n - 1;
    const double dt_adv = max_dt_curved(b, eq, m, u, cfl, bad, nthreads);
    double lam_a = std::nextafter(0.0, 1.0), lam_v = std::nextafter(0.0, 1.0);
    bool bad_any = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(max : lam_a, lam_v) reduction(|| : bad_any)
    for (int e = 0; e < m.n_elements; ++e) {
        double m1 = 0.0, m2 = 0.0;
        bool b_ = false;
        const double ij = m.inv_jac[e];   // Julia linear indexing of the [i, j, element] array
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
    bad = bad || bad_any;
    const double dt_visc = cfl / ((lam_a + lam_v * 2.0 * (2.0 * N + 1.0)) * (2.0 * (2.0 * N + 1.0)));
    return std::min(dt_adv, dt_visc);
}

}  // namespace tlwo
