// tlw_curved.hpp -- test infrastructure only: CPU restatement of the LW right-hand side on curvilinear
// conforming meshes (StructuredMesh{2}, and P4estMesh{2} / UnstructuredMesh2D without mortars), used to
// check the CUDA curvilinear kernels.
//
// Volume: lw_volume_kernel_3! / lw_volume_kernel_4! for Union{StructuredMesh{2}, UnstructuredMesh2D,
// P4estMesh{2}} (src/solvers/dgsem_structured/dg_2d.jl:1379-1685, 1687-2105): the LW procedure of the
// TreeMesh kernels applied to the contravariant fluxes f~ = Ja^1 . (f, g), g~ = Ja^2 . (f, g)
// (contravariant_flux, :541-556) with the per-node inverse Jacobian; the element cache keeps the
// physical time averages F, G for the surface; du = Dhat F~ + Dhat G~.
// Surface: every conforming interface is (primary element, face; secondary element, face; whether the
// secondary's face index runs backwards). The normal is the primary's outward contravariant vector at the
// face node (get_normal_direction); each side's normal flux uses its own outward normal, the secondary's
// negated (prolong2interfaces!, src/solvers/dgsem_p4est/dg_2d.jl:8-84), and the 8-argument surface flux is
// called in the curvilinear order (f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, normal) (dgsem_p4est/dg_2d.jl:165,
// dgsem_structured/dg_2d.jl:2271): for Rusanov the speed comes from the instantaneous u and the jump is
// in the time-averaged U. The primary receives Fn and the secondary -Fn as outward fluxes
// (dgsem_p4est/dg_2d.jl:176-189). A StructuredMesh interface is given with the right element as primary
// (its -x / -y face), which is the normal the StructuredMesh code takes (dgsem_structured/dg_2d.jl:2233-2267).
// Surface integral and apply_jacobian (Trixi): du(face node) += outward flux / w_face, then du *= -J^{-1}
// per node. max_dt (Trixi, curved meshes): 2 / (n max_e max_nodes(|Ja^1 . lambda| J^{-1}) + ...).
// Faces are numbered 0: -xi (i = 1), 1: +xi (i = n), 2: -eta (j = 1), 3: +eta (j = n).
#pragma once
#include "tlw_adjoint.hpp"
#include "tlw_oracle.hpp"

namespace tlwo {

struct CurvedMesh {
    int n_elements = 0;
    std::vector<double> Ja;         // [4, i, j, e]: Ja^1_1, Ja^1_2, Ja^2_1, Ja^2_2 (Trixi contravariant_vectors)
    std::vector<double> inv_jac;    // [i, j, e]
    int n_interfaces = 0;
    std::vector<int32_t> p_elem, p_face, s_elem, s_face, s_rev;   // 0-based elements
    // boundary faces (P4estMesh boundaries: element, face) with their condition (BC_SLIP_WALL_*)
    int n_boundaries = 0;
    std::vector<int32_t> b_elem, b_face, b_kind;
    // L2 mortars (P4estMesh): two small elements (positions 1, 2 along the large face's forward index) on their
    // face m_sface, the large element on m_lface, whose index runs backwards along the mortar when m_lrev
    int n_mortars = 0;
    std::vector<int32_t> m_small1, m_small2, m_sface, m_large, m_lface, m_lrev;
    // lw_mortars.inverse_jacobian [mortar][l] (the J^{-1} of the shock-capturing blend at the mortars); empty:
    // zeros, as the reference holds them until an AMR step loads them
    std::vector<double> m_ij;
    // UnstructuredMesh2D: the caller's outward normals (Trixi elements.normal_directions) by face, [2, l, face, e];
    // empty for StructuredMesh / P4estMesh. The interfaces are then in the unstructured conventions below.
    std::vector<double> unormals;
};

// UnstructuredMesh2D sides (1: bottom j = 1, 2: right i = n, 3: top j = n, 4: left i = 1) as faces, and the
// fn_low slot of a face (load_fn_low! for UnstructuredMesh2D / P4estMesh{2}: bottom, right, top, left,
// src/solvers/dgsem_tree/dg_2d.jl:236-249), which the unstructured path reads by side
inline int face_of_side(int side) { return side == 1 ? 2 : side == 2 ? 1 : side == 3 ? 3 : 0; }
inline int fn_low_slot(int face) { return face == 0 ? 3 : face == 1 ? 1 : face == 2 ? 0 : 2; }


// node (i, j) of face f at face index l
inline void face_node(int n, int f, int l, int& i, int& j) {
    switch (f) {
        case 0: i = 0; j = l; break;
        case 1: i = n - 1; j = l; break;
        case 2: i = l; j = 0; break;
        default: i = l; j = n - 1; break;
    }
}

// outward normal of face f at node (i, j): -+Ja^1 on xi faces, -+Ja^2 on eta faces (get_normal_direction)
inline void outward_normal(const CurvedMesh& m, int n, int f, int i, int j, int e, double* nrm) {
    const double* J = &m.Ja[4 * (i + (size_t)n * (j + (size_t)n * e))];
    const double s = (f == 1 || f == 3) ? 1.0 : -1.0;
    nrm[0] = s * (f < 2 ? J[0] : J[2]);
    nrm[1] = s * (f < 2 ? J[1] : J[3]);
}

// Trixi max_abs_speed_naive / max_abs_speed / min_max_speed_naive with a normal direction
inline double max_abs_speed_normal(const Euler& eq, const double* ul, const double* ur, const double* nrm, int kind,
                                   bool& bad) {
    double rl, v1l, v2l, pl, rr, v1r, v2r, pr;
    eq.cons2prim(ul, rl, v1l, v2l, pl);
    eq.cons2prim(ur, rr, v1r, v2r, pr);
    const double vl = v1l * nrm[0] + v2l * nrm[1], vr = v1r * nrm[0] + v2r * nrm[1];
    const double cl = eq.checked_sqrt(eq.gamma * pl / rl, bad), cr = eq.checked_sqrt(eq.gamma * pr / rr, bad);
    const double nn = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
    if (kind == 0) return std::max(std::fabs(vl), std::fabs(vr)) + std::max(cl, cr) * nn;
    return std::max(std::fabs(vl) + cl * nn, std::fabs(vr) + cr * nn);
}
inline void min_max_speed_normal(const Euler& eq, const double* ul, const double* ur, const double* nrm, double& lmin,
                                 double& lmax, bool& bad) {
    double rl, v1l, v2l, pl, rr, v1r, v2r, pr;
    eq.cons2prim(ul, rl, v1l, v2l, pl);
    eq.cons2prim(ur, rr, v1r, v2r, pr);
    const double nn = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
    lmin = (v1l * nrm[0] + v2l * nrm[1]) - eq.checked_sqrt(eq.gamma * pl / rl, bad) * nn;
    lmax = (v1r * nrm[0] + v2r * nrm[1]) + eq.checked_sqrt(eq.gamma * pr / rr, bad) * nn;
}

// the 8-argument LW surface flux (numerical_fluxes.jl:14-38, compressible_euler_2d.jl:24-40) with a normal
inline void lw_surface_flux_normal(const Euler& eq, int flux_kind, int speed_kind, const double* f_ll,
                                   const double* f_rr, const double* a3, const double* a4, const double* a5,
                                   const double* a6, const double* nrm, double* out, bool& bad) {
    if (flux_kind == RUSANOV) {
        const double lambda = max_abs_speed_normal(eq, a3, a4, nrm, speed_kind, bad);
        for (int v = 0; v < NV; ++v) out[v] = 0.5 * (f_ll[v] + f_rr[v]) + (-0.5 * lambda * (a6[v] - a5[v]));
    } else {
        double lmin, lmax;
        min_max_speed_normal(eq, a5, a6, nrm, lmin, lmax, bad);
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

// One interface node of an UnstructuredMesh2D (prolong2interfaces! and calc_interface_flux!,
// src/solvers/dgsem_unstructured_2d/dg_2d.jl:60-280): the normal is the caller's outward normal of the primary at
// its node l (normal_directions); both sides' normal fluxes are the physical time-averaged flux dotted with that
// normal (the secondary node s(l) = start_index + (l - 1) index_increment is prolonged with the primary's normal at
// its own secondary index, which is the primary's node l); the 8-argument surface flux takes the curvilinear order
// (f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, normal). Returns the primary's outward flux Fn_ (before any blending) and,
// for shock capturing, the first-order flux fn = surface_flux(u_ll, u_rr, normal).
inline void unstructured_interface_node(const Euler& eq, const Options& opt, const CurvedMesh& m, int n, const double* u,
                                        const Workspace& ws, int pe, int pf, int se, int sf, int l, int ls,
                                        double* nP, double* Fn_, double* u_ll, double* u_rr, double* U_ll,
                                        double* U_rr, bool& bad) {
    int ip, jp, is, js;
    face_node(n, pf, l, ip, jp);
    face_node(n, sf, ls, is, js);
    nP[0] = m.unormals[2 * (l + (size_t)n * (pf + 4 * (size_t)pe))];
    nP[1] = m.unormals[2 * (l + (size_t)n * (pf + 4 * (size_t)pe)) + 1];
    double f_ll[NV], f_rr[NV];
    for (int v = 0; v < NV; ++v) {
        // normal_product(f, equations, n) = F[1] n[1] + F[2] n[2] (src/solvers/fr.jl:146-150)
        f_ll[v] = ws.F[idx_F(n, v, 0, ip, jp, pe)] * nP[0] + ws.F[idx_F(n, v, 1, ip, jp, pe)] * nP[1];
        f_rr[v] = ws.F[idx_F(n, v, 0, is, js, se)] * nP[0] + ws.F[idx_F(n, v, 1, is, js, se)] * nP[1];
        u_ll[v] = u[idx_u(n, v, ip, jp, pe)];
        u_rr[v] = u[idx_u(n, v, is, js, se)];
        U_ll[v] = ws.U[idx_u(n, v, ip, jp, pe)];
        U_rr[v] = ws.U[idx_u(n, v, is, js, se)];
    }
    lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, nP, Fn_, bad);
}

// One element of the curvilinear LW volume kernel. du receives Dhat F~ + Dhat G~ (before the surface
// integral and the Jacobian); ws.U / ws.F receive the time-averaged U and the physical F, G.
// alpha: the factor of the Dhat terms (1 - the element's blending factor under shock capturing).
// te: with te->temporal_errors, the error estimate of the Adaptive step control as the curvilinear kernels
// compute it inline (dgsem_structured/dg_2d.jl:1595-1619, 1669-1682 at depth 3; :1983-2007, 2061-2075 at
// depth 4): u_np1 = u - dt J^{-1}(node) (D F~ + D G~) and u_np1_low with F~, G~ before the last stage's term,
// ws.temporal_errors[e] = sum over nodes and variables of ((u_np1 - u_np1_low) / (abstol + reltol max))^2.
// It does not depend on alpha: the shock-capturing path calls the same kernel for every element.
// Source terms (opt->source, the FR volume integral; dgsem_structured/dg_2d.jl:578-964, 1379-2058): each derivative
// gets dt times its stencil of the states before it (at depth 4 the second derivative's is the 5-point
// calc_source_tt_N4, where the TreeMesh kernel takes N23), S = s + s_t/2 + s_tt/6 + s_ttt/24 (+ s_tttt/120) enters
// du unscaled by the node's J^{-1}. The built source does not depend on u, so the stencils are taken by time offsets.
inline void lw_volume_element_curved(const Basis& b, const Euler& eq, int N, const CurvedMesh& m, int e,
                                     const double* u, double* du, double dt, Workspace& ws, double alpha = 1.0,
                                     const Options* te = nullptr, double t = 0.0) {
    const int n = b.n, nn = n * n;
    const LWStencils S = lw_stencils(N);
    const int depth = S.depth;
    auto L = [&](int i, int j) { return NV * (i + n * j); };
    const double* ue = u + idx_u(n, 0, 0, 0, e);
    const double* Jae = &m.Ja[4 * (size_t)nn * e];
    const double* ije = &m.inv_jac[(size_t)nn * e];
    std::vector<double> d(5 * NV * nn, 0.0), ft(NV * nn), gt(NV * nn), Fp(NV * nn), Gp(NV * nn), Ft(NV * nn),
        Gt(NV * nn), Uc(NV * nn), Flow, Glow;
    const bool want_te = te && te->temporal_errors;
    auto Dm = [&](int k) { return d.data() + (size_t)k * NV * nn; };
    // physical and contravariant fluxes of a state at node (i, j) (contravariant_flux)
    auto cflux = [&](const double* s, int i, int j, double* f, double* g, double* cf, double* cg) {
        eq.fluxes(s, f, g);
        const double* J = Jae + 4 * (i + n * j);
        for (int v = 0; v < NV; ++v) {
            cf[v] = J[0] * f[v] + J[1] * g[v];
            cg[v] = J[2] * f[v] + J[3] * g[v];
        }
    };
    // t = -dt J^{-1}(node) (D x + D y) (the per-node Jacobian scaling follows the contraction)
    auto contract = [&](const std::vector<double>& x, const std::vector<double>& y, double* t) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v) {
                    double s = 0.0;
                    for (int k = 0; k < n; ++k) s += -dt * b.D[i * n + k] * x[L(k, j) + v] - dt * b.D[j * n + k] * y[L(i, k) + v];
                    t[L(i, j) + v] = s * ije[i + n * j];
                }
    };
    auto state = [&](int s, int q, int i, int j, double* P) {
        for (int v = 0; v < NV; ++v) {
            double x = ue[L(i, j) + v];
            for (int mm = 1; mm <= s; ++mm) x += S.a[q][mm] * Dm(mm)[L(i, j) + v];
            P[v] = x;
        }
    };
    // stage 0
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            cflux(ue + o, i, j, &Fp[o], &Gp[o], &ft[o], &gt[o]);
            for (int v = 0; v < NV; ++v) { Ft[o + v] = ft[o + v]; Gt[o + v] = gt[o + v]; Uc[o + v] = ue[o + v]; }
        }
    contract(ft, gt, Dm(1));
    const int src_kind = te ? te->source : 0;
    std::vector<double> Ssrc(src_kind ? NV * nn : 0, 0.0);
    // dt * stencil into derivative k, c * stencil into S, at every node
    auto add_source = [&](double* Dk, double c, const double (&w)[5], double scale) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const double* xn = te->xnode + 2 * ((size_t)e * nn + i + (size_t)n * j);
                double st[NV];
                source_stencil_t(src_kind, eq.gamma, xn[0], xn[1], t, dt, scale, w, st);
                for (int v = 0; v < NV; ++v) {
                    Ssrc[L(i, j) + v] += c * st[v];
                    if (Dk) Dk[L(i, j) + v] += dt * st[v];
                }
            }
    };
    static constexpr double W_S[5] = {0, 0, 1, 0, 0}, W_T12[5] = {0, -1, 0, 1, 0}, W_T34[5] = {1, -8, 0, 8, -1},
                            W_TT23[5] = {0, 1, -2, 1, 0}, W_TT4[5] = {-1, 16, -30, 16, -1},
                            W_TTT34[5] = {-1, 2, 0, -2, 1}, W_TTTT4[5] = {1, -4, 6, -4, 1};
    if (src_kind) add_source(Dm(1), 1.0, W_S, 1.0);   // S = s, ut += dt s (:1750-1757)
    // stages 1 .. depth: stencils of physical and contravariant fluxes, time averages, next derivative
    for (int s = 1; s <= depth; ++s) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int o = L(i, j);
                double f[NV], g[NV], cf[NV], cg[NV], pf[NV] = {0, 0, 0, 0}, pg[NV] = {0, 0, 0, 0};
                double tf[NV] = {0, 0, 0, 0}, tg[NV] = {0, 0, 0, 0};
                if (S.w[s][0] != 0.0) {
                    cflux(ue + o, i, j, f, g, cf, cg);
                    for (int v = 0; v < NV; ++v) {
                        pf[v] = S.w[s][0] * f[v]; pg[v] = S.w[s][0] * g[v];
                        tf[v] = S.w[s][0] * cf[v]; tg[v] = S.w[s][0] * cg[v];
                    }
                }
                for (int q = 0; q < 4; ++q) {
                    if (S.w[s][1 + q] == 0.0) continue;
                    double P[NV];
                    state(s, q, i, j, P);
                    cflux(P, i, j, f, g, cf, cg);
                    for (int v = 0; v < NV; ++v) {
                        pf[v] += S.w[s][1 + q] * f[v]; pg[v] += S.w[s][1 + q] * g[v];
                        tf[v] += S.w[s][1 + q] * cf[v]; tg[v] += S.w[s][1 + q] * cg[v];
                    }
                }
                if (want_te && s == depth) {   // F~, G~ before the last stage's term (u_np1_low)
                    if (Flow.empty()) { Flow.assign(NV * nn, 0.0); Glow.assign(NV * nn, 0.0); }
                    for (int v = 0; v < NV; ++v) { Flow[o + v] = Ft[o + v]; Glow[o + v] = Gt[o + v]; }
                }
                for (int v = 0; v < NV; ++v) {
                    Fp[o + v] += S.tw[s] * pf[v]; Gp[o + v] += S.tw[s] * pg[v];
                    Ft[o + v] += S.tw[s] * tf[v]; Gt[o + v] += S.tw[s] * tg[v];
                    Uc[o + v] += S.tw[s] * Dm(s)[o + v];
                    ft[o + v] = tf[v]; gt[o + v] = tg[v];
                }
            }
        if (s < depth) {
            contract(ft, gt, Dm(s + 1));
            if (src_kind) {
                if (s + 1 == 2) {   // s_t: N34 at depths 3 and 4, N12 below (:1815, :1267)
                    if (depth >= 3) add_source(Dm(2), 0.5, W_T34, 1.0 / 12.0);
                    else add_source(Dm(2), 0.5, W_T12, 0.5);
                } else if (s + 1 == 3) {   // s_tt: N4 at depth 4 (:1886), N23 at depth 3 (:1567)
                    if (depth == 4) add_source(Dm(3), 1.0 / 6.0, W_TT4, 1.0 / 12.0);
                    else add_source(Dm(3), 1.0 / 6.0, W_TT23, 1.0);
                } else {   // s_ttt (:1949)
                    add_source(Dm(4), 1.0 / 24.0, W_TTT34, 0.5);
                }
            }
        }
    }
    if (src_kind) {   // the last stencil: s_ttt / 24 at depth 3 (:1649), s_tttt / 120 at depth 4 (:2042)
        if (depth == 3) add_source(nullptr, 1.0 / 24.0, W_TTT34, 0.5);
        else add_source(nullptr, 1.0 / 120.0, W_TTTT4, 1.0);
    }
    // du += Dhat F~ + Dhat G~; element cache
    double* due = du + idx_u(n, 0, 0, 0, e);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int o = L(i, j);
            for (int ii = 0; ii < n; ++ii)
                for (int v = 0; v < NV; ++v) due[L(ii, j) + v] += alpha * b.Dhat[ii * n + i] * Ft[o + v];
            for (int jj = 0; jj < n; ++jj)
                for (int v = 0; v < NV; ++v) due[L(i, jj) + v] += alpha * b.Dhat[jj * n + j] * Gt[o + v];
            for (int v = 0; v < NV; ++v) {
                ws.F[idx_F(n, v, 0, i, j, e)] = Fp[o + v];
                ws.F[idx_F(n, v, 1, i, j, e)] = Gp[o + v];
                ws.U[idx_u(n, v, i, j, e)] = Uc[o + v];
            }
            if (src_kind)
                for (int v = 0; v < NV; ++v) due[o + v] += (-1.0 / ije[i + n * j]) * Ssrc[o + v];
        }
    if (want_te) {
        std::vector<double> hi(NV * nn), lo(NV * nn);
        contract(Ft, Gt, hi.data());
        contract(Flow, Glow, lo.data());
        double err = 0.0;
        for (int k = 0; k < NV * nn; ++k) {
            const double a = ue[k] + hi[k], c = ue[k] + lo[k];
            const double r = (a - c) / (te->abstol + te->reltol * std::max(std::fabs(a), std::fabs(c)));
            err += r * r;
        }
        ws.temporal_errors[e] = err;
    }
}

// Boundary faces with the LW slip walls in their normal-direction form (src/equations/equations.jl:137-169;
// prolong2boundaries! and calc_boundary_flux!, src/solvers/dgsem_p4est/dg_2d.jl:285-393): the inner normal flux
// uses the outward normal, the exterior state mirrors it, and the surface flux takes the inner side as _ll in
// the curvilinear order (f_in, f_out, u_in, u_out, U_in, U_out, normal); the result is the outward flux.
// Time-averaged Dirichlet boundaries in the normal-direction form (src/equations/equations.jl:64-93): U_outer,
// F_outer are GLL time averages of the exterior state and of its flux along the outward normal (levels as for
// the TreeMesh), and the surface flux is called with U_outer in the place of the exterior u:
// (f_in, f_out, u_in, U_out, U_in, U_out, normal).
inline void calc_boundary_flux_curved(const Basis& b, const Euler& eq, const Options& opt, const CurvedMesh& m,
                                      const double* u, Workspace& ws, const BoundaryData* bd = nullptr,
                                      double scaling_factor = 1.0) {
    const int n = b.n;
    for (int k = 0; k < m.n_boundaries; ++k) {
        const int e = m.b_elem[k], f = m.b_face[k], kind = m.b_kind[k];
        if (kind == BC_DIRICHLET && (!bd || !bd->u_levels)) throw std::invalid_argument("boundary data missing");
        for (int l = 0; l < n; ++l) {
            int i, j;
            face_node(n, f, l, i, j);
            double nrm[2], Fi[NV], Ui[NV], ui[NV], Fo[NV] = {0, 0, 0, 0}, Uo[NV] = {0, 0, 0, 0}, uo[NV], Fn[NV];
            outward_normal(m, n, f, i, j, e, nrm);
            for (int v = 0; v < NV; ++v) {
                Fi[v] = ws.F[idx_F(n, v, 0, i, j, e)] * nrm[0] + ws.F[idx_F(n, v, 1, i, j, e)] * nrm[1];
                Ui[v] = ws.U[idx_u(n, v, i, j, e)];
                ui[v] = u[idx_u(n, v, i, j, e)];
            }
            if (kind == BC_DIRICHLET) {
                for (int q = 0; q < n; ++q) {
                    const double* ub = bd->u_levels + NV * (q + (size_t)n * (l + (size_t)n * k));
                    double fx[NV], gy[NV];
                    eq.fluxes(ub, fx, gy);
                    for (int v = 0; v < NV; ++v) {
                        Uo[v] += ub[v] * scaling_factor * b.weights[q] / 2.0;
                        Fo[v] += (fx[v] * nrm[0] + gy[v] * nrm[1]) * scaling_factor * b.weights[q] / 2.0;
                    }
                }
                lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, Fi, Fo, ui, Uo, Ui, Uo, nrm, Fn, ws.bad);
                for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * (f + 4 * (size_t)e))] = Fn[v];
                continue;
            }
            slip_wall_exterior(kind, Fi, Ui, ui, Fo, Uo, uo);
            lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, Fi, Fo, ui, uo, Ui, Uo, nrm, Fn, ws.bad);
            for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * (f + 4 * (size_t)e))] = Fn[v];
        }
    }
}

// Trixi flux(u, normal_direction, equations) of CompressibleEulerEquations2D
inline void euler_flux_along(const Euler& eq, const double* u, const double* nrm, double* f) {
    double rho, v1, v2, p;
    eq.cons2prim(u, rho, v1, v2, p);
    const double vn = v1 * nrm[0] + v2 * nrm[1];
    const double rvn = rho * vn;
    f[0] = rvn;
    f[1] = rvn * v1 + p * nrm[0];
    f[2] = rvn * v2 + p * nrm[1];
    f[3] = (u[3] + p) * vn;
}

// L2 mortars of a curvilinear mesh as the reference's P4estMesh path computes them (prolong2mortars! and
// calc_mortar_flux!, src/solvers/dgsem_p4est/dg_2d.jl:395-603, with Trixi's mortar_fluxes_to_elements!): the
// small side keeps its time-averaged U and F.n along its own outward normal; the large side's u and U are
// interpolated onto the small faces (forward operators), and its normal flux is the instantaneous
// Trixi.flux(u, -n_large / 2) (the reference overwrites the time-averaged product, :455-458); the surface flux
// takes the small side as _ll in the curvilinear order along the small element's normal. The small faces get
// fstar, the large face -2 times its L2 projection (reverse operators), in its own index order.
// blend: called per small node as blend(mortar, position, l, small element, u_ll, u_rr, normal, fstar) after the
// LW flux is formed (the shock-capturing get_blended_flux; nothing without shock capturing).
struct NoMortarBlend {
    void operator()(int, int, int, int, const double*, const double*, const double*, double*) const {}
};
template <class Blend = NoMortarBlend>
inline void calc_mortar_flux_curved(const Basis& b, const Euler& eq, const Options& opt, const CurvedMesh& m,
                                    const double* u, Workspace& ws, bool& bad, const Blend& blend = Blend()) {
    const int n = b.n;
    for (int k = 0; k < m.n_mortars; ++k) {
        const int lg = m.m_large[k], lf = m.m_lface[k], sf = m.m_sface[k];
        const bool rev = m.m_lrev[k] != 0;
        std::vector<double> ub(n * NV), Ub(n * NV), Fb(n * NV), fstar(2 * n * NV);
        for (int i = 0; i < n; ++i) {
            const int li = rev ? n - 1 - i : i;
            int il, jl;
            face_node(n, lf, li, il, jl);
            double nL[2];
            outward_normal(m, n, lf, il, jl, lg, nL);
            nL[0] *= -0.5;
            nL[1] *= -0.5;
            for (int v = 0; v < NV; ++v) {
                ub[i * NV + v] = u[idx_u(n, v, il, jl, lg)];
                Ub[i * NV + v] = ws.U[idx_u(n, v, il, jl, lg)];
            }
            euler_flux_along(eq, &ub[i * NV], nL, &Fb[i * NV]);
        }
        for (int h = 0; h < 2; ++h) {
            const int se = h ? m.m_small2[k] : m.m_small1[k];
            const std::vector<double>& fwd = h ? b.fwd_upper : b.fwd_lower;
            for (int l = 0; l < n; ++l) {
                int is, js;
                face_node(n, sf, l, is, js);
                double nS[2], f_ll[NV], u_ll[NV], U_ll[NV], u_rr[NV] = {0, 0, 0, 0}, U_rr[NV] = {0, 0, 0, 0},
                                                            f_rr[NV] = {0, 0, 0, 0};
                outward_normal(m, n, sf, is, js, se, nS);
                for (int v = 0; v < NV; ++v) {
                    f_ll[v] = ws.F[idx_F(n, v, 0, is, js, se)] * nS[0] + ws.F[idx_F(n, v, 1, is, js, se)] * nS[1];
                    u_ll[v] = u[idx_u(n, v, is, js, se)];
                    U_ll[v] = ws.U[idx_u(n, v, is, js, se)];
                }
                for (int i = 0; i < n; ++i) {
                    const double c = fwd[l * n + i];
                    for (int v = 0; v < NV; ++v) {
                        u_rr[v] += c * ub[i * NV + v];
                        U_rr[v] += c * Ub[i * NV + v];
                        f_rr[v] += c * Fb[i * NV + v];
                    }
                }
                double* out = &fstar[(h * n + l) * NV];
                bool b_ = false;
                lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, nS, out, b_);
                blend(k, h, l, se, u_ll, u_rr, nS, out);
                bad = bad || b_;
                for (int v = 0; v < NV; ++v) ws.surface_flux_values[v + NV * (l + n * (sf + 4 * (size_t)se))] = out[v];
            }
        }
        for (int i = 0; i < n; ++i) {
            const int li = rev ? n - 1 - i : i;
            for (int v = 0; v < NV; ++v) {
                double acc = 0.0;
                for (int l = 0; l < n; ++l)
                    acc += b.rev_upper[i * n + l] * fstar[(n + l) * NV + v] + b.rev_lower[i * n + l] * fstar[l * NV + v];
                ws.surface_flux_values[v + NV * (li + n * (lf + 4 * (size_t)lg))] = -2.0 * acc;
            }
        }
    }
}

// surface integral (outward fluxes) and apply_jacobian (per node) on a curvilinear mesh
inline void surface_integral_and_jacobian_curved(const Basis& b, const CurvedMesh& m, double* du, const Workspace& ws,
                                                 int nthreads = 1) {
    const int n = b.n;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e) {
        for (int f = 0; f < 4; ++f) {
            const double iw = (f == 1 || f == 3) ? b.inv_w_last : b.inv_w_first;
            for (int l = 0; l < n; ++l) {
                int i, j;
                face_node(n, f, l, i, j);
                for (int v = 0; v < NV; ++v)
                    du[idx_u(n, v, i, j, e)] += ws.surface_flux_values[v + NV * (l + n * (f + 4 * (size_t)e))] * iw;
            }
        }
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const double s = -m.inv_jac[i + n * (j + (size_t)n * e)];
                for (int v = 0; v < NV; ++v) du[idx_u(n, v, i, j, e)] *= s;
            }
    }
}

// What the reference can run on an UnstructuredMesh2D: its rhs! (dgsem_unstructured_2d/dg_2d.jl:14-56) is LW only
// (no mesh-level rhs_mdrk1! / rhs_mdrk2! takes an UnstructuredMesh2D), the mesh is conforming (no mortars), and its
// calc_boundary_flux! (:421-450) calls the boundary condition with 11 arguments (U, F.n, normal, x, t, dt,
// surface_flux, equations, dg, time discretization, scaling) that no method of src/equations/equations.jl
// accepts, so only meshes without boundaries (periodic, like its Sedov elixir) run.
inline void check_unstructured(const CurvedMesh& m, int kind) {
    if (m.unormals.empty()) return;
    if (kind != 0) throw std::invalid_argument("UnstructuredMesh2D: LW only");
    if (m.n_boundaries > 0 || m.n_mortars > 0)
        throw std::invalid_argument("UnstructuredMesh2D: conforming and without boundaries");
}

// du = rhs(u) on a conforming curvilinear mesh (LW, FR volume integral; boundaries: slip walls)
// kind 0: LW rhs!; 1: rhs_mdrk1! (keeps U2, F2); 2: rhs_mdrk2! with the stage state u2 in the volume terms and
// u (u^n) at the interfaces (src/solvers/dgsem_structured/multi_derivative_2d.jl:1-80)
inline void rhs_curved(const Basis& b, const Euler& eq, const Options& opt, const CurvedMesh& m, const double* u,
                       double* du, double dt, Workspace& ws, int nthreads = 1, int kind = 0,
                       const double* u2 = nullptr, const BoundaryData* bd = nullptr, double t = 0.0) {
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    ws.U.assign(ndof, nan);
    ws.F.assign(2 * ndof, nan);
    ws.surface_flux_values.assign((size_t)NV * n * 4 * m.n_elements, nan);
    ws.bad = false;
    if (opt.temporal_errors && kind == 0) ws.temporal_errors.assign(m.n_elements, nan);
    if (kind == 1) {
        ws.U2.assign(ndof, nan);
        ws.F2.assign(2 * ndof, nan);
        if (opt.source) ws.S2.assign(ndof, nan);
    }
    if (kind == 2 && (ws.U2.size() != ndof || !u2)) throw std::invalid_argument("rhs_mdrk2 before rhs_mdrk1");
    check_unstructured(m, kind);
    for (size_t k = 0; k < ndof; ++k) du[k] = 0.0;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int e = 0; e < m.n_elements; ++e) {
        const double* Jae = &m.Ja[4 * (size_t)nn * e];
        const double* ije = &m.inv_jac[(size_t)nn * e];
        SourceArgs sa{opt.source, opt.xnode, eq.gamma, t};
        sa.stage2_at_t = true;
        if (kind == 0) lw_volume_element_curved(b, eq, opt.N, m, e, u, du, dt, ws, 1.0, &opt, t);
        else if (kind == 1) mdrk1_volume_element(b, eq, e, u, du, dt, 0.0, 1.0, ws, Jae, ije, &sa);
        else mdrk2_volume_element(b, eq, e, u2, du, dt, 0.0, 1.0, ws, Jae, ije, &sa);
    }
    bool bad = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad)
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int pe = m.p_elem[k], pf = m.p_face[k], se = m.s_elem[k], sf = m.s_face[k];
        for (int l = 0; l < n; ++l) {
            const int ls = m.s_rev[k] ? n - 1 - l : l;
            if (!m.unormals.empty()) {   // UnstructuredMesh2D
                double nP[2], Fn[NV], u_ll[NV], u_rr[NV], U_ll[NV], U_rr[NV];
                bool b_ = false;
                unstructured_interface_node(eq, opt, m, n, u, ws, pe, pf, se, sf, l, ls, nP, Fn, u_ll, u_rr, U_ll, U_rr, b_);
                bad = bad || b_;
                for (int v = 0; v < NV; ++v) {
                    ws.surface_flux_values[v + NV * (l + n * (pf + 4 * (size_t)pe))] = Fn[v];
                    ws.surface_flux_values[v + NV * (ls + n * (sf + 4 * (size_t)se))] = -Fn[v];
                }
                continue;
            }
            int ip, jp, is, js;
            face_node(n, pf, l, ip, jp);
            face_node(n, sf, ls, is, js);
            double nP[2], nS[2], f_ll[NV], f_rr[NV], u_ll[NV], u_rr[NV], U_ll[NV], U_rr[NV], Fn[NV];
            outward_normal(m, n, pf, ip, jp, pe, nP);
            outward_normal(m, n, sf, is, js, se, nS);
            for (int v = 0; v < NV; ++v) {
                f_ll[v] = ws.F[idx_F(n, v, 0, ip, jp, pe)] * nP[0] + ws.F[idx_F(n, v, 1, ip, jp, pe)] * nP[1];
                f_rr[v] = ws.F[idx_F(n, v, 0, is, js, se)] * (-nS[0]) + ws.F[idx_F(n, v, 1, is, js, se)] * (-nS[1]);
                u_ll[v] = u[idx_u(n, v, ip, jp, pe)];
                u_rr[v] = u[idx_u(n, v, is, js, se)];
                U_ll[v] = ws.U[idx_u(n, v, ip, jp, pe)];
                U_rr[v] = ws.U[idx_u(n, v, is, js, se)];
            }
            bool b_ = false;
            lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, nP, Fn, b_);
            bad = bad || b_;
            for (int v = 0; v < NV; ++v) {
                ws.surface_flux_values[v + NV * (l + n * (pf + 4 * (size_t)pe))] = Fn[v];
                ws.surface_flux_values[v + NV * (ls + n * (sf + 4 * (size_t)se))] = -Fn[v];
            }
        }
    }
    ws.bad = ws.bad || bad;
    bad = false;
    calc_mortar_flux_curved(b, eq, opt, m, u, ws, bad);
    ws.bad = ws.bad || bad;
    // MDRK stage 1 scales the time averages by 1/2 (as the P4estMesh path does, multi_derivative_2d.jl:34)
    calc_boundary_flux_curved(b, eq, opt, m, u, ws, bd, kind == 1 ? 0.5 : 1.0);
    surface_integral_and_jacobian_curved(b, m, du, ws, nthreads);
}

// Trixi max_dt for curved meshes: per node lambda~_d = |Ja^d . (|v1| + c, |v2| + c)| |J^{-1}|
inline double max_dt_curved(const Basis& b, const Euler& eq, const CurvedMesh& m, const double* u, double cfl,
                            bool& bad, int nthreads = 1) {
    const int n = b.n;
    double max_scaled = std::nextafter(0.0, 1.0);
    bool bad_any = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(max : max_scaled) reduction(|| : bad_any)
    for (int e = 0; e < m.n_elements; ++e) {
        double m1 = 0.0, m2 = 0.0;
        bool b_ = false;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double l1, l2;
                eq.max_abs_speeds(u + idx_u(n, 0, i, j, e), l1, l2, b_);
                const size_t node = i + n * (j + (size_t)n * e);
                const double* J = &m.Ja[4 * node];
                const double ij = std::fabs(m.inv_jac[node]);
                m1 = std::max(m1, std::fabs(J[0] * l1 + J[1] * l2) * ij);
                m2 = std::max(m2, std::fabs(J[2] * l1 + J[3] * l2) * ij);
            }
        max_scaled = std::max(max_scaled, m1 + m2);
        bad_any = bad_any || b_;
    }
    bad = bad_any;
    return cfl * 2.0 / (n * max_scaled);
}

}  // namespace tlwo
