// oracle_capi.cpp -- C entry points of the CPU oracle (TEST INFRASTRUCTURE ONLY: called from tests/,
// the smoke check and the CPU-baseline leg of bench.py; never from the product path).
// Parity status: unpinned against the reference itself (no Julia here); see tlw_oracle.hpp.
#include <chrono>
#include <cstdio>
#include <memory>

#include "tlw_adjoint.hpp"
#include "tlw_curved.hpp"
#include "tlw_curved_parabolic.hpp"
#include "tlw_curved_sc.hpp"
#include "tlw_dual.hpp"
#include "tlw_limiter.hpp"
#include "tlw_parabolic.hpp"
#include "tlw_oracle.hpp"

using namespace tlwo;

struct oracle_handle {
    Basis basis;
    Euler eq;
    Options opt;
    TreeMesh mesh;
    Workspace ws;
    std::vector<double> us;      // MDRK stage state u*
    std::vector<double> du;
    std::vector<double> bnd_levels, bnd_now;
    bool curved = false;         // conforming curvilinear mesh (cmesh) instead of the TreeMesh
    CurvedMesh cmesh;
    bool parabolic = false;      // compressible Navier-Stokes (TreeMesh, periodic, LW)
    NavierStokes ns;
    PositivityLimiter lim;       // applied after every step of oracle_steps when not empty
    std::vector<double> xnode;   // node coordinates [2, i, j, e] for source terms
    char err[256] = {0};

    int n_elements() const { return curved ? cmesh.n_elements : mesh.n_elements; }
};

namespace {

// LW / MDRK rhs on whichever mesh the handle holds (curvilinear: LW, FR volume integral only)
void any_rhs(oracle_handle* h, const double* u, const double* u2, double* du, double t, double dt,
             const BoundaryData* bd, int kind, int nthreads) {
    if (h->parabolic) {
        if (kind != 0) throw std::runtime_error("parabolic oracle: LW only");
        if (h->curved) rhs_parabolic_curved(h->basis, h->eq, h->ns, h->opt, h->cmesh, u, du, dt, h->ws, nthreads);
        else rhs_parabolic(h->basis, h->eq, h->ns, h->opt, h->mesh, u, du, dt, h->ws, nthreads, bd);
        return;
    }
    if (!h->curved) {
        rhs(h->basis, h->eq, h->opt, h->mesh, u, u2, du, t, dt, bd, kind, h->ws, nthreads);
        return;
    }
    if (h->opt.shock_capturing) {
        rhs_curved_sc(h->basis, h->eq, h->opt, h->cmesh, u, du, dt, h->ws, nthreads, bd, kind, u2);
        return;
    }
    rhs_curved(h->basis, h->eq, h->opt, h->cmesh, u, du, dt, h->ws, nthreads, kind, u2, bd, t);
}

// one application of the positivity limiter on whichever mesh the handle holds
void limit(oracle_handle* h, double* u) {
    if (h->curved) apply_positivity_limiter_curved(h->basis, h->eq, h->cmesh, h->lim, u);
    else apply_positivity_limiter(h->basis, h->eq, h->mesh, h->n_elements(), h->lim, u);
}

double any_max_dt(oracle_handle* h, const double* u, double cfl, bool& bad, int nthreads) {
    if (h->parabolic && h->curved) return max_dt_parabolic_curved(h->basis, h->eq, h->ns, h->cmesh, u, cfl, bad, nthreads);
    if (h->parabolic) return max_dt_parabolic(h->basis, h->eq, h->ns, h->mesh, u, cfl, bad, nthreads);
    if (h->curved) return max_dt_curved(h->basis, h->eq, h->cmesh, u, cfl, bad, nthreads);
    return max_dt(h->basis, h->eq, h->mesh, u, cfl, bad, nthreads);
}

}  // namespace

extern "C" {

int oracle_basis(int N, double* nodes, double* weights, double* D, double* Dhat) {
    try {
        Basis b = make_basis(N);
        for (int i = 0; i < b.n; ++i) { nodes[i] = b.nodes[i]; weights[i] = b.weights[i]; }
        for (int k = 0; k < b.n * b.n; ++k) { D[k] = b.D[k]; Dhat[k] = b.Dhat[k]; }
        return 0;
    } catch (...) { return 1; }
}

oracle_handle* oracle_create(int N, double gamma, int flux_kind, int speed_kind, int E, const double* inv_jac,
                             int I, const int32_t* left, const int32_t* right, const int32_t* orient, int B,
                             const int32_t* b_elem, const int32_t* b_orient, const int32_t* b_side,
                             const int32_t* b_dir) {
    try {
        auto h = std::make_unique<oracle_handle>();
        h->basis = make_basis(N);
        h->eq.gamma = gamma;
        h->opt.N = N;
        h->opt.flux_kind = flux_kind;
        h->opt.speed_kind = speed_kind;
        h->mesh.n_elements = E;
        h->mesh.inverse_jacobian.assign(inv_jac, inv_jac + E);
        h->mesh.n_interfaces = I;
        h->mesh.interface_left.assign(left, left + I);
        h->mesh.interface_right.assign(right, right + I);
        h->mesh.interface_orientation.assign(orient, orient + I);
        h->mesh.n_boundaries = B;
        if (B > 0) {
            h->mesh.boundary_element.assign(b_elem, b_elem + B);
            h->mesh.boundary_orientation.assign(b_orient, b_orient + B);
            h->mesh.boundary_side.assign(b_side, b_side + B);
            h->mesh.boundary_direction.assign(b_dir, b_dir + B);
        }
        return h.release();
    } catch (...) { return nullptr; }
}

// Conforming curvilinear mesh: Ja [4, i, j, e] (Trixi contravariant_vectors order Ja^1_1, Ja^1_2, Ja^2_1,
// Ja^2_2), inv_jac [i, j, e]; interfaces (primary element, face; secondary element, face; reversed), 0-based,
// faces 0: -xi, 1: +xi, 2: -eta, 3: +eta.
oracle_handle* oracle_create_curved(int N, double gamma, int flux_kind, int speed_kind, int E, const double* Ja,
                                    const double* inv_jac, int I, const int32_t* pe, const int32_t* pf,
                                    const int32_t* se, const int32_t* sf, const int32_t* rev) {
    try {
        auto h = std::make_unique<oracle_handle>();
        h->basis = make_basis(N);
        h->eq.gamma = gamma;
        h->opt.N = N;
        h->opt.flux_kind = flux_kind;
        h->opt.speed_kind = speed_kind;
        const size_t nn = (size_t)h->basis.n * h->basis.n;
        h->curved = true;
        h->mesh.n_elements = E;   // element count for the shared step loop
        h->cmesh.n_elements = E;
        h->cmesh.Ja.assign(Ja, Ja + 4 * nn * E);
        h->cmesh.inv_jac.assign(inv_jac, inv_jac + nn * E);
        h->cmesh.n_interfaces = I;
        h->cmesh.p_elem.assign(pe, pe + I);
        h->cmesh.p_face.assign(pf, pf + I);
        h->cmesh.s_elem.assign(se, se + I);
        h->cmesh.s_face.assign(sf, sf + I);
        h->cmesh.s_rev.assign(rev, rev + I);
        return h.release();
    } catch (...) { return nullptr; }
}

// L2 mortars of a TreeMesh: lower, upper, large element (0-based), large side (1: large on the -side), orientation
int oracle_set_mortars(oracle_handle* h, int M, const int32_t* lower, const int32_t* upper, const int32_t* large,
                       const int32_t* large_side, const int32_t* orientation) {
    if (h->curved) return 1;
    h->mesh.n_mortars = M;
    h->mesh.mortar_lower.assign(lower, lower + M);
    h->mesh.mortar_upper.assign(upper, upper + M);
    h->mesh.mortar_large.assign(large, large + M);
    h->mesh.mortar_large_side.assign(large_side, large_side + M);
    h->mesh.mortar_orientation.assign(orientation, orientation + M);
    return 0;
}

// the mortar operators of degree N: [4][n][n] = forward_upper, forward_lower, reverse_upper, reverse_lower
int oracle_mortar_operators(int N, double* out) {
    try {
        const Basis b = make_basis(N);
        const int nn = b.n * b.n;
        for (int k = 0; k < nn; ++k) {
            out[k] = b.fwd_upper[k];
            out[nn + k] = b.fwd_lower[k];
            out[2 * nn + k] = b.rev_upper[k];
            out[3 * nn + k] = b.rev_lower[k];
        }
        return 0;
    } catch (...) { return 1; }
}

// compressible Navier-Stokes: dynamic viscosity mu and Prandtl number (the handle's gamma)
int oracle_set_parabolic(oracle_handle* h, double mu, double Pr) {
    h->parabolic = true;
    h->ns.gamma = h->eq.gamma;
    h->ns.mu = mu;
    h->ns.Pr = Pr;
    return 0;
}

// boundary faces of a curvilinear mesh: element (0-based), face 0..3, slip wall kind 1 (vertical) / 2 (horizontal)
int oracle_set_curved_boundaries(oracle_handle* h, int B, const int32_t* elem, const int32_t* face, const int32_t* kind) {
    if (!h->curved) return 1;
    h->cmesh.n_boundaries = B;
    h->cmesh.b_elem.assign(elem, elem + B);
    h->cmesh.b_face.assign(face, face + B);
    h->cmesh.b_kind.assign(kind, kind + B);
    for (int k = 0; k < B; ++k)
        if (kind[k] != BC_DIRICHLET && kind[k] != BC_SLIP_WALL_VERTICAL && kind[k] != BC_SLIP_WALL_HORIZONTAL) return 1;
    return 0;
}

// L2 mortars of a curvilinear mesh (0-based elements): small elements at positions 1, 2, their face, the large
// element, its face and whether its index runs backwards along the mortar
int oracle_set_curved_mortars(oracle_handle* h, int M, const int32_t* small1, const int32_t* small2, const int32_t* sface,
                              const int32_t* large, const int32_t* lface, const int32_t* lrev) {
    if (!h->curved) return 1;
    CurvedMesh& m = h->cmesh;
    m.n_mortars = M;
    m.m_small1.assign(small1, small1 + M);
    m.m_small2.assign(small2, small2 + M);
    m.m_sface.assign(sface, sface + M);
    m.m_large.assign(large, large + M);
    m.m_lface.assign(lface, lface + M);
    m.m_lrev.assign(lrev, lrev + M);
    m.m_ij.clear();
    return 0;
}

// lw_mortars.inverse_jacobian [mortar][l] for the shock-capturing blend at the mortars (null: zeros)
// UnstructuredMesh2D: the caller's outward normals by face [2, l, face, e] (faces as the curved interfaces);
// null switches back to the StructuredMesh / P4estMesh interface conventions
// source terms on the TreeMesh (LW and MDRK): kind 0 none, 1 source_terms_convergence_test; node coordinates
// [2, i, j, e]
int oracle_set_source(oracle_handle* h, int kind, const double* node_coordinates) {
    if (h->parabolic || kind < 0 || kind > 1 || (kind && !node_coordinates)) return 1;
    if (kind) h->xnode.assign(node_coordinates, node_coordinates + (size_t)2 * h->basis.n * h->basis.n * h->n_elements());
    else h->xnode.clear();
    h->opt.source = kind;
    h->opt.xnode = kind ? h->xnode.data() : nullptr;
    return 0;
}

int oracle_set_unstructured_normals(oracle_handle* h, const double* normals) {
    if (!h->curved) return 1;
    CurvedMesh& m = h->cmesh;
    if (!normals) m.unormals.clear();
    else m.unormals.assign(normals, normals + (size_t)2 * h->basis.n * 4 * m.n_elements);
    return 0;
}

int oracle_set_curved_mortar_jacobian(oracle_handle* h, const double* inv_jac) {
    if (!h->curved) return 1;
    CurvedMesh& m = h->cmesh;
    if (!inv_jac) m.m_ij.clear();
    else m.m_ij.assign(inv_jac, inv_jac + (size_t)m.n_mortars * h->basis.n);
    return 0;
}

// per boundary: 0 time-averaged Dirichlet, 1 slip wall vertical, 2 slip wall horizontal
int oracle_set_boundary_kinds(oracle_handle* h, const int32_t* kinds) {
    if (h->curved) return 1;
    h->mesh.boundary_kind.assign(kinds, kinds + h->mesh.n_boundaries);
    return 0;
}

// Navier-Stokes walls per boundary (1 no-slip adiabatic, 2 no-slip isothermal) and their data [3, l, B]
int oracle_set_walls(oracle_handle* h, const int32_t* kinds, const double* data) {
    const size_t B = h->curved ? h->cmesh.n_boundaries : h->mesh.n_boundaries, n = h->basis.n;
    h->ns.wall_kind.assign(kinds, kinds + B);
    h->ns.wall.assign(data, data + 3 * n * B);
    return 0;
}

void oracle_destroy(oracle_handle* h) { delete h; }

// VolumeIntegralFRShockCapturing with IndicatorHennemannGassner(alpha_max, alpha_min, alpha_smooth;
// variable = density_pressure) and first-order subcell reconstruction.
void oracle_set_shock_capturing(oracle_handle* h, int on, double alpha_max, double alpha_min, int alpha_smooth) {
    h->opt.shock_capturing = on != 0;
    h->opt.alpha_max = alpha_max;
    h->opt.alpha_min = alpha_min;
    h->opt.alpha_smooth = alpha_smooth != 0;
}

// the subcell reconstruction of blended elements on curvilinear meshes: 0 first order, 1 MUSCL
void oracle_set_reconstruction(oracle_handle* h, int reconstruction) { h->opt.reconstruction = reconstruction; }

void oracle_set_temporal_errors(oracle_handle* h, int on, double abstol, double reltol) {
    h->opt.temporal_errors = on != 0;
    h->opt.abstol = abstol;
    h->opt.reltol = reltol;
}

// Exterior boundary states: levels [v, k, l, B] at t + 0.5 dt_scaled (x_k + 1), now [v, l, B] at t.
int oracle_set_boundary_data(oracle_handle* h, const double* levels, const double* now) {
    const size_t n = h->basis.n, B = h->curved ? h->cmesh.n_boundaries : h->mesh.n_boundaries;
    h->bnd_levels.assign(levels, levels + NV * n * n * B);
    h->bnd_now.assign(now, now + NV * n * B);
    return 0;
}

// kind: 0 LW rhs!, 1 rhs_mdrk1!, 2 rhs_mdrk2! (u2 = u* for stage 2). Returns 0, or 3 when a square root of
// a negative number occurred (the reference raises DomainError there).
int oracle_rhs(oracle_handle* h, int kind, const double* u, const double* u2, double* du, double t, double dt,
               int nthreads) {
    try {
        BoundaryData bd{h->bnd_levels.empty() ? nullptr : h->bnd_levels.data(),
                        h->bnd_now.empty() ? nullptr : h->bnd_now.data()};
        any_rhs(h, u, u2, du, t, dt, &bd, kind, nthreads);
        return h->ws.bad ? 3 : 0;
    } catch (const std::exception& ex) {
        std::snprintf(h->err, sizeof(h->err), "%s", ex.what());
        return 1;
    }
}

// lam_out = (d u_new / d u)^T lam_in for one LW step u_new = u + dt rhs(u) at fixed dt (periodic mesh,
// FR volume integral, Rusanov flux). Returns 0, 3 (non-admissible state), 4 (unsupported options).
int oracle_adjoint_step(oracle_handle* h, const double* u, double dt, const double* lam_in, double* lam_out,
                        int nthreads) {
    try {
        if (h->opt.flux_kind != RUSANOV || h->opt.shock_capturing || h->mesh.n_boundaries || h->opt.N < 3) return 4;
        h->ws.bad = false;
        adjoint_step(h->basis, h->eq, h->opt, h->mesh, u, dt, lam_in, lam_out, h->ws, nthreads);
        return h->ws.bad ? 3 : 0;
    } catch (const std::exception& ex) {
        std::snprintf(h->err, sizeof(h->err), "%s", ex.what());
        return 1;
    }
}

// One step (kind 0 LW, 1 MDRK) u_out of the scalar-templated restatement (periodic TreeMesh, FR, Rusanov, N >= 3):
// with dir == null in double; otherwise with dual numbers seeded by dir, and d_out = the step's directional
// derivative along dir.
int oracle_dual_step(oracle_handle* h, int kind, const double* u, const double* dir, double dt, double* u_out,
                     double* d_out) {
    try {
        if (h->curved || h->opt.flux_kind != RUSANOV || h->opt.shock_capturing || h->mesh.n_boundaries ||
            h->mesh.n_mortars || h->opt.N < 3)
            return 4;
        const size_t nd = (size_t)NV * h->basis.n * h->basis.n * h->mesh.n_elements;
        const bool mdrk = kind == 1;
        if (!dir) {
            if (mdrk) mdrk_step_templated<double>(h->basis, h->eq.gamma, h->opt.speed_kind, h->mesh, u, dt, u_out);
            else lw_step_templated<double>(h->basis, h->eq.gamma, h->opt.speed_kind, h->mesh, h->opt.N, u, dt, u_out);
            return 0;
        }
        std::vector<Dual> x(nd), y(nd);
        for (size_t k = 0; k < nd; ++k) x[k] = Dual(u[k], dir[k]);
        if (mdrk) mdrk_step_templated<Dual>(h->basis, h->eq.gamma, h->opt.speed_kind, h->mesh, x.data(), dt, y.data());
        else lw_step_templated<Dual>(h->basis, h->eq.gamma, h->opt.speed_kind, h->mesh, h->opt.N, x.data(), dt, y.data());
        for (size_t k = 0; k < nd; ++k) {
            u_out[k] = y[k].v;
            d_out[k] = y[k].d;
        }
        return 0;
    } catch (const std::exception& ex) {
        std::snprintf(h->err, sizeof(h->err), "%s", ex.what());
        return 1;
    }
}

// which: 0 U [v,i,j,e], 1 F [v,d,i,j,e], 2 U2, 3 F2, 4 temporal_errors [e], 5 surface_flux_values [v,l,face,e],
//        6 alpha [e], 7 fn_low [v,l,face,e], 8 mortar_fixes [2] (curvilinear shock capturing)
int oracle_get(oracle_handle* h, int which, double* out) {
    const std::vector<double>* src = nullptr;
    switch (which) {
        case 0: src = &h->ws.U; break;
        case 1: src = &h->ws.F; break;
        case 2: src = &h->ws.U2; break;
        case 3: src = &h->ws.F2; break;
        case 4: src = &h->ws.temporal_errors; break;
        case 5: src = &h->ws.surface_flux_values; break;
        case 6: src = &h->ws.alpha; break;
        case 7: src = &h->ws.fn_low; break;
        case 8: src = &h->ws.mortar_fixes; break;
        default: return 1;
    }
    std::copy(src->begin(), src->end(), out);
    return 0;
}

double oracle_max_dt(oracle_handle* h, const double* u, double cfl) {
    bool bad = false;
    const double dt = any_max_dt(h, u, cfl, bad, 1);
    return bad ? -1.0 : dt;
}

// The CFL-based step loop of solve_lwfr / perform_step! (src/solvers/lwfr.jl:212-230, 76-103;
// src/solvers/mdrk.jl:1-29): dt = cfl * max_dt(u), clamped to t_end, u <- u + dt * du.
// kind 0 = LW, 1 = MDRK. Runs at most nsteps steps or until t reaches t_end; returns steps taken, or
// a negative number on error. t_inout is advanced.
int oracle_steps(oracle_handle* h, int kind, double* u, int nsteps, double cfl, double fixed_dt, double* t_inout,
                 double t_end, int nthreads) {
    const size_t ndof = (size_t)NV * h->basis.n * h->basis.n * h->mesh.n_elements;
    try {
    h->du.resize(ndof);
    h->us.resize(ndof);
    double t = *t_inout;
    int s = 0;
    for (; s < nsteps; ++s) {
        // isfinished: t ≈ t_end, Julia isapprox with rtol = sqrt(eps(Float64)) (src/solvers/lwfr.jl:146-148)
        if (t == t_end) break;
        if (std::isfinite(t_end) &&
            (t >= t_end || std::fabs(t - t_end) <= 1.4901161193847656e-8 * std::max(std::fabs(t), std::fabs(t_end))))
            break;
        bool bad = false;
        double dt = fixed_dt > 0 ? fixed_dt : any_max_dt(h, u, cfl, bad, nthreads);
        if (bad) return -3;
        if (t + dt > t_end) dt = t_end - t;
        BoundaryData bd{h->bnd_levels.empty() ? nullptr : h->bnd_levels.data(),
                        h->bnd_now.empty() ? nullptr : h->bnd_now.data()};
        if (kind == 0) {
            any_rhs(h, u, nullptr, h->du.data(), t, dt, &bd, 0, nthreads);
            if (h->ws.bad) return -3;
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long long k = 0; k < (long long)ndof; ++k) u[k] = u[k] + dt * h->du[k];
        } else {
            any_rhs(h, u, nullptr, h->du.data(), t, dt, &bd, 1, nthreads);
            if (h->ws.bad) return -3;
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long long k = 0; k < (long long)ndof; ++k) h->us[k] = u[k] + dt * h->du[k];
            any_rhs(h, u, h->us.data(), h->du.data(), t, dt, &bd, 2, nthreads);
            if (h->ws.bad) return -3;
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long long k = 0; k < (long long)ndof; ++k) u[k] = u[k] + dt * h->du[k];
        }
        // the positivity limiter as solve_lwfr applies it: LW twice (perform_step!, src/solvers/lwfr.jl:226,
        // and the loop, :257), MDRK once (the loop; the mid-step call at src/solvers/mdrk.jl:19 acts on u^n,
        // which the previous step's application has limited already)
        if (!h->lim.thresholds.empty())
            for (int a = 0; a < (kind == 0 ? 2 : 1); ++a)
                limit(h, u);
        t += dt;
    }
    *t_inout = t;
    return s;
    } catch (const std::exception& ex) {
        std::snprintf(h->err, sizeof(h->err), "%s", ex.what());
        return -1;
    }
}

// Zhang-Shu positivity limiter pairs (PositivityPreservingLimiterZhangShu(thresholds, variables));
// variables: 0 density, 1 pressure, 2 density_pressure. count 0 switches it off.
int oracle_set_limiter(oracle_handle* h, int count, const double* thresholds, const int32_t* variables) {
    if (count < 0) return 1;
    h->lim.thresholds.assign(thresholds, thresholds + count);
    h->lim.variables.assign(variables, variables + count);
    for (int v : h->lim.variables)
        if (v < 0 || v > 2) return 1;
    return 0;
}

// one application of the limiter to u in place
int oracle_apply_limiter(oracle_handle* h, double* u) {
    limit(h, u);
    return 0;
}

const char* oracle_last_error(oracle_handle* h) { return h->err; }

}  // extern "C"
