// tlw_curved_sc.hpp -- test infrastructure only: CPU restatement of shock capturing on conforming curvilinear
// meshes as the P4estMesh{2} path of the reference computes it, used to check the CUDA kernels.
//
// Volume (calc_volume_integral!(..., ::VolumeIntegralFRShockCapturing, ...), src/solvers/dgsem_tree/
// dg_2d.jl:1648-1804, whose mesh Union covers P4estMesh{2}): the Hennemann-Gassner factor alpha_e of every
// element (density_pressure, smoothed over the interfaces), the LW volume terms scaled by (1 - alpha_e), and
//  * on blended elements (alpha_e not within 1e-12 of 0) fv_kernel! (dg_2d.jl:251-282, 326-365): du +=
//    alpha_e (w_i^-1 (f*_{i+1} - f*_i) + w_j^-1 (g*_{j+1} - g*_j)) with the subcell fluxes of Trixi's
//    curvilinear calcflux_fv! (FirstOrderReconstruction) or calcflux_muscl! (MUSCLReconstruction,
//    src/solvers/dgsem_structured/dg_2d.jl:176-311, first order on elements with a boundary face);
//  * on pure DG elements calc_fn_low! (dgsem_structured/dg_2d.jl:111-174), which evaluates only the subcell
//    faces next to the element faces and, looping over the tuple (2, nnodes), accumulates the subcell normal
//    of the last inner face from the first and the last metric increments only;
//  * load_fn_low! for P4estMesh (dgsem_tree/dg_2d.jl:236-249) stores those face-adjacent fluxes in the order
//    (bottom, right, top, left).
// Subcell normals: along xi, face f (between nodes f-1 and f) has Ja^1(0, j) + sum_{k < f} w_k sum_m
// D[k][m] Ja^1(m, j); along eta likewise with Ja^2. The subcell flux is volume_flux_fv (flux_lax_friedrichs)
// in its normal-direction form.
// Interfaces (calc_interface_flux!, src/solvers/dgsem_p4est/dg_2d.jl:149-191; prolong2interfaces!, :8-84):
// the LW flux Fn_ and the first-order flux fn at u along the primary's normal are blended by get_blended_flux
// (:227-250): alp = (alpha_P + alpha_S) / 2, Fn = (1 - alp) Fn_ + alp fn, and where the subcell update
// u - c (Fn - fn_inner) (c = dt J^{-1} / (w / 2), J^{-1} of the primary's face node for both sides) is not
// admissible, zhang_shu_flux_fix (:199-225) pulls Fn towards fn, first for density, then for pressure.
// fn_inner of a side is fn_low[:, l, direction, element] with the primary's node index l on both sides and
// the direction numbering (-xi, +xi, -eta, +eta), while load_fn_low! filled the slots as (bottom, right, top,
// left): both are kept as the reference has them. Boundary faces are not blended (dgsem_p4est/dg_2d.jl:366-393).
#pragma once
#include <cmath>
#include <vector>

#include "tlw_curved.hpp"
#include "tlw_limiter.hpp"

namespace tlwo {

enum Reconstruction { REC_FIRST_ORDER = 0, REC_MUSCL = 1, REC_MUSCL_HANCOCK = 2 };

// Trixi flux(u, normal_direction, equations) of CompressibleEulerEquations2D
inline void flux_normal(const Euler& eq, const double* u, const double* nrm, double* f) {
    double rho, v1, v2, p;
    eq.cons2prim(u, rho, v1, v2, p);
    const double vn = v1 * nrm[0] + v2 * nrm[1];
    const double rvn = rho * vn;
    f[0] = rvn;
    f[1] = rvn * v1 + p * nrm[0];
    f[2] = rvn * v2 + p * nrm[1];
    f[3] = (u[3] + p) * vn;
}

// Trixi flux_lax_friedrichs(u_ll, u_rr, normal_direction, equations)
inline void rusanov_normal(const Euler& eq, int speed_kind, const double* ul, const double* ur, const double* nrm,
                           double* out, bool& bad) {
    double fl[NV], gl[NV], fr[NV], gr[NV];
    eq.fluxes(ul, fl, gl);
    eq.fluxes(ur, fr, gr);
    const double lambda = max_abs_speed_normal(eq, ul, ur, nrm, speed_kind, bad);
    for (int v = 0; v < NV; ++v) {
        const double fnl = fl[v] * nrm[0] + gl[v] * nrm[1], fnr = fr[v] * nrm[0] + gr[v] * nrm[1];
        out[v] = 0.5 * (fnl + fnr) + (-0.5 * lambda * (ur[v] - ul[v]));
    }
}

// metric increment w_k sum_m D[k][m] Ja^d(m along the line) of contravariant direction d (0: xi, 1: eta) on
// the line `line` (j for xi, i for eta) at line position k
inline void metric_increment(const Basis& b, const double* Jae, int d, int line, int k, double* inc) {
    const int n = b.n;
    inc[0] = inc[1] = 0.0;
    for (int m = 0; m < n; ++m) {
        const double* J = Jae + 4 * (d == 0 ? m + n * line : line + n * m);
        const double c = b.weights[k] * b.D[k * n + m];
        inc[0] += c * J[2 * d];
        inc[1] += c * J[2 * d + 1];
    }
}

// Subcell fluxes of one element: X(f, j) on xi faces f = 0..n (0 and n zero), Y(i, f) on eta faces.
struct SubcellFluxes {
    int n = 0;
    std::vector<double> fx, fy;
    void init(int nn) {
        n = nn;
        fx.assign((size_t)NV * (n + 1) * n, 0.0);
        fy.assign((size_t)NV * n * (n + 1), 0.0);
    }
    double* X(int f, int j) { return fx.data() + NV * (f + (n + 1) * j); }
    double* Y(int i, int f) { return fy.data() + NV * (i + n * f); }
};

// subcell fluxes from the face states: uL(d, f, line) / uR(d, f, line) give the states left / right of inner
// face f; fn_low_only: only faces 1 and n-1, with the normal accumulated over the faces visited (calc_fn_low!)
template <class GetL, class GetR>
inline void subcell_fluxes_curved(const Basis& b, const Euler& eq, int speed_kind, const double* Jae, bool fn_low_only,
                                  GetL uL, GetR uR, SubcellFluxes& S, bool& bad) {
    const int n = b.n;
    for (int d = 0; d < 2; ++d)
        for (int line = 0; line < n; ++line) {
            // normal_direction = Ja^d at the line's first node, then the increments of the faces visited
            const double* J0 = Jae + 4 * (d == 0 ? 0 + n * line : line + 0);
            double nrm[2] = {J0[2 * d], J0[2 * d + 1]};
            for (int f = 1; f < n; ++f) {
                if (fn_low_only && f != 1 && f != n - 1) continue;
                double inc[2];
                metric_increment(b, Jae, d, line, f - 1, inc);
                nrm[0] += inc[0];
                nrm[1] += inc[1];
                double out[NV];
                rusanov_normal(eq, speed_kind, uL(d, f, line), uR(d, f, line), nrm, out, bad);
                double* dst = d == 0 ? S.X(f, line) : S.Y(line, f);
                for (int v = 0; v < NV; ++v) dst[v] = out[v];
            }
        }
}

// Julia sign
inline double julia_sign(double x) { return x == 0.0 || std::isnan(x) ? x : (x > 0.0 ? 1.0 : -1.0); }

// minmod(a, b, Mdx2) of dgsem_structured/dg_2d.jl:97-109 (Julia min propagates NaN; NaN signs differ)
inline double minmod2(double a, double b, double Mdx2) {
    if (std::fabs(b) < Mdx2 && std::fabs(a) < Mdx2) return b;
    const double slope = julia_min(std::fabs(a), std::fabs(b));
    const double s1 = julia_sign(a), s2 = julia_sign(b);
    if (s1 != s2) return 0.0;
    return s1 * slope;
}

// limit_variable_slope (src/equations/equations.jl:262-287) for `variable` (LIMIT_DENSITY / LIMIT_PRESSURE)
inline void limit_variable_slope(const Euler& eq, int variable, double* slope, double* usl, double* usr,
                                 const double* ue, double xl, double xr) {
    const double vsl = limiter_value(eq, variable, usl), vsr = limiter_value(eq, variable, usr);
    const double vlow = limiter_value(eq, variable, ue);
    const double eps = 1e-10;
    const double threshold = 0.1 * vlow;
    if (vsl < eps || vsr < eps) {
        const double rl = std::fabs(threshold - vlow) / (std::fabs(vsl - vlow) + 1e-13);
        const double rr = std::fabs(threshold - vlow) / (std::fabs(vsr - vlow) + 1e-13);
        const double theta = julia_min(julia_min(rl, rr), 1.0);
        for (int v = 0; v < NV; ++v) {
            slope[v] *= theta;
            usl[v] = ue[v] + (2.0 * theta) * (xl * slope[v]);
            usr[v] = ue[v] + (2.0 * theta) * (xr * slope[v]);
        }
    }
}

// limit_slope (src/equations/compressible_euler_2d.jl:9-21): density, then pressure; face values from the slope
inline void limit_slope(const Euler& eq, double* slope, double* usl, double* usr, const double* ue, double xl,
                        double xr, double* ufl, double* ufr) {
    limit_variable_slope(eq, LIMIT_DENSITY, slope, usl, usr, ue, xl, xr);
    limit_variable_slope(eq, LIMIT_PRESSURE, slope, usl, usr, ue, xl, xr);
    for (int v = 0; v < NV; ++v) {
        ufl[v] = ue[v] + slope[v] * xl;
        ufr[v] = ue[v] + slope[v] * xr;
    }
}

// compute_subcells (dgsem_tree/dg_2d.jl:1806-1824): subcell faces and the extended node positions
struct Subcells {
    std::vector<double> faces;   // [0..n]: -1, -1 + w_0, ..., 1
    std::vector<double> xi_ext;  // [0..n+1]: -1, nodes, 1
};
inline Subcells compute_subcells(const Basis& b) {
    const int n = b.n;
    Subcells s;
    s.faces.assign(n + 1, -1.0);
    for (int i = 1; i <= n; ++i) {
        double acc = 0.0;
        for (int k = 0; k < i; ++k) acc += b.weights[k];
        s.faces[i] = -1.0 + acc;
    }
    s.xi_ext.assign(n + 2, -1.0);
    for (int i = 0; i < n; ++i) s.xi_ext[i + 1] = b.nodes[i];
    s.xi_ext[n + 1] = 1.0;
    return s;
}

// The face values of the MUSCL reconstruction of one element (calcflux_muscl!, dgsem_structured/dg_2d.jl:
// 196-253): uf[node][k][v], k = 0 left, 1 right, 2 down, 3 up; element-local (the extended state copies the
// edge nodes, so the one-sided difference into the copy is 0 / 0 and the edge subcells get a zero slope)
inline void muscl_face_values(const Basis& b, const Euler& eq, const Subcells& sc, const double* u, int e,
                              std::vector<double>& uf) {
    const int n = b.n;
    uf.assign((size_t)4 * NV * n * n, 0.0);
    auto ue = [&](int i, int j) {   // extended indices 0..n+1
        i = std::min(std::max(i, 1), n);
        j = std::min(std::max(j, 1), n);
        return u + idx_u(n, 0, i - 1, j - 1, e);
    };
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) {
            const double *u_ = ue(i, j), *ul = ue(i - 1, j), *ur = ue(i + 1, j), *ud = ue(i, j - 1),
                         *uu = ue(i, j + 1);
            const double dx1 = sc.xi_ext[i] - sc.xi_ext[i - 1], dx2 = sc.xi_ext[i + 1] - sc.xi_ext[i];
            const double dy1 = sc.xi_ext[j] - sc.xi_ext[j - 1], dy2 = sc.xi_ext[j + 1] - sc.xi_ext[j];
            double sx[NV], sy[NV];
            for (int v = 0; v < NV; ++v) {
                const double bx = (u_[v] - ul[v]) / dx1, fx = (ur[v] - u_[v]) / dx2;
                const double by = (u_[v] - ud[v]) / dy1, fy = (uu[v] - u_[v]) / dy2;
                sx[v] = minmod2(bx, fx, 0.0);
                sy[v] = minmod2(by, fy, 0.0);
            }
            const double xl = sc.faces[i - 1] - sc.xi_ext[i], xr = sc.faces[i] - sc.xi_ext[i];
            const double yl = sc.faces[j - 1] - sc.xi_ext[j], yr = sc.faces[j] - sc.xi_ext[j];
            double usl[NV], usr[NV], usd[NV], usu[NV];
            for (int v = 0; v < NV; ++v) {
                usl[v] = u_[v] + 2.0 * sx[v] * xl;
                usr[v] = u_[v] + 2.0 * sx[v] * xr;
                usd[v] = u_[v] + 2.0 * sy[v] * yl;
                usu[v] = u_[v] + 2.0 * sy[v] * yr;
            }
            double* o = uf.data() + (size_t)4 * NV * ((i - 1) + n * (j - 1));
            limit_slope(eq, sx, usl, usr, u_, xl, xr, o + 0 * NV, o + 1 * NV);
            limit_slope(eq, sy, usd, usu, u_, yl, yr, o + 2 * NV, o + 3 * NV);
        }
}

// minmod(a, b, c, beta, Mdx2) of dgsem_structured/dg_2d.jl:83-95 (with Mdx2 = 0)
inline double minmod3(double a, double b, double c, double beta) {
    const double slope = julia_min(julia_min(beta * std::fabs(a), std::fabs(b)), beta * std::fabs(c));
    const double s1 = julia_sign(a), s2 = julia_sign(b), s3 = julia_sign(c);
    if (s1 != s2 || s2 != s3) return 0.0;
    return s1 * slope;
}

// The half-step face values of the MUSCL-Hancock reconstruction of one element (calcflux_mh!,
// dgsem_structured/dg_2d.jl:313-483): slopes from minmod(backward, centred, forward; beta = 2 - alpha) of the
// element-local extended state (finite_differences, :75-81), limited face values as in MUSCL, then every face
// value of a subcell gets the same multi-D half-step increment, built as the reference builds it: along xi,
// cell c receives +dt/2 J^{-1}(c) / w_{c+1} f(u_left(c)).n_c (1 <= c <= n-2) and -dt/2 J^{-1}(c) / w_{c+1}
// f(u_right(c)).n_{c+1} (c <= n-2); along eta, +dt/2 J^{-1}(c+1) / w_{c+1} f(u_down(c)).n_c and -dt/2
// J^{-1}(c+1) / w_{c+1} f(u_up(c)).n_{c+1} (the next cell's J^{-1}), with the subcell normals n.
inline void muscl_hancock_face_values(const Basis& b, const Euler& eq, const Subcells& sc, const double* Jae,
                                      const double* ije, const double* u, int e, double alpha, double dt,
                                      std::vector<double>& uf) {
    const int n = b.n;
    uf.assign((size_t)4 * NV * n * n, 0.0);
    auto ue = [&](int i, int j) {
        i = std::min(std::max(i, 1), n);
        j = std::min(std::max(j, 1), n);
        return u + idx_u(n, 0, i - 1, j - 1, e);
    };
    const double beta = 2.0 - alpha;
    for (int j = 1; j <= n; ++j)
        for (int i = 1; i <= n; ++i) {
            const double *u_ = ue(i, j), *ul = ue(i - 1, j), *ur = ue(i + 1, j), *ud = ue(i, j - 1),
                         *uu = ue(i, j + 1);
            const double h1x = sc.xi_ext[i] - sc.xi_ext[i - 1], h2x = sc.xi_ext[i + 1] - sc.xi_ext[i];
            const double h1y = sc.xi_ext[j] - sc.xi_ext[j - 1], h2y = sc.xi_ext[j + 1] - sc.xi_ext[j];
            const double ax = -(h2x / (h1x * (h1x + h2x))), bx = (h2x - h1x) / (h1x * h2x), cx = (h1x / (h2x * (h1x + h2x)));
            const double ay = -(h2y / (h1y * (h1y + h2y))), by = (h2y - h1y) / (h1y * h2y), cy = (h1y / (h2y * (h1y + h2y)));
            double sx[NV], sy[NV];
            for (int v = 0; v < NV; ++v) {
                const double bkx = (u_[v] - ul[v]) / h1x, fwx = (ur[v] - u_[v]) / h2x;
                const double cnx = ax * ul[v] + bx * u_[v] + cx * ur[v];
                const double bky = (u_[v] - ud[v]) / h1y, fwy = (uu[v] - u_[v]) / h2y;
                const double cny = ay * ud[v] + by * u_[v] + cy * uu[v];
                sx[v] = minmod3(bkx, cnx, fwx, beta);
                sy[v] = minmod3(bky, cny, fwy, beta);
            }
            const double xl = sc.faces[i - 1] - sc.xi_ext[i], xr = sc.faces[i] - sc.xi_ext[i];
            const double yl = sc.faces[j - 1] - sc.xi_ext[j], yr = sc.faces[j] - sc.xi_ext[j];
            double usl[NV], usr[NV], usd[NV], usu[NV];
            for (int v = 0; v < NV; ++v) {
                usl[v] = u_[v] + 2.0 * sx[v] * xl;
                usr[v] = u_[v] + 2.0 * sx[v] * xr;
                usd[v] = u_[v] + 2.0 * sy[v] * yl;
                usu[v] = u_[v] + 2.0 * sy[v] * yr;
            }
            double* o = uf.data() + (size_t)4 * NV * ((i - 1) + n * (j - 1));
            limit_slope(eq, sx, usl, usr, u_, xl, xr, o + 0 * NV, o + 1 * NV);
            limit_slope(eq, sy, usd, usu, u_, yl, yr, o + 2 * NV, o + 3 * NV);
        }
    // the half-step increments, from the limited face values of each cell (0-based cell c = (i, j))
    auto normal = [&](int d, int line, int f, double* nrm) {   // subcell face f (1..n-1) of line `line`
        const double* J0 = Jae + 4 * (d == 0 ? 0 + n * line : line + 0);
        nrm[0] = J0[2 * d];
        nrm[1] = J0[2 * d + 1];
        for (int k = 0; k < f; ++k) {
            double o[2];
            metric_increment(b, Jae, d, line, k, o);
            nrm[0] += o[0];
            nrm[1] += o[1];
        }
    };
    std::vector<double> unph = uf;
    auto F = [&](int i, int j, int k) { return uf.data() + (size_t)4 * NV * (i + n * j) + NV * k; };
    auto add = [&](int i, int j, const double* r) {
        for (int k = 0; k < 4; ++k)
            for (int v = 0; v < NV; ++v) unph[(size_t)4 * NV * (i + n * j) + NV * k + v] += r[v];
    };
    // xi lines: faces f = 1..n-1 in order; at face f the cell f-1 gets its "ll" part, the cell f (f < n-1) its
    // "rr" part
    for (int j = 0; j < n; ++j)
        for (int f = 1; f < n; ++f) {
            double nrm[2], fl[NV], r[NV];
            normal(0, j, f, nrm);
            flux_normal(eq, F(f - 1, j, 1), nrm, fl);
            const double cl = -0.5 * dt * ije[(f - 1) + n * j] / b.weights[f];
            for (int v = 0; v < NV; ++v) r[v] = cl * fl[v];
            add(f - 1, j, r);
            if (f < n - 1) {
                flux_normal(eq, F(f, j, 0), nrm, fl);
                const double cr = 0.5 * dt * ije[f + n * j] / b.weights[f + 1];
                for (int v = 0; v < NV; ++v) r[v] = cr * fl[v];
                add(f, j, r);
            }
        }
    for (int i = 0; i < n; ++i)
        for (int f = 1; f < n; ++f) {
            double nrm[2], fl[NV], r[NV];
            normal(1, i, f, nrm);
            flux_normal(eq, F(i, f - 1, 3), nrm, fl);
            const double cd = -0.5 * dt * ije[i + n * f] / b.weights[f];
            for (int v = 0; v < NV; ++v) r[v] = cd * fl[v];
            add(i, f - 1, r);
            if (f < n - 1) {
                flux_normal(eq, F(i, f, 2), nrm, fl);
                const double cu = 0.5 * dt * ije[i + n * (f + 1)] / b.weights[f + 1];
                for (int v = 0; v < NV; ++v) r[v] = cu * fl[v];
                add(i, f, r);
            }
        }
    uf.swap(unph);
}

// One element's subcell pass: blended elements add alpha_e times the FV divergence to du; every element fills
// its fn_low slots (P4est order: bottom, right, top, left).
// dt_fv: the time step fv_kernel! is given (MUSCL-Hancock's half step: dt for LW and MDRK stage 2, dt / 2 for
// MDRK stage 1, src/solvers/dgsem_tree/multi_derivative_2d.jl:199, 256).
inline void curved_subcells(const Basis& b, const Euler& eq, const Options& opt, const CurvedMesh& m,
                            const Subcells& sc, const std::vector<char>& at_boundary, int e, const double* u,
                            double* du, double alpha, bool blended, Workspace& ws, bool& bad, double dt_fv = 0.0) {
    const int n = b.n, nn = n * n;
    const double* Jae = &m.Ja[4 * (size_t)nn * e];
    SubcellFluxes S;
    S.init(n);
    auto node = [&](int i, int j) { return u + idx_u(n, 0, i, j, e); };
    // the states left / right of inner face f on line `line` of direction d from the nodes
    auto nodeL = [&](int d, int f, int line) { return d == 0 ? node(f - 1, line) : node(line, f - 1); };
    auto nodeR = [&](int d, int f, int line) { return d == 0 ? node(f, line) : node(line, f); };
    if (!blended) {
        subcell_fluxes_curved(b, eq, opt.speed_kind, Jae, true, nodeL, nodeR, S, bad);
    } else if ((opt.reconstruction == REC_MUSCL || opt.reconstruction == REC_MUSCL_HANCOCK) && !at_boundary[e]) {
        std::vector<double> uf;
        if (opt.reconstruction == REC_MUSCL) muscl_face_values(b, eq, sc, u, e, uf);
        else muscl_hancock_face_values(b, eq, sc, Jae, &m.inv_jac[(size_t)nn * e], u, e, alpha, dt_fv, uf);
        auto F = [&](int i, int j, int k) { return uf.data() + (size_t)4 * NV * (i + n * j) + NV * k; };
        // u_ll: the right (up) face value of the node before the face, u_rr: the left (down) value after it
        auto fL = [&](int d, int f, int line) { return d == 0 ? F(f - 1, line, 1) : F(line, f - 1, 3); };
        auto fR = [&](int d, int f, int line) { return d == 0 ? F(f, line, 0) : F(line, f, 2); };
        subcell_fluxes_curved(b, eq, opt.speed_kind, Jae, false, fL, fR, S, bad);
    } else {
        subcell_fluxes_curved(b, eq, opt.speed_kind, Jae, false, nodeL, nodeR, S, bad);
    }
    if (blended) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int v = 0; v < NV; ++v)
                    du[idx_u(n, v, i, j, e)] += alpha * (1.0 / b.weights[i] * (S.X(i + 1, j)[v] - S.X(i, j)[v]) +
                                                         1.0 / b.weights[j] * (S.Y(i, j + 1)[v] - S.Y(i, j)[v]));
    }
    for (int l = 0; l < n; ++l)
        for (int v = 0; v < NV; ++v) {
            ws.fn_low[v + NV * (l + n * (0 + 4 * (size_t)e))] = S.Y(l, 1)[v];       // bottom
            ws.fn_low[v + NV * (l + n * (1 + 4 * (size_t)e))] = S.X(n - 1, l)[v];   // right
            ws.fn_low[v + NV * (l + n * (2 + 4 * (size_t)e))] = S.Y(l, n - 1)[v];   // top
            ws.fn_low[v + NV * (l + n * (3 + 4 * (size_t)e))] = S.X(1, l)[v];       // left
        }
}

// Hennemann-Gassner factors on a curvilinear mesh, smoothed over its interfaces (Trixi apply_smoothing!)
inline void indicator_curved(const Basis& b, const Euler& eq, const Options& opt, const CurvedMesh& m, const double* u,
                             std::vector<double>& alpha) {
    TreeMesh none;
    none.n_elements = m.n_elements;
    none.n_interfaces = 0;
    Options o = opt;
    o.alpha_smooth = false;
    indicator_hennemann_gassner(b, eq, o, none, u, alpha);
    if (opt.alpha_smooth) {
        const std::vector<double> tmp = alpha;
        auto pair = [&](int l, int r) {
            alpha[l] = std::max(std::max(tmp[l], 0.5 * tmp[r]), alpha[l]);
            alpha[r] = std::max(std::max(tmp[r], 0.5 * tmp[l]), alpha[r]);
        };
        for (int k = 0; k < m.n_interfaces; ++k) pair(m.p_elem[k], m.s_elem[k]);
        // Trixi's apply_smoothing! for a P4estMesh continues over the mortars: each small element with the
        // large one
        for (int k = 0; k < m.n_mortars; ++k) {
            pair(m.m_small1[k], m.m_large[k]);
            pair(m.m_small2[k], m.m_large[k]);
        }
    }
}

// zhang_shu_flux_fix (src/solvers/dgsem_p4est/dg_2d.jl:199-225)
inline void zhang_shu_flux_fix(const Euler& eq, const double* uprev, const double* ulow, double* Fn,
                               const double* fn_inner, const double* fn, double c) {
    double uhigh[NV];
    for (int v = 0; v < NV; ++v) uhigh[v] = uprev[v] - c * (Fn[v] - fn_inner[v]);
    double lo = ulow[0], hi = uhigh[0];
    double eps = 0.1 * lo;
    double theta = julia_min(std::fabs(eps - lo) / (std::fabs(hi - lo) + 1e-13), 1.0);
    if (theta < 1.0)
        for (int v = 0; v < NV; ++v) Fn[v] = theta * Fn[v] + (1.0 - theta) * fn[v];
    for (int v = 0; v < NV; ++v) uhigh[v] = uprev[v] - c * (Fn[v] - fn_inner[v]);
    lo = limiter_value(eq, LIMIT_PRESSURE, ulow);
    hi = limiter_value(eq, LIMIT_PRESSURE, uhigh);
    eps = 0.1 * lo;
    theta = julia_min(std::fabs(eps - lo) / (std::fabs(hi - lo) + 1e-13), 1.0);
    if (theta < 1.0)
        for (int v = 0; v < NV; ++v) Fn[v] = theta * Fn[v] + (1.0 - theta) * fn[v];
}

// get_blended_flux (src/solvers/dgsem_p4est/dg_2d.jl:227-250); J = the primary face node's J^{-1}. Returns which
// sides took zhang_shu_flux_fix: bit 0 the primary (ll), bit 1 the secondary (rr).
inline int get_blended_flux(const Basis& b, const Euler& eq, const double* u_ll, const double* u_rr, double alpha_p,
                             double alpha_s, double J, double dt, const double* fn, const double* Fn_,
                             const double* fil, const double* fir, double* Fn) {
    const int n = b.n;
    const double alp = 0.5 * (alpha_p + alpha_s);
    for (int v = 0; v < NV; ++v) Fn[v] = (1.0 - alp) * Fn_[v] + alp * fn[v];
    const double lam = 0.5;
    const double c_ll = dt * J / (b.weights[n - 1] * lam);
    double test[NV], low[NV];
    for (int v = 0; v < NV; ++v) {
        test[v] = u_ll[v] - c_ll * (Fn[v] - fil[v]);
        low[v] = u_ll[v] - c_ll * (fn[v] - fil[v]);
    }
    int fixed = 0;
    if (!eq.is_admissible(test)) {
        zhang_shu_flux_fix(eq, u_ll, low, Fn, fil, fn, c_ll);
        fixed |= 1;
    }
    const double c_rr = -dt * J / (b.weights[0] * lam);
    for (int v = 0; v < NV; ++v) {
        test[v] = u_rr[v] - c_rr * (Fn[v] - fir[v]);
        low[v] = u_rr[v] - c_rr * (fn[v] - fir[v]);
    }
    if (!eq.is_admissible(test)) {
        zhang_shu_flux_fix(eq, u_rr, low, Fn, fir, fn, c_rr);
        fixed |= 2;
    }
    return fixed;
}

// du = rhs(u) with VolumeIntegralFRShockCapturing on a conforming curvilinear mesh (Rusanov surface flux); the
// factors of the call are left in ws.alpha. kind 0: LW; 1: rhs_mdrk1!; 2: rhs_mdrk2! with the stage state u2 in
// the DG volume terms (calc_volume_integral_mdrk1! / _mdrk2!, src/solvers/dgsem_tree/multi_derivative_2d.jl:
// 150-262: the indicator and the subcells take u in both stages; the interfaces blend with the full dt and the
// instantaneous u, the boundaries of stage 1 halve their time averages).
// compute_alp for Union{StructuredMesh, UnstructuredMesh2D} (src/solvers/dgsem_structured/dg_2d.jl:2169-2191), as
// the UnstructuredMesh2D interface calls it (dgsem_unstructured_2d/dg_2d.jl:255-262): alp = (alpha_P + alpha_S) / 2,
// or 1 when the first-order subcell update of either side with the blended flux is not admissible; the updates
// start from the time-averaged U of each side (the call passes U as u_ll / u_rr) with J^{-1} of the primary's face
// node (load_inverse_jacobian!, :452-472) for both. The interface flux is then alp fn + (1 - alp) Fn_. fn_low is
// oriented along +xi / +eta, so the primary's test has the sign of its outward flux only when its side is the right
// or the top one; restated as written (the result depends on which element an interface lists first).
inline double compute_alp_unstructured(const Basis& b, const Euler& eq, const double* U_ll, const double* U_rr,
                                       double alpha_p, double alpha_s, double J, double dt, const double* fn,
                                       const double* Fn_, const double* fil, const double* fir) {
    const double alp = 0.5 * (alpha_p + alpha_s);
    double Fn[NV], low[NV];
    for (int v = 0; v < NV; ++v) Fn[v] = (1.0 - alp) * Fn_[v] + alp * fn[v];
    const double lam = 0.5;
    for (int v = 0; v < NV; ++v) low[v] = U_ll[v] - dt * J / (b.weights[b.n - 1] * lam) * (Fn[v] - fil[v]);
    if (!eq.is_admissible(low)) return 1.0;
    for (int v = 0; v < NV; ++v) low[v] = U_rr[v] - dt * J / (b.weights[0] * lam) * (fir[v] - Fn[v]);
    if (!eq.is_admissible(low)) return 1.0;
    return alp;
}

inline void rhs_curved_sc(const Basis& b, const Euler& eq, const Options& opt, const CurvedMesh& m, const double* u,
                          double* du, double dt, Workspace& ws, int nthreads = 1, const BoundaryData* bd = nullptr,
                          int kind = 0, const double* u2 = nullptr) {
    if (opt.flux_kind != RUSANOV) throw std::invalid_argument("curvilinear shock capturing: Rusanov surface flux");
    const int n = b.n, nn = n * n;
    const size_t ndof = (size_t)NV * nn * m.n_elements;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    ws.U.assign(ndof, nan);
    ws.F.assign(2 * ndof, nan);
    ws.surface_flux_values.assign((size_t)NV * n * 4 * m.n_elements, nan);
    ws.fn_low.assign((size_t)NV * n * 4 * m.n_elements, 0.0);
    ws.bad = false;
    if (opt.temporal_errors && kind == 0) ws.temporal_errors.assign(m.n_elements, nan);
    if (kind == 1) {
        ws.U2.assign(ndof, nan);
        ws.F2.assign(2 * ndof, nan);
    }
    if (kind == 2 && (ws.U2.size() != ndof || !u2)) throw std::invalid_argument("rhs_mdrk2 before rhs_mdrk1");
    check_unstructured(m, kind);
    for (size_t k = 0; k < ndof; ++k) du[k] = 0.0;
    indicator_curved(b, eq, opt, m, u, ws.alpha);
    const Subcells sc = compute_subcells(b);
    std::vector<char> at_boundary(m.n_elements, 0);
    for (int k = 0; k < m.n_boundaries; ++k) at_boundary[m.b_elem[k]] = 1;
    bool bad = false;
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad)
    for (int e = 0; e < m.n_elements; ++e) {
        const double a = ws.alpha[e];
        const double* Jae = &m.Ja[4 * (size_t)nn * e];
        const double* ije = &m.inv_jac[(size_t)nn * e];
        if (kind == 0) lw_volume_element_curved(b, eq, opt.N, m, e, u, du, dt, ws, 1.0 - a, &opt);
        else if (kind == 1) mdrk1_volume_element(b, eq, e, u, du, dt, 0.0, 1.0 - a, ws, Jae, ije);
        else mdrk2_volume_element(b, eq, e, u2, du, dt, 0.0, 1.0 - a, ws, Jae, ije);
        // pure_and_blended_element_ids!: DG only where isapprox(alpha, 0, atol = 1e-12)
        const bool blended = !(std::fabs(a) <= 1e-12);
        bool b_ = false;
        curved_subcells(b, eq, opt, m, sc, at_boundary, e, u, du, a, blended, ws, b_, kind == 1 ? 0.5 * dt : dt);
        bad = bad || b_;
    }
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(|| : bad)
    for (int k = 0; k < m.n_interfaces; ++k) {
        const int pe = m.p_elem[k], pf = m.p_face[k], se = m.s_elem[k], sf = m.s_face[k];
        for (int l = 0; l < n; ++l) {
            const int ls = m.s_rev[k] ? n - 1 - l : l;
            if (!m.unormals.empty()) {
                // UnstructuredMesh2D (dgsem_unstructured_2d/dg_2d.jl:211-280): fn_low by side, each side at its
                // own node index (the interface cache keeps them by local index, :72-75, read at :236-243)
                double nP[2], Fn_[NV], fn[NV], u_ll[NV], u_rr[NV], U_ll[NV], U_rr[NV], fil[NV], fir[NV];
                bool b_ = false;
                unstructured_interface_node(eq, opt, m, n, u, ws, pe, pf, se, sf, l, ls, nP, Fn_, u_ll, u_rr, U_ll,
                                            U_rr, b_);
                rusanov_normal(eq, opt.speed_kind, u_ll, u_rr, nP, fn, b_);
                bad = bad || b_;
                for (int v = 0; v < NV; ++v) {
                    fil[v] = ws.fn_low[v + NV * (l + n * (fn_low_slot(pf) + 4 * (size_t)pe))];
                    fir[v] = ws.fn_low[v + NV * (ls + n * (fn_low_slot(sf) + 4 * (size_t)se))];
                }
                int ip, jp;
                face_node(n, pf, l, ip, jp);
                const double J = m.inv_jac[ip + n * (jp + (size_t)n * pe)];
                const double alp = compute_alp_unstructured(b, eq, U_ll, U_rr, ws.alpha[pe], ws.alpha[se], J, dt, fn,
                                                            Fn_, fil, fir);
                for (int v = 0; v < NV; ++v) {
                    const double F = alp * fn[v] + (1.0 - alp) * Fn_[v];
                    ws.surface_flux_values[v + NV * (l + n * (pf + 4 * (size_t)pe))] = F;
                    ws.surface_flux_values[v + NV * (ls + n * (sf + 4 * (size_t)se))] = -F;
                }
                continue;
            }
            int ip, jp, is, js;
            face_node(n, pf, l, ip, jp);
            face_node(n, sf, ls, is, js);
            double nP[2], nS[2], f_ll[NV], f_rr[NV], u_ll[NV], u_rr[NV], U_ll[NV], U_rr[NV], Fn_[NV], fn[NV];
            double fil[NV], fir[NV], Fn[NV];
            outward_normal(m, n, pf, ip, jp, pe, nP);
            outward_normal(m, n, sf, is, js, se, nS);
            for (int v = 0; v < NV; ++v) {
                f_ll[v] = ws.F[idx_F(n, v, 0, ip, jp, pe)] * nP[0] + ws.F[idx_F(n, v, 1, ip, jp, pe)] * nP[1];
                f_rr[v] = ws.F[idx_F(n, v, 0, is, js, se)] * (-nS[0]) + ws.F[idx_F(n, v, 1, is, js, se)] * (-nS[1]);
                u_ll[v] = u[idx_u(n, v, ip, jp, pe)];
                u_rr[v] = u[idx_u(n, v, is, js, se)];
                U_ll[v] = ws.U[idx_u(n, v, ip, jp, pe)];
                U_rr[v] = ws.U[idx_u(n, v, is, js, se)];
                // the primary's node index on both sides, slots as load_fn_low! filled them
                fil[v] = ws.fn_low[v + NV * (l + n * (pf + 4 * (size_t)pe))];
                fir[v] = ws.fn_low[v + NV * (l + n * (sf + 4 * (size_t)se))];
            }
            bool b_ = false;
            lw_surface_flux_normal(eq, opt.flux_kind, opt.speed_kind, f_ll, f_rr, u_ll, u_rr, U_ll, U_rr, nP, Fn_, b_);
            rusanov_normal(eq, opt.speed_kind, u_ll, u_rr, nP, fn, b_);
            const double J = m.inv_jac[ip + n * (jp + (size_t)n * pe)];
            get_blended_flux(b, eq, u_ll, u_rr, ws.alpha[pe], ws.alpha[se], J, dt, fn, Fn_, fil, fir, Fn);
            bad = bad || b_;
            for (int v = 0; v < NV; ++v) {
                ws.surface_flux_values[v + NV * (l + n * (pf + 4 * (size_t)pe))] = Fn[v];
                ws.surface_flux_values[v + NV * (ls + n * (sf + 4 * (size_t)se))] = -Fn[v];
            }
        }
    }
    ws.bad = ws.bad || bad;
    // mortars (calc_mortar_flux!, src/solvers/dgsem_p4est/dg_2d.jl:506-603): get_blended_flux with the small
    // element as the primary, u_rr the large element's u interpolated onto the small node, fn the first-order
    // flux along the small element's normal, fn_inner_ll the small element's fn_low slot of its face at the
    // node, fn_inner_rr the large element's fn_low slot of its face read in mortar order (index i, no
    // reversal) and interpolated like u (prolong2mortars!, :429-500), and J^{-1} = lw_mortars.inverse_jacobian
    bad = false;
    ws.mortar_fixes.assign(2, 0.0);
    auto mortar_blend = [&](int k, int h, int l, int se, const double* u_ll, const double* u_rr, const double* nS,
                            double* fstar) {
        const int lg = m.m_large[k], lf = m.m_lface[k], sf = m.m_sface[k];
        const std::vector<double>& fwd = h ? b.fwd_upper : b.fwd_lower;
        double fil[NV], fir[NV] = {0, 0, 0, 0}, fn[NV], Fn[NV];
        for (int v = 0; v < NV; ++v) fil[v] = ws.fn_low[v + NV * (l + n * (sf + 4 * (size_t)se))];
        for (int i = 0; i < n; ++i)
            for (int v = 0; v < NV; ++v) fir[v] += fwd[l * n + i] * ws.fn_low[v + NV * (i + n * (lf + 4 * (size_t)lg))];
        bool b_ = false;
        rusanov_normal(eq, opt.speed_kind, u_ll, u_rr, nS, fn, b_);
        bad = bad || b_;
        const double J = m.m_ij.empty() ? 0.0 : m.m_ij[(size_t)k * n + l];
        const int fixed =
            get_blended_flux(b, eq, u_ll, u_rr, ws.alpha[se], ws.alpha[lg], J, dt, fn, fstar, fil, fir, Fn);
        if (fixed & 1) ws.mortar_fixes[0] += 1.0;
        if (fixed & 2) ws.mortar_fixes[1] += 1.0;
        for (int v = 0; v < NV; ++v) fstar[v] = Fn[v];
    };
    calc_mortar_flux_curved(b, eq, opt, m, u, ws, bad, mortar_blend);
    ws.bad = ws.bad || bad;
    calc_boundary_flux_curved(b, eq, opt, m, u, ws, bd, kind == 1 ? 0.5 : 1.0);
    surface_integral_and_jacobian_curved(b, m, du, ws, nthreads);
}

// limit_mortars! for P4estMesh{2} (src/callbacks/callbacks_stage/positivity_zhang_shu_dg2d.jl:178-260): per
// mortar in order, the large element's face in the mortar's forward order interpolated onto both halves; the
// minimum of the variable over the first four nodes of each half (the loop `for i = 1:4`); theta = min(|(mean -
// threshold) / (mean - min)|, 1) blends the large element unconditionally.
inline void limit_mortars_p4est(const Basis& b, const Euler& eq, const CurvedMesh& m, double* u, double threshold,
                                int variable) {
    const int n = b.n;
    std::vector<double> face(n * NV);
    for (int k = 0; k < m.n_mortars; ++k) {
        const int le = m.m_large[k], lf = m.m_lface[k];
        const bool rev = m.m_lrev[k] != 0;
        for (int i = 0; i < n; ++i) {
            int il, jl;
            face_node(n, lf, rev ? n - 1 - i : i, il, jl);
            for (int v = 0; v < NV; ++v) face[i * NV + v] = u[idx_u(n, v, il, jl, le)];
        }
        double mean[NV];
        element_mean(b, u, le, mean);
        const double vmean = limiter_value(eq, variable, mean);
        double vmin = std::numeric_limits<double>::infinity();
        for (int jm = 0; jm < std::min(4, n); ++jm) {
            double lo[NV] = {0, 0, 0, 0}, up[NV] = {0, 0, 0, 0};
            for (int l = 0; l < n; ++l)
                for (int v = 0; v < NV; ++v) {
                    lo[v] += b.fwd_lower[jm * n + l] * face[l * NV + v];
                    up[v] += b.fwd_upper[jm * n + l] * face[l * NV + v];
                }
            vmin = julia_min(julia_min(vmin, limiter_value(eq, variable, lo)), limiter_value(eq, variable, up));
        }
        const double theta = julia_min(std::fabs((vmean - threshold) / (vmean - vmin)), 1.0);
        blend_element(b, u, le, theta, mean);
    }
}

// one application of the limiter on a curvilinear mesh: every pair in order, elements then the mortars
inline void apply_positivity_limiter_curved(const Basis& b, const Euler& eq, const CurvedMesh& m,
                                            const PositivityLimiter& lim, double* u) {
    for (size_t p = 0; p < lim.thresholds.size(); ++p) {
        limit_elements(b, eq, m.n_elements, u, lim.thresholds[p], lim.variables[p]);
        if (m.n_mortars > 0) limit_mortars_p4est(b, eq, m, u, lim.thresholds[p], lim.variables[p]);
    }
}

}  // namespace tlwo
