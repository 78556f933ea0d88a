// tlw_curved.cuh -- surface and CFL kernels for conforming curvilinear meshes (StructuredMesh{2}, and
// P4estMesh{2} / UnstructuredMesh2D without mortars). The volume kernel is lw_volume_kernel<..., CURVED>.
//
// An interface is (primary element, face; secondary element, face; whether the secondary's face index runs
// backwards), faces 0: -xi, 1: +xi, 2: -eta, 3: +eta. The volume kernel leaves, per face node, the time
// averaged U and the contravariant flux along the face's coordinate direction (F~ on xi faces, G~ on eta
// faces), i.e. the physical flux dotted with +Ja^1 / +Ja^2 of that node. With sigma = +1 on faces 1, 3 and -1
// on faces 0, 2 the outward normal flux of a side is sigma * trace. As prolong2interfaces! and
// calc_interface_flux! for P4estMesh{2} (src/solvers/dgsem_p4est/dg_2d.jl:8-191):
//   n     = outward normal of the primary at the node (get_normal_direction: sigma_P Ja^d_P)
//   f_ll  = F_P . n_P (its own outward normal), f_rr = F_S . (-n_S) (the secondary's own normal, negated)
//   Fn    = surface_flux(f_ll, f_rr, u_P, u_S, U_P, U_S, n)   (curvilinear argument order: Rusanov speed from
//           the instantaneous u, jump in the time-averaged U; HLL speeds from U, jump in u)
//   outward flux Fn on the primary, -Fn on the secondary; surface integral + apply_jacobian:
//   du(face node) += -J^{-1}(node) / w_face * outward flux.
// Corner nodes are shared by an element's xi and eta faces, so the host colours the interfaces such that no
// launch touches both classes of faces of one element (two colours on a StructuredMesh); the launches of
// one step run in colour order on one stream.
#pragma once
#include "tlw_device.cuh"
#include "tlw_surface.cuh"

namespace tlw {

// Trixi max_abs_speed_naive (kind 0) / max_abs_speed (kind 1) with a normal direction
__device__ __forceinline__ double max_abs_speed_normal(double gamma, const double* ul, const double* ur,
                                                       const double* nrm, int kind, unsigned* status) {
    const double gm1 = gamma - 1.0;
    const double irl = 1.0 / ul[0], irr = 1.0 / ur[0];
    const double v1l = ul[1] * irl, v2l = ul[2] * irl, v1r = ur[1] * irr, v2r = ur[2] * irr;
    const double pl = gm1 * (ul[3] - 0.5 * (ul[1] * v1l + ul[2] * v2l));
    const double pr = gm1 * (ur[3] - 0.5 * (ur[1] * v1r + ur[2] * v2r));
    const double vl = v1l * nrm[0] + v2l * nrm[1];
    const double vr = v1r * nrm[0] + v2r * nrm[1];
    const double cl = checked_sqrt(gamma * pl * irl, status);
    const double cr = checked_sqrt(gamma * pr * irr, status);
    const double nn = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
    if (kind == 0) return fmax(fabs(vl), fabs(vr)) + fmax(cl, cr) * nn;
    return fmax(fabs(vl) + cl * nn, fabs(vr) + cr * nn);
}

// Trixi min_max_speed_naive with a normal direction
__device__ __forceinline__ void min_max_speed_normal(double gamma, const double* ul, const double* ur,
                                                     const double* nrm, double* lmin, double* lmax,
                                                     unsigned* status) {
    const double gm1 = gamma - 1.0;
    const double irl = 1.0 / ul[0], irr = 1.0 / ur[0];
    const double v1l = ul[1] * irl, v2l = ul[2] * irl, v1r = ur[1] * irr, v2r = ur[2] * irr;
    const double pl = gm1 * (ul[3] - 0.5 * (ul[1] * v1l + ul[2] * v2l));
    const double pr = gm1 * (ur[3] - 0.5 * (ur[1] * v1r + ur[2] * v2r));
    const double nn = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
    *lmin = (v1l * nrm[0] + v2l * nrm[1]) - checked_sqrt(gamma * pl * irl, status) * nn;
    *lmax = (v1r * nrm[0] + v2r * nrm[1]) + checked_sqrt(gamma * pr * irr, status) * nn;
}

// the 8-argument LW surface flux with a normal direction, arguments (f_ll, f_rr, a3, a4, a5, a6)
__device__ __forceinline__ void lw_surface_flux_normal(double gamma, int flux_kind, int speed_kind,
                                                       const double* fl, const double* fr, const double* a3,
                                                       const double* a4, const double* a5, const double* a6,
                                                       const double* nrm, double* out, unsigned* status) {
    if (flux_kind == 0) {
        const double lambda = max_abs_speed_normal(gamma, a3, a4, nrm, speed_kind, status);
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v] = 0.5 * (fl[v] + fr[v]) + (-0.5 * lambda * (a6[v] - a5[v]));
    } else {
        double lmin, lmax;
        min_max_speed_normal(gamma, a5, a6, nrm, &lmin, &lmax, status);
        if (lmin >= 0.0 && lmax >= 0.0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) out[v] = fl[v];
        } else if (lmax <= 0.0 && lmin <= 0.0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) out[v] = fr[v];
        } else {
            const double inv = 1.0 / (lmax - lmin);
            const double fll = lmax * inv, frr = lmin * inv, fd = lmin * lmax * inv;
#pragma unroll
            for (int v = 0; v < NV; ++v) out[v] = fll * fl[v] - frr * fr[v] + fd * (a4[v] - a3[v]);
        }
    }
}

// node (i, j) of face f at face index l
__device__ __forceinline__ int face_node_index(int n, int f, int l) {
    return f == 0 ? n * l : f == 1 ? (n - 1) + n * l : f == 2 ? l : l + n * (n - 1);
}

struct CurvedSurfArgs {
    const double* u;          // [v, i, j, e]
    double* out;              // du (rhs) or the updated state (step)
    const double* tU;         // [v, l, face, e]
    const double* tF;         // contravariant flux traces [v, l, face, e]
    const double* metrics;    // [4, i, j, e]
    const double* inv_jac;    // [i, j, e]
    const int* p_elem;        // interfaces of this colour
    const int* s_elem;
    const int* faces;         // p_face | s_face << 2 | reversed << 4
    int count;
    const double* dt;
    int step_mode;
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
    const double* tFv;        // Navier-Stokes: contravariant viscous flux traces (or null)
    // shock capturing (or null): blending factors [e] and the face-adjacent subcell fluxes fn_low [v, l, slot, e]
    const double* alpha;
    const double* tFn;
    double w_first, w_last;
    // UnstructuredMesh2D (or null): physical flux traces tF <- F, tG <- G, and the caller's outward normals
    // [2, l, face, e]
    const double* tG;
    const double* unorm;
};

// fn_low slot of a face: load_fn_low! fills (bottom, right, top, left) (src/solvers/dgsem_tree/dg_2d.jl:236-249)
__device__ __forceinline__ int fn_low_slot(int f) { return f == 0 ? 3 : f == 1 ? 1 : f == 2 ? 0 : 2; }

// zhang_shu_flux_fix (src/solvers/dgsem_p4est/dg_2d.jl:199-225): Fn is pulled towards the first-order fn until
// the density, then the pressure, of the subcell update uprev - c (Fn - fn_inner) is no further from the
// first-order update's than 9/10 of that value
__device__ __forceinline__ void zhang_shu_flux_fix(double gm1, const double* uprev, const double* ulow, double* Fn,
                                                   const double* fin, const double* fn, double c) {
    double uh[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uh[v] = uprev[v] - c * (Fn[v] - fin[v]);
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
#pragma unroll
            for (int v = 0; v < NV; ++v) uh[v] = uprev[v] - c * (Fn[v] - fin[v]);
        }
        const double lo = pass == 0 ? ulow[0] : gm1 * (ulow[3] - 0.5 * (ulow[1] * ulow[1] + ulow[2] * ulow[2]) / ulow[0]);
        const double hi = pass == 0 ? uh[0] : gm1 * (uh[3] - 0.5 * (uh[1] * uh[1] + uh[2] * uh[2]) / uh[0]);
        const double eps = 0.1 * lo;
        const double theta = julia_min(fabs(eps - lo) / (fabs(hi - lo) + 1e-13), 1.0);
        if (theta < 1.0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) Fn[v] = theta * Fn[v] + (1.0 - theta) * fn[v];
        }
    }
}

// get_blended_flux (src/solvers/dgsem_p4est/dg_2d.jl:227-250) at an interface node: Fn <- (1 - alp) Fn + alp fn
// with fn = flux_lax_friedrichs(u_P, u_S, n) and alp = (alpha_P + alpha_S) / 2, then the Zhang-Shu fix on each
// side whose subcell update is not admissible. As in prolong2interfaces! (:8-84), both sides' fn_inner come from
// fn_low at the primary's node index l, and J^{-1} is the primary face node's for both.
template <int N>
__device__ __forceinline__ void blend_curved_flux(const CurvedSurfArgs& a, int pe, int se, int pf, int sf, int l, int np,
                                                  const double* uP, const double* uS, const double* nrm, double* Fn) {
    constexpr int n = N + 1, nn = n * n;
    const double gm1 = a.gamma - 1.0;
    double fP[NV], gP[NV], fS[NV], gS[NV], fn[NV], fil[NV], fir[NV];
    euler_fluxes(gm1, uP[0], uP[1], uP[2], uP[3], fP, gP);
    euler_fluxes(gm1, uS[0], uS[1], uS[2], uS[3], fS, gS);
    const double lam = max_abs_speed_normal(a.gamma, uP, uS, nrm, a.speed_kind, a.status);
#pragma unroll
    for (int v = 0; v < NV; ++v)
        fn[v] = 0.5 * ((fP[v] * nrm[0] + gP[v] * nrm[1]) + (fS[v] * nrm[0] + gS[v] * nrm[1])) + (-0.5 * lam * (uS[v] - uP[v]));
    load4(a.tFn + (((size_t)pe * 4 + pf) * n + l) * NV, fil);
    load4(a.tFn + (((size_t)se * 4 + sf) * n + l) * NV, fir);
    const double alp = 0.5 * (__ldg(a.alpha + pe) + __ldg(a.alpha + se));
#pragma unroll
    for (int v = 0; v < NV; ++v) Fn[v] = (1.0 - alp) * Fn[v] + alp * fn[v];
    const double dt = *a.dt;
    const double J = __ldg(a.inv_jac + (size_t)pe * nn + np);
    double test[NV], low[NV];
    const double cl = dt * J / (a.w_last * 0.5);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        test[v] = uP[v] - cl * (Fn[v] - fil[v]);
        low[v] = uP[v] - cl * (fn[v] - fil[v]);
    }
    if (!admissible(gm1, test)) zhang_shu_flux_fix(gm1, uP, low, Fn, fil, fn, cl);
    const double cr = -dt * J / (a.w_first * 0.5);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        test[v] = uS[v] - cr * (Fn[v] - fir[v]);
        low[v] = uS[v] - cr * (fn[v] - fir[v]);
    }
    if (!admissible(gm1, test)) zhang_shu_flux_fix(gm1, uS, low, Fn, fir, fn, cr);
}

// compute_alp for Union{StructuredMesh, UnstructuredMesh2D} (src/solvers/dgsem_structured/dg_2d.jl:2169-2191) as the
// UnstructuredMesh2D interface calls it (src/solvers/dgsem_unstructured_2d/dg_2d.jl:234-268): fn = Rusanov(u_P, u_S,
// n); alp = (alpha_P + alpha_S) / 2, or 1 when the first-order subcell update of either side with the blended flux
// is not admissible, the updates starting from the time-averaged U of each side with J^{-1} of the primary face
// node; fn_low by side slot, each side at its own node index. Fn <- alp fn + (1 - alp) Fn.
template <int N>
__device__ __forceinline__ void blend_unstructured_flux(const CurvedSurfArgs& a, int pe, int se, int pf, int sf, int l,
                                                        int ls, int np, const double* uP, const double* uS,
                                                        const double* UP, const double* US, const double* nrm,
                                                        double* Fn) {
    constexpr int n = N + 1, nn = n * n;
    const double gm1 = a.gamma - 1.0;
    double fP[NV], gP[NV], fS[NV], gS[NV], fn[NV], fil[NV], fir[NV];
    euler_fluxes(gm1, uP[0], uP[1], uP[2], uP[3], fP, gP);
    euler_fluxes(gm1, uS[0], uS[1], uS[2], uS[3], fS, gS);
    const double lam = max_abs_speed_normal(a.gamma, uP, uS, nrm, a.speed_kind, a.status);
#pragma unroll
    for (int v = 0; v < NV; ++v)
        fn[v] = 0.5 * ((fP[v] * nrm[0] + gP[v] * nrm[1]) + (fS[v] * nrm[0] + gS[v] * nrm[1])) + (-0.5 * lam * (uS[v] - uP[v]));
    load4(a.tFn + (((size_t)pe * 4 + fn_low_slot(pf)) * n + l) * NV, fil);
    load4(a.tFn + (((size_t)se * 4 + fn_low_slot(sf)) * n + ls) * NV, fir);
    double alp = 0.5 * (__ldg(a.alpha + pe) + __ldg(a.alpha + se));
    const double dt = *a.dt;
    const double J = __ldg(a.inv_jac + (size_t)pe * nn + np);
    double Fb[NV], low[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) Fb[v] = (1.0 - alp) * Fn[v] + alp * fn[v];
#pragma unroll
    for (int v = 0; v < NV; ++v) low[v] = UP[v] - dt * J / (a.w_last * 0.5) * (Fb[v] - fil[v]);
    if (!admissible(gm1, low)) {
        alp = 1.0;
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) low[v] = US[v] - dt * J / (a.w_first * 0.5) * (fir[v] - Fb[v]);
        if (!admissible(gm1, low)) alp = 1.0;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) Fn[v] = alp * fn[v] + (1.0 - alp) * Fn[v];
}

// An UnstructuredMesh2D interface node (prolong2interfaces!, calc_interface_flux!, src/solvers/dgsem_unstructured_2d/
// dg_2d.jl:60-280): the normal is the caller's outward normal of the primary at its node l; both sides' normal
// fluxes are their physical time-averaged fluxes dotted with it (the secondary's node s(l) = start_index +
// (l - 1) index_increment is prolonged with the primary normal at that index, i.e. at l); the curvilinear argument
// order; Fn on the primary, -Fn on the secondary at s(l).
template <int N>
__device__ __forceinline__ void unstructured_interface_flux(const CurvedSurfArgs& a, int pe, int se, int pf, int sf,
                                                            int l, int ls, int np, const double* uP, const double* uS,
                                                            const double* UP, const double* US, double* Fn) {
    constexpr int n = N + 1;
    const size_t tp = (((size_t)pe * 4 + pf) * n + l) * NV, ts = (((size_t)se * 4 + sf) * n + ls) * NV;
    double FP[NV], GP[NV], FS[NV], GS[NV], fl[NV], fr[NV];
    load4(a.tF + tp, FP);
    load4(a.tG + tp, GP);
    load4(a.tF + ts, FS);
    load4(a.tG + ts, GS);
    const double2 nv = __ldg(reinterpret_cast<const double2*>(a.unorm) + ((size_t)pe * 4 + pf) * n + l);
    const double nrm[2] = {nv.x, nv.y};
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        fl[v] = fma(FP[v], nrm[0], GP[v] * nrm[1]);   // normal_product (src/solvers/fr.jl:146-150)
        fr[v] = fma(FS[v], nrm[0], GS[v] * nrm[1]);
    }
    lw_surface_flux_normal(a.gamma, a.flux_kind, a.speed_kind, fl, fr, uP, uS, UP, US, nrm, Fn, a.status);
    if (a.alpha) blend_unstructured_flux<N>(a, pe, se, pf, sf, l, ls, np, uP, uS, UP, US, nrm, Fn);
}

template <int N>
static __global__ void __launch_bounds__(128) curved_interface_kernel(CurvedSurfArgs a) {
    constexpr int n = N + 1;
    constexpr int nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n;
    const int l = t - k * n;
    if (k >= a.count) return;
    const int pe = __ldg(a.p_elem + k), se = __ldg(a.s_elem + k), code = __ldg(a.faces + k);
    const int pf = code & 3, sf = (code >> 2) & 3;
    const int ls = (code >> 4) & 1 ? n - 1 - l : l;
    const int np = face_node_index(n, pf, l), ns = face_node_index(n, sf, ls);
    const double sgP = (pf & 1) ? 1.0 : -1.0, sgS = (sf & 1) ? 1.0 : -1.0;
    double uP[NV], uS[NV], UP[NV], US[NV], FP[NV], FS[NV], Fn[NV], J[4];
    // (node records, traces and metrics move as one 256-bit access each)
    load4w(a.u + ((size_t)pe * nn + np) * NV, uP);
    load4w(a.u + ((size_t)se * nn + ns) * NV, uS);
    const size_t tp = (((size_t)pe * 4 + pf) * n + l) * NV, ts = (((size_t)se * 4 + sf) * n + ls) * NV;
    load4w(a.tU + tp, UP);
    load4w(a.tU + ts, US);
    if (a.tG) {
        unstructured_interface_flux<N>(a, pe, se, pf, sf, l, ls, np, uP, uS, UP, US, Fn);
    } else {
        load4w(a.tF + tp, FP);
        load4w(a.tF + ts, FS);
        load4w(a.metrics + ((size_t)pe * nn + np) * 4, J);
        const double nrm[2] = {sgP * (pf < 2 ? J[0] : J[2]), sgP * (pf < 2 ? J[1] : J[3])};
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            FP[v] *= sgP;     // F_P . n_P
            FS[v] *= -sgS;    // F_S . (-n_S)
        }
        lw_surface_flux_normal(a.gamma, a.flux_kind, a.speed_kind, FP, FS, uP, uS, UP, US, nrm, Fn, a.status);
        if (a.alpha) blend_curved_flux<N>(a, pe, se, pf, sf, l, np, uP, uS, nrm, Fn);
    }
    if (a.tFv) {
        // minus the mean of both sides' viscous normal fluxes (calc_interface_flux_hyperbolic_parabolic!,
        // src/solvers/dgsem_p4est/dg_2d_parabolic.jl:1878-1958)
        double vP[NV], vS[NV];
        load4(a.tFv + tp, vP);
        load4(a.tFv + ts, vS);
#pragma unroll
        for (int v = 0; v < NV; ++v) Fn[v] -= 0.5 * (sgP * vP[v] + (-sgS) * vS[v]);
    }
    const double dts = a.step_mode ? *a.dt : 1.0;
    const double cP = -dts * __ldg(a.inv_jac + (size_t)pe * nn + np) * ((pf & 1) ? a.inv_w_last : a.inv_w_first);
    const double cS = dts * __ldg(a.inv_jac + (size_t)se * nn + ns) * ((sf & 1) ? a.inv_w_last : a.inv_w_first);
    double* oP = a.out + ((size_t)pe * nn + np) * NV;
    double* oS = a.out + ((size_t)se * nn + ns) * NV;
    double x[NV];
    load4w_rw(oP, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(cP, Fn[v], x[v]);
    store4w(oP, x);
    load4w_rw(oS, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(cS, Fn[v], x[v]);
    store4w(oS, x);
}

// Boundary faces of a curvilinear mesh: the LW slip walls in their normal-direction form
// (src/equations/equations.jl:137-169; prolong2boundaries! / calc_boundary_flux!, src/solvers/dgsem_p4est/
// dg_2d.jl:285-393): inner normal flux with the outward normal, the mirrored exterior, the surface flux with the
// inner side as _ll in the curvilinear order; for Navier-Stokes minus the wall's viscous flux
// (calc_boundary_flux_lw!, src/solvers/dgsem_p4est/dg_2d_parabolic.jl:2057-2127). One launch per class of faces
// (xi, eta): a corner node is shared only between the classes.
struct CurvedBndArgs {
    const double* u;
    double* out;
    const double* tU;
    const double* tF;         // contravariant flux traces [v, l, face, e]
    const double* tFv;        // viscous ones (Navier-Stokes) or null
    const double* metrics;
    const double* inv_jac;    // [i, j, e]
    const int* elem;          // boundaries of this class
    const int* face;
    const int* kind;          // BC_SLIP_WALL_*
    const int* index;         // original boundary index (wall data)
    int count;
    const int* wall_kind;
    const double* wall;       // [3, l, B]
    const double* dt;
    int step_mode;
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
    // time-averaged Dirichlet: exterior states at the GLL time levels [v, q, l, B], GLL weights, the MDRK
    // stage-1 scaling
    const double* levels;
    const double* weights;
    double scaling_factor;
};

template <int N>
static __global__ void __launch_bounds__(128) curved_boundary_kernel(CurvedBndArgs a) {
    constexpr int n = N + 1;
    constexpr int nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n;
    const int l = t - k * n;
    if (k >= a.count) return;
    const int e = __ldg(a.elem + k), f = __ldg(a.face + k), kind = __ldg(a.kind + k);
    const int node = face_node_index(n, f, l);
    const double sg = (f & 1) ? 1.0 : -1.0;
    double ui[NV], Ui[NV], Fi[NV], uo[NV], Uo[NV], Fo[NV], Fn[NV], J[4];
    load4(a.u + ((size_t)e * nn + node) * NV, ui);
    const size_t tb = (((size_t)e * 4 + f) * n + l) * NV;
    load4(a.tU + tb, Ui);
    load4(a.tF + tb, Fi);
    load4(a.metrics + ((size_t)e * nn + node) * 4, J);
    const double nrm[2] = {sg * (f < 2 ? J[0] : J[2]), sg * (f < 2 ? J[1] : J[3])};
#pragma unroll
    for (int v = 0; v < NV; ++v) Fi[v] *= sg;
    if (kind == BC_DIRICHLET) {
        // (src/equations/equations.jl:64-93): GLL time averages of the exterior state and of its flux along the
        // normal; the surface flux gets U_outer in the place of the exterior u
        const int b = __ldg(a.index + k);
        const double gm1 = a.gamma - 1.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) Uo[v] = Fo[v] = 0.0;
        for (int q = 0; q < n; ++q) {
            double ub[NV], fx[NV], gy[NV];
            load4(a.levels + (((size_t)b * n + l) * n + q) * NV, ub);
            euler_fluxes(gm1, ub[0], ub[1], ub[2], ub[3], fx, gy);
            const double w = a.scaling_factor * a.weights[q] / 2.0;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Uo[v] += ub[v] * w;
                Fo[v] += (fx[v] * nrm[0] + gy[v] * nrm[1]) * w;
            }
        }
        lw_surface_flux_normal(a.gamma, a.flux_kind, a.speed_kind, Fi, Fo, ui, Uo, Ui, Uo, nrm, Fn, a.status);
    } else {
        slip_wall_exterior(kind, Fi, Ui, ui, Fo, Uo, uo);
        lw_surface_flux_normal(a.gamma, a.flux_kind, a.speed_kind, Fi, Fo, ui, uo, Ui, Uo, nrm, Fn, a.status);
    }
    if (a.tFv) {
        double fv[NV];
        load4(a.tFv + tb, fv);
#pragma unroll
        for (int v = 0; v < NV; ++v) fv[v] *= sg;
        const int b = __ldg(a.index + k);
        if (__ldg(a.wall_kind + b) == WALL_ADIABATIC) {
            const double* w = a.wall + 3 * ((size_t)b * n + l);
            fv[3] = fma(__ldg(w), fv[1], fma(__ldg(w + 1), fv[2], __ldg(w + 2)));
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) Fn[v] -= fv[v];
    }
    const double dts = a.step_mode ? *a.dt : 1.0;
    const double c = -dts * __ldg(a.inv_jac + (size_t)e * nn + node) * ((f & 1) ? a.inv_w_last : a.inv_w_first);
    double* o = a.out + ((size_t)e * nn + node) * NV;
    double x[NV];
    load4_rw(o, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(c, Fn[v], x[v]);
    store4(o, x);
}

// CFL reduction on curvilinear meshes (Trixi max_dt): per element max_nodes |Ja^1 . (l1, l2)| |J^{-1}| +
// max_nodes |Ja^2 . (l1, l2)| |J^{-1}|, l_d = |v_d| + c. A CTA takes MsCfg<N>::ELEMS elements: a coalesced pass
// over their nodes into shared memory, then one thread per element reduces its nodes.
template <int N>
static __global__ void __launch_bounds__(MS_THREADS) curved_max_speed_kernel(const double* __restrict__ u,
                                                                             const double* __restrict__ metrics,
                                                                             const double* __restrict__ inv_jac,
                                                                             int E, double gamma, StepState* s) {
    constexpr int n = N + 1;
    constexpr int nn = n * n;
    constexpr int ELEMS = MsCfg<N>::ELEMS;
    __shared__ double l1s[ELEMS * nn], l2s[ELEMS * nn];
    __shared__ double wmax[MS_THREADS / 32];
    const int e0 = blockIdx.x * ELEMS;
    const int ne = min(ELEMS, E - e0);
    const double gm1 = gamma - 1.0;
    for (int k = threadIdx.x; k < ne * nn; k += MS_THREADS) {
        const size_t node = (size_t)e0 * nn + k;
        double x[NV], J[4];
        load4w(u + node * NV, x);
        load4w(metrics + node * 4, J);
        const double ir = 1.0 / x[0];
        const double v1 = x[1] * ir, v2 = x[2] * ir;
        const double p = gm1 * (x[3] - 0.5 * (x[1] * v1 + x[2] * v2));
        const double c = checked_sqrt(gamma * p * ir, &s->status);
        const double l1 = fabs(v1) + c, l2 = fabs(v2) + c;
        const double ij = fabs(__ldg(inv_jac + node));
        l1s[k] = fabs(J[0] * l1 + J[1] * l2) * ij;
        l2s[k] = fabs(J[2] * l1 + J[3] * l2) * ij;
    }
    __syncthreads();
    double m = 0.0;
    if (threadIdx.x < ne) {
        double m1 = 0.0, m2 = 0.0;
        for (int k = 0; k < nn; ++k) {
            m1 = fmax(m1, l1s[threadIdx.x * nn + k]);
            m2 = fmax(m2, l2s[threadIdx.x * nn + k]);
        }
        m = m1 + m2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmax[0];
        for (int w = 1; w < MS_THREADS / 32; ++w) b = fmax(b, wmax[w]);
        if (b > 0.0) atomicMax(&s->max_bits, (unsigned long long)__double_as_longlong(b));
    }
}

}  // namespace tlw
