// tlw_volume.cuh -- fused per-element LW / MDRK volume kernels for TreeMesh{2} (FP64, sm_100a).
//
// Work split inside a CTA of EB whole elements (N=3: 8 x 16 nodes in 128 threads, N=4: 5 x 25 in 128,
// N=5: 7 x 36 in 256):
//  * node phase - one thread per GLL node ("owner") evaluates the Euler fluxes at the perturbed states and
//    keeps all LW stage state (u +- ut, u +- 2ut, the time averages U, F, G) in registers;
//  * line phase - each 1-D derivative contraction is done by one thread per (variable, element, line
//    index) that reads a whole row of f and a whole column of g from shared memory once, multiplies by
//    the derivative matrix held in constant memory (compile-time indices: the matrix entries are FMA
//    operands, no loads), and writes the row/column results back in place.
// Shared memory holds, per variable and element, a row-major plane of the node values with a padded
// plane stride chosen so that the owner accesses and the row/column accesses of the line phase are
// (nearly) bank-conflict free. Per stage a node writes 8 doubles and reads 8 back; a line reads and
// writes 2n. HBM traffic per element: read u once, write du (or u^{n+1}) once, write the face traces of
// U and F.n for the interface kernels.
//
// Restates, per element (TreeMesh, no source terms):
//   LW depth 4 (N>=4): lw_volume_kernel_4!  src/solvers/dgsem_tree/dg_2d.jl:918-1249
//   LW depth 3 (N=3):  lw_volume_kernel_3!  src/solvers/dgsem_tree/dg_2d.jl:674-913
//   LW depth 2 (N=2):  lw_volume_kernel_2!  src/solvers/dgsem_tree/dg_2d.jl:495-669
//   LW depth 1 (N=1):  lw_volume_kernel_1!  src/solvers/dgsem_tree/dg_2d.jl:370-490
//   MDRK stage 1/2:    mdrk_kernel_1!/2!    src/solvers/dgsem_tree/multi_derivative_2d.jl:263-421, 423-555
// then the Trixi apply_jacobian! factor -J^{-1} is folded into the written result.
#pragma once
#include "tlw_device.cuh"

namespace tlw {

// EBX = 0: the default number of elements per CTA; another value selects a tuned variant
// elements per CTA at N = 5: 3 (108 of 128 threads busy, 5 CTAs per SM) measured 4 % faster than 7 (252 of
// 256 threads, 2 CTAs per SM) and 10 % faster than 10 on the 512^2 step
#ifndef TLW_EB_N5
#define TLW_EB_N5 3
#endif
#ifndef TLW_VOLUME_MIN_BLOCKS
#define TLW_VOLUME_MIN_BLOCKS 5
#endif

template <int N, int EBX = 0>
struct VolCfg {
    static constexpr int n = N + 1;
    static constexpr int nn = n * n;
    // whole elements per CTA, chosen so that the CTA is (nearly) full warps
    static constexpr int EB = EBX ? EBX : N == 1 ? 32 : N == 2 ? 14 : N == 3 ? 8 : N == 4 ? 5 : N == 5 ? TLW_EB_N5 : N == 6 ? 5 : 2;
    static constexpr int THREADS = ((EB * nn + 31) / 32) * 32;
    // resident CTAs per SM the register allocation must allow (5 CTAs of 128 threads: <= 96 registers, measured
    // 4 % faster than 4 CTAs at 128 registers on the N = 4 workload; 6 CTAs spill)
    static constexpr int MIN_BLOCKS = THREADS <= 128 ? TLW_VOLUME_MIN_BLOCKS : 2;
    static constexpr int MDRK_MIN_BLOCKS = THREADS <= 128 ? 5 : 2;
    // curvilinear shock capturing (subcell normals, MUSCL face values): 4 CTAs of 128 threads, 128 registers
    static constexpr int SC_CURVED_MIN_BLOCKS = THREADS <= 128 ? 4 : 2;
    // plane layout: node (i, j) of (variable v, element e) at (v*EB + e)*P + i + R*j
    static constexpr int R = n;
    static constexpr int P = n == 4 ? 19 : nn;
    static constexpr int PLANES = 4 * EB * P;          // doubles of one 4-variable field
    static constexpr int LINES = 4 * n * EB;           // (variable, element, line index)
    // regions: X (f / x-results), Y (g / y-results), F0X, F0Y (fluxes at u, kept for stages 2 and 4);
    // shock capturing adds UU (u), VC (v1, v2, c), FVX, FVY (first-order subcell fluxes)
    static constexpr size_t smem_bytes(int regions) { return (size_t)regions * PLANES * sizeof(double); }
};

enum VolMode { MODE_RHS = 0, MODE_STEP = 1 };

struct VolArgs {
    const double* u;        // state the stage fluxes are evaluated at  [v,i,j,e]
    const double* u_base;   // MODE_STEP: out = u_base + dt * du        [v,i,j,e]
    double* out;            // du (MODE_RHS) or the updated state (MODE_STEP)
    double* tU;             // face traces of U   [v, l, face, e]
    double* tF;             // face traces of F.n [v, l, face, e]
    double* tG;             // UnstructuredMesh2D: physical flux traces, tF <- F and tG <- G (null otherwise)
    // source terms (TreeMesh, FR volume integral): kind (1: source_terms_convergence_test), node coordinates
    // [2, i, j, e], the time of this rhs (device scalar), MDRK stage 1's S2 = s + s_t/6 [v, i, j, e]
    int source;
    const double* xnode;
    const double* tnow;
    double* S2;
    int compact;            // MDRK step on a plain TreeMesh: u_t between the stages instead of U2, F2
    double* U2;             // MDRK: stage-1 U2 [v,i,j,e] (written by stage 1, read by stage 2)
    double* F2;             // MDRK: stage-1 F2 [v,d,i,j,e]
    const double* inv_jac;  // [e]
    const double* dt;       // device scalar
    const Basis* basis;
    int E;
    double gamma;
    // shock capturing (VolumeIntegralFRShockCapturing, first-order subcells)
    const double* alpha;    // blending factor per element
    double* tFn;            // first-order subcell flux next to each face [v, l, face, e] (fn_low)
    unsigned* status;
    int speed_kind;
    const int* inst;        // batched form: instance of each element (dt indexed by it); null otherwise
    // curvilinear meshes: contravariant vectors per node [4, i, j, e] (Ja^1_1, Ja^1_2, Ja^2_1, Ja^2_2) and the
    // inverse Jacobian per node [i, j, e] (inv_jac is then unused)
    const double* metrics;
    const double* inv_jac_node;
    unsigned long long* cfl_slots;   // plain LW step on a periodic TreeMesh: per-element CFL slots (or null)
    // temporal error estimate of the Adaptive step control (lw_volume_kernel_4!'s u_np1 / u_np1_low tail)
    double* temporal_errors;          // [e]
    double abstol, reltol;
    double* dstore;                   // [m][e][v][node]: the stage derivatives d_1..d_depth (DSTORE kernels)
    // shock capturing on curvilinear meshes: subcell-face normals [e][d][line][f - 1][2] (d 0: xi faces on row
    // j, 1: eta faces on column i; f = 1..n-1), the normals the reference's calc_fn_low! takes for face n-1 of
    // pure DG elements [e][d][line][2], elements with a boundary face [e] (MUSCL: first order there), and the
    // MUSCL geometry: subcell faces [0..n] then the extended nodes [0..n+1] of the reference element
    const double* subn;
    const double* subq;
    const unsigned char* atb;
    const double* muscl_geom;
    int reconstruction;               // 0 first order, 1 MUSCL, 2 MUSCL-Hancock
};

// curvilinear: contravariant fluxes f~ = Ja^1_1 f + Ja^1_2 g, g~ = Ja^2_1 f + Ja^2_2 g of a node
// (contravariant_flux, src/solvers/dgsem_structured/dg_2d.jl:541-556)
__device__ __forceinline__ void contravariant(const double* Ja, const double* f, const double* g, double* ft,
                                              double* gt) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        ft[v] = fma(Ja[0], f[v], Ja[1] * g[v]);
        gt[v] = fma(Ja[2], f[v], Ja[3] * g[v]);
    }
}

// owner: store the node's f (into X) and g (into Y)
template <int N, class C>
__device__ __forceinline__ void node_put(double* X, double* Y, int e, int i, int j, const double* f, const double* g) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const int a = (v * C::EB + e) * C::P + i + C::R * j;
        X[a] = f[v];
        Y[a] = g[v];
    }
}
template <int N, class C>
__device__ __forceinline__ void node_get(const double* X, const double* Y, int e, int i, int j, double* f, double* g) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const int a = (v * C::EB + e) * C::P + i + C::R * j;
        f[v] = X[a];
        g[v] = Y[a];
    }
}
// owner: x-result + y-result at the node
template <int N, class C>
__device__ __forceinline__ void node_sum(const double* X, const double* Y, int e, int i, int j, double* d) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const int a = (v * C::EB + e) * C::P + i + C::R * j;
        d[v] = X[a] + Y[a];
    }
}

// line phase, in place: X row (v,e,idx) <- M X row, Y column (v,e,idx) <- M Y column, with
// M = D (HAT = false) or Dhat (HAT = true):  x-result(i, j) = sum_k M[i,k] f(k, j),
// y-result(i, j) = sum_k M[j,k] g(i, k). Each row and column is read and written by one thread only.
// TLW_LINE_EVENODD = 1: lines of n >= 5 nodes take the even-odd form of M (c_tlw_D_eo / c_tlw_Dhat_eo), 2h^2 + 2h
// instead of n^2 multiply-adds per row (n = 5: 12 + 4 sums against 25); n <= 4 gains nothing and keeps M.
// Measured on the 512^2 steps (volume kernel, with the third-order reciprocal): N = 5 0.846 -> 0.809 ms, warped
// N = 4 0.535 -> 0.515 ms, N = 4 0.511 -> 0.509 ms; MDRK and shock capturing within 0.5 %.
#ifndef TLW_LINE_EVENODD
#define TLW_LINE_EVENODD 1
#endif
template <int N, class C, bool HAT>
__device__ __forceinline__ void line_contract(double* X, double* Y, int tid) {
    constexpr int n = C::n;
#if TLW_LINE_EVENODD
    if constexpr (n >= 5) {
        constexpr int h = n / 2;
        constexpr int hh = h * h;
        const double* E = HAT ? c_tlw_Dhat_eo[N] : c_tlw_D_eo[N];
#pragma unroll 1
        for (int t = tid; t < C::LINES; t += C::THREADS) {
            const int idx = t % n;
            const int r = t / n;
            const int e = r % C::EB;
            const int v = r / C::EB;
            const int pb = (v * C::EB + e) * C::P;
            // one line at a time (the row of X, then the column of Y) keeps the sums and differences of one
            // line live, not two
            auto line = [&](double* L, int base, int stride) {
                double a[n];
#pragma unroll
                for (int k = 0; k < n; ++k) a[k] = L[base + stride * k];
                double as[h], ad[h];
#pragma unroll
                for (int k = 0; k < h; ++k) {
                    as[k] = a[k] + a[n - 1 - k];
                    ad[k] = a[k] - a[n - 1 - k];
                }
#pragma unroll
                for (int o = 0; o < h; ++o) {
                    double xa = E[o * h] * as[0], xb = E[hh + o * h] * ad[0];
#pragma unroll
                    for (int k = 1; k < h; ++k) {
                        xa = fma(E[o * h + k], as[k], xa);
                        xb = fma(E[hh + o * h + k], ad[k], xb);
                    }
                    if constexpr (n % 2) xa = fma(E[2 * hh + o], a[h], xa);
                    L[base + stride * o] = xb + xa;
                    L[base + stride * (n - 1 - o)] = xb - xa;
                }
                if constexpr (n % 2) {
                    double xm = E[2 * hh + h] * ad[0];
#pragma unroll
                    for (int k = 1; k < h; ++k) xm = fma(E[2 * hh + h + k], ad[k], xm);
                    L[base + stride * h] = xm;
                }
            };
            line(X, pb + C::R * idx, 1);
            line(Y, pb + idx, C::R);
        }
        return;
    }
#endif
    const double* M = HAT ? c_tlw_Dhat[N] : c_tlw_D[N];
#pragma unroll 1
    for (int t = tid; t < C::LINES; t += C::THREADS) {
        const int idx = t % n;
        const int r = t / n;
        const int e = r % C::EB;
        const int v = r / C::EB;
        const int pb = (v * C::EB + e) * C::P;
        double a[n], b[n];
#pragma unroll
        for (int k = 0; k < n; ++k) {
            a[k] = X[pb + k + C::R * idx];
            b[k] = Y[pb + idx + C::R * k];
        }
#pragma unroll
        for (int o = 0; o < n; ++o) {
            double sx = 0.0, sy = 0.0;
#pragma unroll
            for (int k = 0; k < n; ++k) {
                sx = fma(M[o * n + k], a[k], sx);
                sy = fma(M[o * n + k], b[k], sy);
            }
            X[pb + o + C::R * idx] = sx;
            Y[pb + idx + C::R * o] = sy;
        }
    }
}

// ---- shock capturing helpers (src/solvers/dgsem_tree/dg_2d.jl:251-282, 1948-1991; Trixi calcflux_fv!) ----
// stage 0: park u and (v1, v2, c) of the node for the first-order subcell fluxes of its neighbours
template <int N, class C>
__device__ __forceinline__ void sc_park(double* UU, double* VC, int el, int i, int j, const double* u, double gamma,
                                        unsigned* status) {
    const double ir = 1.0 / u[0];
    const double v1 = u[1] * ir, v2 = u[2] * ir;
    const double p = (gamma - 1.0) * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    const double c = checked_sqrt(gamma * p * ir, status);
    const double vc[NV] = {v1, v2, c, 0.0};
    node_put<N, C>(UU, VC, el, i, j, u, vc);
}

// Rusanov (Trixi flux_lax_friedrichs, 4 arguments) between node L and node R of one element, from the
// parked states, fluxes (fx: x-fluxes if orientation 1, else y-fluxes) and speeds
template <int N, class C>
__device__ __forceinline__ void sc_face_flux(const double* UU, const double* VC, const double* FL, int el, int iL,
                                             int jL, int iR, int jR, int orientation, int speed_kind, double* out) {
    const int aL = el * C::P + iL + C::R * jL, aR = el * C::P + iR + C::R * jR;
    constexpr int PV = C::EB * C::P;   // stride between variable planes
    const double vL = VC[(orientation == 1 ? 0 : PV) + aL], vR = VC[(orientation == 1 ? 0 : PV) + aR];
    const double cL = VC[2 * PV + aL], cR = VC[2 * PV + aR];
    const double lambda = speed_kind == 0 ? fmax(fabs(vL), fabs(vR)) + fmax(cL, cR)
                                          : fmax(fabs(vL) + cL, fabs(vR) + cR);
#pragma unroll
    for (int v = 0; v < NV; ++v)
        out[v] = 0.5 * (FL[v * PV + aL] + FL[v * PV + aR]) + (-0.5 * lambda * (UU[v * PV + aR] - UU[v * PV + aL]));
}

// final stage: each node computes the subcell flux on its left (x) and lower (y) subcell face
template <int N, class C>
__device__ __forceinline__ void sc_faces(const double* UU, const double* VC, const double* F0X, const double* F0Y,
                                         double* FVX, double* FVY, int el, int i, int j, int speed_kind) {
    constexpr int PV = C::EB * C::P;
    const int a = el * C::P + i + C::R * j;
    double f[NV];
    if (i >= 1) {
        sc_face_flux<N, C>(UU, VC, F0X, el, i - 1, j, i, j, 1, speed_kind, f);
#pragma unroll
        for (int v = 0; v < NV; ++v) FVX[v * PV + a] = f[v];
    }
    if (j >= 1) {
        sc_face_flux<N, C>(UU, VC, F0Y, el, i, j - 1, i, j, 2, speed_kind, f);
#pragma unroll
        for (int v = 0; v < NV; ++v) FVY[v * PV + a] = f[v];
    }
}

// epilogue: fv = w_i^-1 (f*_{i+1/2} - f*_{i-1/2}) + w_j^-1 (g*_{j+1/2} - g*_{j-1/2}) (element-boundary
// subcell fluxes are zero); acc <- (1 - alpha) acc + alpha fv; fn_low traces of the four faces
template <int N, class C>
__device__ __forceinline__ void sc_blend(const VolArgs& a, const double* FVX, const double* FVY, int el, int e, int i,
                                         int j, double alpha, double* acc) {
    constexpr int n = C::n;
    constexpr int PV = C::EB * C::P;
    const int base = el * C::P;
    const double iwi = 1.0 / c_tlw_w[N][i], iwj = 1.0 / c_tlw_w[N][j];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double xr = i + 1 < n ? FVX[v * PV + base + (i + 1) + C::R * j] : 0.0;
        const double xl = i >= 1 ? FVX[v * PV + base + i + C::R * j] : 0.0;
        const double yt = j + 1 < n ? FVY[v * PV + base + i + C::R * (j + 1)] : 0.0;
        const double yb = j >= 1 ? FVY[v * PV + base + i + C::R * j] : 0.0;
        const double fv = iwi * (xr - xl) + iwj * (yt - yb);
        acc[v] = (1.0 - alpha) * acc[v] + alpha * fv;
    }
    // fn_low [v, l, face, e]: faces -x, +x use the subcell faces between nodes 0|1 and n-2|n-1 of row j
    const size_t tb = (size_t)e * 4 * n * NV;
    double f[NV];
    if (i == 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = FVX[v * PV + base + 1 + C::R * j];
        store4(a.tFn + tb + (0 * n + j) * NV, f);
    }
    if (i == n - 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = FVX[v * PV + base + (n - 1) + C::R * j];
        store4(a.tFn + tb + (1 * n + j) * NV, f);
    }
    if (j == 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = FVY[v * PV + base + i + C::R * 1];
        store4(a.tFn + tb + (2 * n + i) * NV, f);
    }
    if (j == n - 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = FVY[v * PV + base + i + C::R * (n - 1)];
        store4(a.tFn + tb + (3 * n + i) * NV, f);
    }
}

// ---- shock capturing on curvilinear meshes, the reference's P4estMesh{2} path (src/solvers/dgsem_tree/
// dg_2d.jl:236-365, src/solvers/dgsem_structured/dg_2d.jl:75-311; Trixi calcflux_fv! for curved meshes) ----
// flux_lax_friedrichs(uL, uR, nrm) from the states, their physical fluxes, normal velocities and sound speeds
__device__ __forceinline__ void sc_normal_flux(int speed_kind, const double* uL, const double* fL, const double* gL,
                                               double vnL, double cL, const double* uR, const double* fR,
                                               const double* gR, double vnR, double cR, const double* nrm,
                                               double* out) {
    const double nn = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
    const double lambda = speed_kind == 0 ? fmax(fabs(vnL), fabs(vnR)) + fmax(cL, cR) * nn
                                          : fmax(fabs(vnL) + cL * nn, fabs(vnR) + cR * nn);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double fnL = fL[v] * nrm[0] + gL[v] * nrm[1], fnR = fR[v] * nrm[0] + gR[v] * nrm[1];
        out[v] = 0.5 * (fnL + fnR) + (-0.5 * lambda * (uR[v] - uL[v]));
    }
}

// Julia sign
__device__ __forceinline__ double julia_sign(double x) { return (x == 0.0 || isnan(x)) ? x : (x > 0.0 ? 1.0 : -1.0); }

// minmod(a, b, 0) (src/solvers/dgsem_structured/dg_2d.jl:97-109): a NaN difference (0 / 0 at the element
// edges, where the extended state copies the edge node) has no sign equal to the other's and gives 0
__device__ __forceinline__ double minmod2(double a, double b) {
    const double slope = julia_min(fabs(a), fabs(b));
    const double s1 = julia_sign(a), s2 = julia_sign(b);
    if (s1 != s2) return 0.0;
    return s1 * slope;
}

// limit_variable_slope (src/equations/equations.jl:262-287), variable 0 density, 1 pressure
__device__ __forceinline__ double sc_limit_value(double gm1, int variable, const double* u) {
    return variable == 0 ? u[0] : gm1 * (u[3] - 0.5 * (u[1] * u[1] + u[2] * u[2]) / u[0]);
}
__device__ __forceinline__ void limit_variable_slope(double gm1, int variable, double* slope, double* usl, double* usr,
                                                     const double* ue, double xl, double xr) {
    const double vsl = sc_limit_value(gm1, variable, usl), vsr = sc_limit_value(gm1, variable, usr);
    const double vlow = sc_limit_value(gm1, variable, ue);
    const double threshold = 0.1 * vlow;
    if (vsl < 1e-10 || vsr < 1e-10) {
        const double rl = fabs(threshold - vlow) / (fabs(vsl - vlow) + 1e-13);
        const double rr = fabs(threshold - vlow) / (fabs(vsr - vlow) + 1e-13);
        const double theta = julia_min(julia_min(rl, rr), 1.0);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            slope[v] *= theta;
            usl[v] = ue[v] + (2.0 * theta) * (xl * slope[v]);
            usr[v] = ue[v] + (2.0 * theta) * (xr * slope[v]);
        }
    }
}

// Trixi flux(u, normal_direction, equations) of CompressibleEulerEquations2D
__device__ __forceinline__ void euler_flux_normal(double gm1, const double* u, const double* nrm, double* f) {
    const double rho = u[0], v1 = u[1] / rho, v2 = u[2] / rho;
    const double p = gm1 * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    const double vn = v1 * nrm[0] + v2 * nrm[1];
    const double rvn = rho * vn;
    f[0] = rvn;
    f[1] = rvn * v1 + p * nrm[0];
    f[2] = rvn * v2 + p * nrm[1];
    f[3] = (u[3] + p) * vn;
}

// minmod(a, b, c, beta, 0) (src/solvers/dgsem_structured/dg_2d.jl:83-95)
__device__ __forceinline__ double minmod3(double a, double b, double c, double beta) {
    const double slope = julia_min(julia_min(beta * fabs(a), fabs(b)), beta * fabs(c));
    const double s1 = julia_sign(a), s2 = julia_sign(b), s3 = julia_sign(c);
    if (s1 != s2 || s2 != s3) return 0.0;
    return s1 * slope;
}

// MUSCL (REC 1) and MUSCL-Hancock (REC 2) face values of node (i, j) into the UF regions k = 0 left, 1 right,
// 2 down, 3 up: slopes of the element-local extended state (calcflux_muscl! / calcflux_mh!,
// src/solvers/dgsem_structured/dg_2d.jl:196-253, 313-483: minmod of the one-sided differences, or with the centred
// one and beta = 2 - alpha for MUSCL-Hancock), limited for density then pressure (limit_slope,
// src/equations/compressible_euler_2d.jl:9-21). MUSCL-Hancock then adds to all four face values the multi-D
// half-step increments of the subcell, as the reference builds them: along xi +dt/2 J^{-1}(i, j) / w_{i+1}
// f(left).n_i (1 <= i <= n-2) and -dt/2 J^{-1}(i, j) / w_{i+1} f(right).n_{i+1} (i <= n-2); along eta the
// same with J^{-1}(i, j+1) (dt_fv: the time step fv_kernel! is given).
template <int N, class C, int REC>
__device__ __forceinline__ void sc_muscl_faces(const VolArgs& a, const double* UU, double* UF, int el, int e, int i,
                                               int j, double gm1, double alpha, double dt_fv, double ij) {
    constexpr int n = C::n, nn = n * n;
    constexpr int PV = C::EB * C::P;
    const double* sf = a.muscl_geom;           // subcell faces [0..n]
    const double* xe = a.muscl_geom + n + 1;   // extended nodes [0..n+1]
    auto at = [&](int ii, int jj, int v) {
        ii = ii < 0 ? 0 : (ii > n - 1 ? n - 1 : ii);
        jj = jj < 0 ? 0 : (jj > n - 1 ? n - 1 : jj);
        return UU[v * PV + el * C::P + ii + C::R * jj];
    };
    const int I = i + 1, J = j + 1;
    const double h1x = __ldg(xe + I) - __ldg(xe + I - 1), h2x = __ldg(xe + I + 1) - __ldg(xe + I);
    const double h1y = __ldg(xe + J) - __ldg(xe + J - 1), h2y = __ldg(xe + J + 1) - __ldg(xe + J);
    double u_[NV], sx[NV], sy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        u_[v] = at(i, j, v);
        const double ul = at(i - 1, j, v), ur = at(i + 1, j, v), ud = at(i, j - 1, v), uu = at(i, j + 1, v);
        if (REC == 1) {
            sx[v] = minmod2((u_[v] - ul) / h1x, (ur - u_[v]) / h2x);
            sy[v] = minmod2((u_[v] - ud) / h1y, (uu - u_[v]) / h2y);
        } else {
            // finite_differences (dg_2d.jl:75-81)
            const double beta = 2.0 - alpha;
            const double ax = -(h2x / (h1x * (h1x + h2x))), bx = (h2x - h1x) / (h1x * h2x), cx = (h1x / (h2x * (h1x + h2x)));
            const double ay = -(h2y / (h1y * (h1y + h2y))), by = (h2y - h1y) / (h1y * h2y), cy = (h1y / (h2y * (h1y + h2y)));
            sx[v] = minmod3((u_[v] - ul) / h1x, ax * ul + bx * u_[v] + cx * ur, (ur - u_[v]) / h2x, beta);
            sy[v] = minmod3((u_[v] - ud) / h1y, ay * ud + by * u_[v] + cy * uu, (uu - u_[v]) / h2y, beta);
        }
    }
    const double xl = __ldg(sf + I - 1) - __ldg(xe + I), xr = __ldg(sf + I) - __ldg(xe + I);
    const double yl = __ldg(sf + J - 1) - __ldg(xe + J), yr = __ldg(sf + J) - __ldg(xe + J);
    double fv[4][NV];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        double* s = d == 0 ? sx : sy;
        const double lo = d == 0 ? xl : yl, hi = d == 0 ? xr : yr;
        double pa[NV], pb[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            pa[v] = u_[v] + 2.0 * s[v] * lo;
            pb[v] = u_[v] + 2.0 * s[v] * hi;
        }
        limit_variable_slope(gm1, 0, s, pa, pb, u_, lo, hi);
        limit_variable_slope(gm1, 1, s, pa, pb, u_, lo, hi);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            fv[2 * d][v] = u_[v] + s[v] * lo;
            fv[2 * d + 1][v] = u_[v] + s[v] * hi;
        }
    }
    if (REC == 2) {
        // increments in the reference's order: xi "rr", xi "ll", eta "uu", eta "dd"
        double inc[4][NV];
        const double ijn = j + 1 < n ? __ldg(a.inv_jac_node + (size_t)e * nn + i + n * (j + 1)) : 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int d = q >> 1, c = d == 0 ? i : j, line = d == 0 ? j : i;
            // q 0: the cell's own face c (its left / lower value, +), q 1: face c + 1 (right / upper value, -)
            const int f = (q & 1) ? c + 1 : c;
            const bool on = (q & 1) ? c <= n - 2 : (c >= 1 && c <= n - 2);
            double r[NV] = {0.0, 0.0, 0.0, 0.0};
            if (on) {
                const double* np = a.subn + ((((size_t)e * 2 + d) * n + line) * (n - 1) + (f - 1)) * 2;
                const double nrm[2] = {__ldg(np), __ldg(np + 1)};
                double fl[NV];
                euler_flux_normal(gm1, fv[2 * d + (q & 1)], nrm, fl);
                const double jj = d == 0 ? ij : ijn;
                const double cf = ((q & 1) ? -0.5 : 0.5) * dt_fv * jj / c_tlw_w[N][c + 1];
#pragma unroll
                for (int v = 0; v < NV; ++v) r[v] = cf * fl[v];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) inc[q][v] = r[v];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int v = 0; v < NV; ++v) fv[k][v] = (((fv[k][v] + inc[0][v]) + inc[1][v]) + inc[2][v]) + inc[3][v];
    }
    const int o = el * C::P + i + C::R * j;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int v = 0; v < NV; ++v) UF[k * C::PLANES + v * PV + o] = fv[k][v];
}

// final stage on a curvilinear mesh: the subcell flux on the node's left (xi) and lower (eta) face along the
// subcell normal; pure DG elements only need faces 1 and n-1, the latter with the reference's calc_fn_low!
// normal; MUSCL elements take the reconstructed face values (their fluxes and speeds computed here)
template <int N, class C, int REC>
__device__ __forceinline__ void sc_faces_curved(const VolArgs& a, const double* UU, const double* VC, const double* F0X,
                                                const double* F0Y, const double* UF, double* FVX, double* FVY, int el,
                                                int e, int i, int j, bool blended, bool muscl) {
    constexpr int n = C::n;
    constexpr int PV = C::EB * C::P;
    const double gm1 = a.gamma - 1.0;
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        const int f = d == 0 ? i : j, line = d == 0 ? j : i;
        if (f < 1 || (!blended && f != 1 && f != n - 1)) continue;
        const double* np = (!blended && f == n - 1)
                               ? a.subq + (((size_t)e * 2 + d) * n + line) * 2
                               : a.subn + ((((size_t)e * 2 + d) * n + line) * (n - 1) + (f - 1)) * 2;
        const double nrm[2] = {__ldg(np), __ldg(np + 1)};
        const int aL = el * C::P + (d == 0 ? i - 1 : i) + C::R * (d == 0 ? j : j - 1);
        const int aR = el * C::P + i + C::R * j;
        double uL[NV], uR[NV], fL[NV], gL[NV], fR[NV], gR[NV], vnL, vnR, cL, cR, out[NV];
        if (REC >= 1 && muscl) {
            // the right (up) face value of the node before the face, the left (down) one of the node after it
            const double* PL = UF + (d == 0 ? 1 : 3) * C::PLANES;
            const double* PR = UF + (d == 0 ? 0 : 2) * C::PLANES;
#pragma unroll
            for (int v = 0; v < NV; ++v) { uL[v] = PL[v * PV + aL]; uR[v] = PR[v * PV + aR]; }
            euler_fluxes(gm1, uL[0], uL[1], uL[2], uL[3], fL, gL);
            euler_fluxes(gm1, uR[0], uR[1], uR[2], uR[3], fR, gR);
            const double irL = 1.0 / uL[0], irR = 1.0 / uR[0];
            const double v1L = uL[1] * irL, v2L = uL[2] * irL, v1R = uR[1] * irR, v2R = uR[2] * irR;
            cL = checked_sqrt(a.gamma * (gm1 * (uL[3] - 0.5 * (uL[1] * v1L + uL[2] * v2L))) * irL, a.status);
            cR = checked_sqrt(a.gamma * (gm1 * (uR[3] - 0.5 * (uR[1] * v1R + uR[2] * v2R))) * irR, a.status);
            vnL = v1L * nrm[0] + v2L * nrm[1];
            vnR = v1R * nrm[0] + v2R * nrm[1];
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                uL[v] = UU[v * PV + aL]; uR[v] = UU[v * PV + aR];
                fL[v] = F0X[v * PV + aL]; gL[v] = F0Y[v * PV + aL];
                fR[v] = F0X[v * PV + aR]; gR[v] = F0Y[v * PV + aR];
            }
            vnL = VC[aL] * nrm[0] + VC[PV + aL] * nrm[1];
            vnR = VC[aR] * nrm[0] + VC[PV + aR] * nrm[1];
            cL = VC[2 * PV + aL];
            cR = VC[2 * PV + aR];
        }
        sc_normal_flux(a.speed_kind, uL, fL, gL, vnL, cL, uR, fR, gR, vnR, cR, nrm, out);
        double* dst = d == 0 ? FVX : FVY;
#pragma unroll
        for (int v = 0; v < NV; ++v) dst[v * PV + aR] = out[v];
    }
}

// epilogue on a curvilinear mesh: acc <- (1 - alpha) acc (+ alpha fv on blended elements); fn_low of the four
// faces in load_fn_low!'s P4estMesh order (slot 0 bottom, 1 right, 2 top, 3 left)
template <int N, class C>
__device__ __forceinline__ void sc_blend_curved(const VolArgs& a, const double* FVX, const double* FVY, int el, int e,
                                                int i, int j, double alpha, bool blended, double* acc) {
    constexpr int n = C::n;
    constexpr int PV = C::EB * C::P;
    const int base = el * C::P;
    if (blended) {
        const double iwi = 1.0 / c_tlw_w[N][i], iwj = 1.0 / c_tlw_w[N][j];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double xr = i + 1 < n ? FVX[v * PV + base + (i + 1) + C::R * j] : 0.0;
            const double xl = i >= 1 ? FVX[v * PV + base + i + C::R * j] : 0.0;
            const double yt = j + 1 < n ? FVY[v * PV + base + i + C::R * (j + 1)] : 0.0;
            const double yb = j >= 1 ? FVY[v * PV + base + i + C::R * j] : 0.0;
            const double fv = iwi * (xr - xl) + iwj * (yt - yb);
            acc[v] = (1.0 - alpha) * acc[v] + alpha * fv;
        }
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = (1.0 - alpha) * acc[v];
    }
    const size_t tb = (size_t)e * 4 * n * NV;
    double f[NV];
    if (i == 1 || i == n - 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = FVX[v * PV + base + i + C::R * j];
        store4(a.tFn + tb + ((i == 1 ? 3 : 1) * n + j) * NV, f);
    }
    if (j == 1 || j == n - 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = FVY[v * PV + base + i + C::R * j];
        store4(a.tFn + tb + ((j == 1 ? 0 : 2) * n + i) * NV, f);
    }
}

// out/traces epilogue shared by all volume kernels. acc = Dhat-contraction of (F, G).
template <int n, int MODE>
__device__ __forceinline__ void volume_epilogue(const VolArgs& a, int e, int i, int j, int node, double ij, double dt,
                                                const double* acc, const double* U, const double* F,
                                                const double* G, double* o, const double* S = nullptr) {
    const size_t off = ((size_t)e * n * n + node) * NV;
    if (MODE == MODE_RHS) {
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = -ij * acc[v];
        if (S) {   // du += S (the source enters unscaled by J^{-1})
#pragma unroll
            for (int v = 0; v < NV; ++v) o[v] += S[v];
        }
    } else {
        double ub[NV];
        load4(a.u_base + off, ub);
        const double s = -dt * ij;
        if (S) {
#pragma unroll
            for (int v = 0; v < NV; ++v) ub[v] = fma(dt, S[v], ub[v]);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = fma(s, acc[v], ub[v]);
    }
    store4(a.out + off, o);
    // face traces [v, l, face, e]; face 0 = -x, 1 = +x, 2 = -y, 3 = +y
    const size_t tb = (size_t)e * 4 * n * NV;
    const bool nf = a.tG == nullptr;   // UnstructuredMesh2D: the flux traces were written before (physical)
    if (i == 0) { store4(a.tU + tb + (0 * n + j) * NV, U); if (nf) store4(a.tF + tb + (0 * n + j) * NV, F); }
    if (i == n - 1) { store4(a.tU + tb + (1 * n + j) * NV, U); if (nf) store4(a.tF + tb + (1 * n + j) * NV, F); }
    if (j == 0) { store4(a.tU + tb + (2 * n + i) * NV, U); if (nf) store4(a.tF + tb + (2 * n + i) * NV, G); }
    if (j == n - 1) { store4(a.tU + tb + (3 * n + i) * NV, U); if (nf) store4(a.tF + tb + (3 * n + i) * NV, G); }
}

// UnstructuredMesh2D: the physical time-averaged fluxes F (x) and G (y) on every face the node lies on, which its
// interfaces dot with the caller's normals (prolong2interfaces!, src/solvers/dgsem_unstructured_2d/dg_2d.jl:60-200)
template <int n>
__device__ __forceinline__ void physical_flux_traces(const VolArgs& a, int e, int i, int j, const double* F,
                                                     const double* G) {
    const size_t tb = (size_t)e * 4 * n * NV;
    if (i == 0) { store4(a.tF + tb + (0 * n + j) * NV, F); store4(a.tG + tb + (0 * n + j) * NV, G); }
    if (i == n - 1) { store4(a.tF + tb + (1 * n + j) * NV, F); store4(a.tG + tb + (1 * n + j) * NV, G); }
    if (j == 0) { store4(a.tF + tb + (2 * n + i) * NV, F); store4(a.tG + tb + (2 * n + i) * NV, G); }
    if (j == n - 1) { store4(a.tF + tb + (3 * n + i) * NV, F); store4(a.tG + tb + (3 * n + i) * NV, G); }
}

// ---- source terms (calc_source / calc_source_t_N12 ... _tttt_N4, src/solvers/dgsem_tree/dg_2d.jl:89-175) ----
// Kind 1, Trixi's source_terms_convergence_test for CompressibleEulerEquations2D: the source of the manufactured
// solution rho = rho v1 = rho v2 = c + A sin(w (x + y - t)), rho e = rho^2 (c = 2, A = 0.1, w = 2 pi / L, L = 2):
// with rho' = w A cos(w (x + y - t)) and tmp = (2 rho - 1)(gamma - 1), s = (rho', rho' (1 + tmp), rho' (1 + tmp),
// 2 rho' (rho + tmp)). It does not depend on u, so every stencil of the reference is a combination of
// s(x, t + k dt), k = -2..2, and the reference's argument-order slips in two of its calls (dg_2d.jl:891-897,
// :1227-1233: states in the wrong slots) leave the values unchanged.
struct SrcNode {
    double x1, x2, t, dt, gamma;
};
__device__ __forceinline__ void src_eval(const SrcNode& q, double k, double* s) {
    const double w = 2.0 * 3.14159265358979323846 * (1.0 / 2.0);
    const double arg = w * (q.x1 + q.x2 - (q.t + k * q.dt));
    const double si = sin(arg), co = cos(arg);
    const double rho = 2.0 + 0.1 * si;
    const double rho_x = w * 0.1 * co;
    const double tmp = (2.0 * rho - 1.0) * (q.gamma - 1.0);
    s[0] = rho_x;
    s[1] = rho_x * (1.0 + tmp);
    s[2] = s[1];
    s[3] = 2.0 * rho_x * (rho + tmp);
}
// o = c * sum_k w_k s(t + k dt), k = -2..2 (zero weights skipped)
__device__ __forceinline__ void src_term(const SrcNode& q, double w, double k, double* acc) {
    if (w == 0.0) return;
    double s[NV];
    src_eval(q, k, s);
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = fma(w, s[v], acc[v]);
}
__device__ __forceinline__ void src_stencil(const SrcNode& q, double c, double wm2, double wm1, double w0, double wp1,
                                            double wp2, double* o) {
    double acc[NV] = {0.0, 0.0, 0.0, 0.0};
    src_term(q, wm2, -2.0, acc);
    src_term(q, wm1, -1.0, acc);
    src_term(q, w0, 0.0, acc);
    src_term(q, wp1, 1.0, acc);
    src_term(q, wp2, 2.0, acc);
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = c * acc[v];
}
// the reference's stencils (each with its own time offsets)
__device__ __forceinline__ void src_t_N12(const SrcNode& q, double* o) { src_stencil(q, 0.5, 0.0, -1.0, 0.0, 1.0, 0.0, o); }
__device__ __forceinline__ void src_t_N34(const SrcNode& q, double* o) {
    src_stencil(q, 1.0 / 12.0, 1.0, -8.0, 0.0, 8.0, -1.0, o);
}
__device__ __forceinline__ void src_tt_N23(const SrcNode& q, double* o) { src_stencil(q, 1.0, 0.0, 1.0, -2.0, 1.0, 0.0, o); }
__device__ __forceinline__ void src_tt_N4(const SrcNode& q, double* o) {
    src_stencil(q, 1.0 / 12.0, -1.0, 16.0, -30.0, 16.0, -1.0, o);
}
__device__ __forceinline__ void src_ttt_N34(const SrcNode& q, double* o) {
    src_stencil(q, 0.5, -1.0, 2.0, 0.0, -2.0, 1.0, o);
}
__device__ __forceinline__ void src_tttt_N4(const SrcNode& q, double* o) {
    src_stencil(q, 1.0, 1.0, -4.0, 6.0, -4.0, 1.0, o);
}

// The per-element CFL slots of a step's final values (plain TreeMesh step): after the epilogue, every thread has
// the speeds of its node in l1, l2 (interior nodes; zero otherwise); through the (now free) X plane, one thread per
// (element, component) writes slot 0 (interior maxima) and clears the face slots, which the surfaces fill.
// Every thread of the CTA calls it (barriers inside).
template <int N, class C>
__device__ __forceinline__ void write_interior_slots(const VolArgs& a, double* X, bool active, int el, int i, int j,
                                                     int tid, double l1, double l2) {
    constexpr int n = C::n, EB = C::EB;
    __syncthreads();
    if (active) {
        X[el * C::P + i + C::R * j] = l1;
        X[(EB + el) * C::P + i + C::R * j] = l2;
    }
    __syncthreads();
    const int ee = blockIdx.x * EB + (tid >> 1);
    if (tid < 2 * EB && ee < a.E) {
        const double* p = X + ((tid & 1) * EB + (tid >> 1)) * C::P;
        double m = 0.0;
#pragma unroll
        for (int jj = 1; jj < n - 1; ++jj)
#pragma unroll
            for (int ii = 1; ii < n - 1; ++ii) m = fmax(m, p[ii + C::R * jj]);
        unsigned long long* sl = a.cfl_slots + (size_t)ee * CFL_SLOTS;
        sl[tid & 1] = (unsigned long long)__double_as_longlong(m);
#pragma unroll
        for (int k = 1; k < CFL_SLOTS / 2; ++k) sl[2 * k + (tid & 1)] = 0ull;
    }
}

// The stage's four flux pairs at upp, up, um, umm. With TLW_VOL_ILP the four reciprocals 1/rho are refined
// first, as four independent Newton chains, instead of one chain per flux pair; same operations, same bits.
#ifndef TLW_VOL_ILP
#define TLW_VOL_ILP 1
#endif

struct Recip4 {
    double pp, p, m, mm;
};
__device__ __forceinline__ Recip4 recip4(const double* upp, const double* up, const double* um, const double* umm) {
    Recip4 r;
    r.pp = nr_reciprocal(upp[0]);
    r.p = nr_reciprocal(up[0]);
    r.m = nr_reciprocal(um[0]);
    r.mm = nr_reciprocal(umm[0]);
    return r;
}

// ------------------------------------------------------------------------------------------------
// Plain LW volume kernel (depth = min(N, 4)).
// The finite-difference stencils are accumulated unscaled ("raw"); their constant factors and -dt J^{-1}
// are applied to the contraction result (s below) and folded into the F/G update coefficients:
//   depth 4: f_t = raw1/12, f_tt = raw2/12, f_ttt = raw3/2, f_tttt = raw4/2
//   depth 3: f_t = raw1/12, f_tt = raw2,    f_ttt = raw3/2
//   depth 2: f_t = raw1/2,  f_tt = raw2;    depth 1: f_t = raw1/2
// ------------------------------------------------------------------------------------------------
// DSTORE: also write each stage derivative d_m (dt-scaled time derivative of u) to a.dstore, for the discrete
// adjoint's reverse sweep, which then reads them instead of recomputing them. Layout [m][e][v][node]: one
// element's d_m is contiguous (a bulk copy per tile of elements) with the nodes innermost (conflict-free
// shared-memory reads, one thread per node).
template <int nn>
__device__ __forceinline__ void store_stage_derivative(const VolArgs& a, int m, long long e, int node, const double* d) {
    double* p = a.dstore + ((size_t)(m - 1) * a.E + e) * NV * nn + node;
#pragma unroll
    for (int v = 0; v < NV; ++v) p[v * nn] = d[v];
}

// REC (curvilinear shock capturing): 0 first-order subcells, 1 MUSCL subcells
// SRC: source terms (a.source, FR volume integral): S = s + s_t/2 + s_tt/6 + ... with each stencil added to its time
// derivative (dt s_k) before the perturbed states move, and S enters the update unscaled by J^{-1}. The curvilinear
// kernel of depth 4 takes the 5-point s_tt (calc_source_tt_N4, dgsem_structured/dg_2d.jl:1886) where the TreeMesh
// one takes the 3-point calc_source_tt_N23 (dgsem_tree/dg_2d.jl:1093-1104).
template <int N, int MODE, bool SC, int EBX = 0, bool CURVED = false, bool TE = false, bool DSTORE = false, int REC = 0,
          bool SRC = false>
static __global__ void __launch_bounds__(VolCfg<N, EBX>::THREADS, (SC && CURVED) ? VolCfg<N, EBX>::SC_CURVED_MIN_BLOCKS
                                                                  : SRC ? VolCfg<N, EBX>::MDRK_MIN_BLOCKS - 1
                                                                        : VolCfg<N, EBX>::MIN_BLOCKS)
    lw_volume_kernel(VolArgs a) {
    static_assert(REC == 0 || (SC && CURVED), "MUSCL subcells: curvilinear shock capturing");
    static_assert(!SRC || (!SC && !TE && !DSTORE), "source terms: the FR volume integral, without the error estimate");
    // the temporal error estimate of the Adaptive step control: the TreeMesh computes it at depth 4 only
    // (lw_volume_kernel_3! of dgsem_tree has none), the curvilinear kernels at depths 3 and 4
    static_assert(!TE || (CURVED ? N >= 3 : N >= 4), "temporal errors: TreeMesh N >= 4, curvilinear N >= 3");
    static_assert(!DSTORE || (!SC && !CURVED && !TE), "stored stage derivatives: the plain TreeMesh kernel");
    using C = VolCfg<N, EBX>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB;
    constexpr int DEPTH = N >= 4 ? 4 : N;
    constexpr double C1 = DEPTH >= 3 ? 1.0 / 12.0 : 0.5;
    constexpr double C2 = DEPTH == 4 ? 1.0 / 12.0 : 1.0;
    constexpr double C3 = 0.5;
    constexpr double C4 = 0.5;
    extern __shared__ double smem_d[];
    double* X = smem_d;
    double* Y = X + C::PLANES;
    double* F0X = Y + C::PLANES;
    double* F0Y = F0X + C::PLANES;
    double* UU = F0Y + C::PLANES;      // shock capturing only
    double* VC = UU + C::PLANES;
    double* FVX = VC + C::PLANES;
    double* FVY = FVX + C::PLANES;
    double* UF = FVY + C::PLANES;      // curvilinear MUSCL: face values, 4 regions (left, right, down, up)

    const int tid = threadIdx.x;
    const double gm1 = a.gamma - 1.0;
    const int el = tid / nn;
    const int node = tid - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    // curvilinear shock capturing: pure_and_blended_element_ids! (DG only where alpha is within 1e-12 of 0);
    // MUSCL subcells on blended elements without a boundary face
    double alpha_e = 0.0;
    bool blended = false, muscl = false;
    if (SC && CURVED && active) {
        alpha_e = __ldg(a.alpha + e);
        blended = !(fabs(alpha_e) <= 1e-12);
        muscl = REC >= 1 && blended && !__ldg(a.atb + e);
    }
    // dt of this element's instance (batched form) or the single dt
    const double dt = a.inst ? a.dt[__ldg(a.inst + min(e, a.E - 1))] : *a.dt;
    // per-element maxima of the interior nodes' speeds for the next step's CFL (plain LW step only)
    constexpr bool SLOTS = MODE == MODE_STEP && !SC && !CURVED;

    double U[NV], F[NV], G[NV], up[NV], um[NV], upp[NV], umm[NV];
    double Ssrc[NV] = {0.0, 0.0, 0.0, 0.0};   // SRC: the source's time average S
    SrcNode sq{};
    double s0 = 0.0, ij = 0.0;   // s0 = -dt J^{-1} (of the element, or of the node on curvilinear meshes)
    double Ja[4] = {0.0, 0.0, 0.0, 0.0};
    double dF[NV], dG[NV], u0[NV];   // TE: the last stage's term of F, G, and u
    // stage fluxes into the contraction planes (contravariant on curvilinear meshes)
    auto put = [&](const double* f, const double* g) {
        if (CURVED) {
            double ft[NV], gt[NV];
            contravariant(Ja, f, g, ft, gt);
            node_put<N, C>(X, Y, el, i, j, ft, gt);
        } else {
            node_put<N, C>(X, Y, el, i, j, f, g);
        }
    };
    // a flux pair at a perturbed state, from its precomputed 1/rho (TLW_VOL_ILP) or its own reciprocal
    auto flux = [&](const double* st, double irr, double* f, double* g) {
        if (TLW_VOL_ILP) euler_fluxes_ir(gm1, irr, st[1], st[2], st[3], f, g);
        else euler_fluxes(gm1, st[0], st[1], st[2], st[3], f, g);
    };
    // stage 0: f, g at u (dg_2d.jl:941-971; dgsem_structured/dg_2d.jl:1709-1740)
    if (active) {
        double uu[NV], f[NV], g[NV];
        load4(a.u + ((size_t)e * nn + node) * NV, uu);
        if (TE) {
#pragma unroll
            for (int v = 0; v < NV; ++v) u0[v] = uu[v];
        }
        if (CURVED) {
            load4(a.metrics + ((size_t)e * nn + node) * 4, Ja);
            ij = __ldg(a.inv_jac_node + (size_t)e * nn + node);
        } else {
            ij = __ldg(a.inv_jac + e);
        }
        s0 = -dt * ij;
        if (SRC) {
            // S = s(u, x, t) (dg_2d.jl:979-987)
            const double* xn = a.xnode + 2 * ((size_t)e * nn + node);
            sq = SrcNode{__ldg(xn), __ldg(xn + 1), *a.tnow, dt, a.gamma};
            src_eval(sq, 0.0, Ssrc);
        }
        euler_fluxes(gm1, uu[0], uu[1], uu[2], uu[3], f, g);
        put(f, g);
        if (DEPTH >= 2 || SC) node_put<N, C>(F0X, F0Y, el, i, j, f, g);
        if (SC) sc_park<N, C>(UU, VC, el, i, j, uu, a.gamma, a.status);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            F[v] = f[v]; G[v] = g[v]; U[v] = uu[v];
            up[v] = um[v] = upp[v] = umm[v] = uu[v];
        }
    }
    __syncthreads();
    line_contract<N, C, false>(X, Y, tid);
    __syncthreads();
    if (SC && CURVED && REC >= 1 && muscl) sc_muscl_faces<N, C, REC>(a, UU, UF, el, e, i, j, gm1, alpha_e, dt, ij);

    // stage 1: ut; perturbed states; f_t (dg_2d.jl:972-1023 / :725-775 / :543-582 / :417-454)
    if (active) {
        double d[NV], r[NV], q[NV], f[NV], g[NV];
        node_sum<N, C>(X, Y, el, i, j, d);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            d[v] *= s0;
            if (SRC) d[v] = fma(dt, Ssrc[v], d[v]);   // ut += dt s
            U[v] = fma(0.5, d[v], U[v]);
            up[v] += d[v];
            um[v] -= d[v];
            if (DEPTH >= 3) { upp[v] = fma(2.0, d[v], upp[v]); umm[v] = fma(-2.0, d[v], umm[v]); }
        }
        if (DSTORE) store_stage_derivative<nn>(a, 1, e, node, d);
        if (DEPTH >= 3) {
            // raw1 = -f(u+2ut) + 8 f(u+ut) - 8 f(u-ut) + f(u-2ut)
            const Recip4 rc = TLW_VOL_ILP ? recip4(upp, up, um, umm) : Recip4{0.0, 0.0, 0.0, 0.0};
            flux(upp, rc.pp, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = -f[v]; q[v] = -g[v]; }
            flux(up, rc.p, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(8.0, f[v], r[v]); q[v] = fma(8.0, g[v], q[v]); }
            flux(um, rc.m, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-8.0, f[v], r[v]); q[v] = fma(-8.0, g[v], q[v]); }
            flux(umm, rc.mm, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] += f[v]; q[v] += g[v]; }
        } else {
            // raw1 = f(u+ut) - f(u-ut)
            euler_fluxes(gm1, up[0], up[1], up[2], up[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = f[v]; q[v] = g[v]; }
            euler_fluxes(gm1, um[0], um[1], um[2], um[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] -= f[v]; q[v] -= g[v]; }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) { F[v] = fma(0.5 * C1, r[v], F[v]); G[v] = fma(0.5 * C1, q[v], G[v]); }
        if (DEPTH >= 2) put(r, q);
    }
    if (DEPTH >= 2) {
        __syncthreads();
        line_contract<N, C, false>(X, Y, tid);
        __syncthreads();
        // stage 2: utt; f_tt (dg_2d.jl:1025-1083 / :777-831 / :597-634)
        if (active) {
            double d[NV], f0[NV], g0[NV], r[NV], q[NV], f[NV], g[NV];
            node_sum<N, C>(X, Y, el, i, j, d);
            node_get<N, C>(F0X, F0Y, el, i, j, f0, g0);
            const double s = s0 * C1;
            double sk[NV];
            if (SRC) {   // s_t from the states after ut: N34 at depths 3, 4, N12 at depth 2 (dg_2d.jl:1027-1040)
                if (DEPTH >= 3) src_t_N34(sq, sk);
                else src_t_N12(sq, sk);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                d[v] *= s;
                if (SRC) {
                    Ssrc[v] = fma(0.5, sk[v], Ssrc[v]);
                    d[v] = fma(dt, sk[v], d[v]);
                }
                U[v] = fma(1.0 / 6.0, d[v], U[v]);
                up[v] = fma(0.5, d[v], up[v]);
                um[v] = fma(0.5, d[v], um[v]);
                if (DEPTH >= 3) { upp[v] = fma(2.0, d[v], upp[v]); umm[v] = fma(2.0, d[v], umm[v]); }
            }
            if (DSTORE) store_stage_derivative<nn>(a, 2, e, node, d);
            if (DEPTH == 4) {
                // raw2 = -f(upp) + 16 f(up) - 30 f0 + 16 f(um) - f(umm)
                const Recip4 rc = TLW_VOL_ILP ? recip4(upp, up, um, umm) : Recip4{0.0, 0.0, 0.0, 0.0};
                flux(upp, rc.pp, f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    r[v] = fma(-30.0, f0[v], -f[v]);
                    q[v] = fma(-30.0, g0[v], -g[v]);
                }
                flux(up, rc.p, f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] = fma(16.0, f[v], r[v]); q[v] = fma(16.0, g[v], q[v]); }
                flux(um, rc.m, f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] = fma(16.0, f[v], r[v]); q[v] = fma(16.0, g[v], q[v]); }
                flux(umm, rc.mm, f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] -= f[v]; q[v] -= g[v]; }
            } else {
                // raw2 = f(up) - 2 f0 + f(um)
                euler_fluxes(gm1, up[0], up[1], up[2], up[3], f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] = fma(-2.0, f0[v], f[v]); q[v] = fma(-2.0, g0[v], g[v]); }
                euler_fluxes(gm1, um[0], um[1], um[2], um[3], f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] += f[v]; q[v] += g[v]; }
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                F[v] = fma(C2 / 6.0, r[v], F[v]);
                G[v] = fma(C2 / 6.0, q[v], G[v]);
            }
            if (DEPTH >= 3) put(r, q);
        }
    }
    if (DEPTH >= 3) {
        __syncthreads();
        line_contract<N, C, false>(X, Y, tid);
        __syncthreads();
        // stage 3: uttt; f_ttt (dg_2d.jl:1085-1138 / :833-875)
        if (active) {
            double d[NV], r[NV], q[NV], f[NV], g[NV];
            node_sum<N, C>(X, Y, el, i, j, d);
            const double s = s0 * C2;
            double sk[NV];
            if (SRC) {   // s_tt: N23 at depths 3 and 4 on the TreeMesh (dg_2d.jl:1093-1104), N4 on curvilinear depth 4
                if (CURVED && DEPTH == 4) src_tt_N4(sq, sk);
                else src_tt_N23(sq, sk);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                d[v] *= s;
                if (SRC) {
                    Ssrc[v] = fma(1.0 / 6.0, sk[v], Ssrc[v]);
                    d[v] = fma(dt, sk[v], d[v]);
                }
                U[v] = fma(1.0 / 24.0, d[v], U[v]);
                um[v] = fma(-1.0 / 6.0, d[v], um[v]);
                up[v] = fma(1.0 / 6.0, d[v], up[v]);
                umm[v] = fma(-4.0 / 3.0, d[v], umm[v]);
                upp[v] = fma(4.0 / 3.0, d[v], upp[v]);
            }
            if (DSTORE) store_stage_derivative<nn>(a, 3, e, node, d);
            // raw3 = f(upp) - 2 f(up) + 2 f(um) - f(umm)
            const Recip4 rc = TLW_VOL_ILP ? recip4(upp, up, um, umm) : Recip4{0.0, 0.0, 0.0, 0.0};
            flux(upp, rc.pp, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = f[v]; q[v] = g[v]; }
            flux(up, rc.p, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-2.0, f[v], r[v]); q[v] = fma(-2.0, g[v], q[v]); }
            flux(um, rc.m, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(2.0, f[v], r[v]); q[v] = fma(2.0, g[v], q[v]); }
            flux(umm, rc.mm, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                r[v] -= f[v];
                q[v] -= g[v];
                F[v] = fma(C3 / 24.0, r[v], F[v]);
                G[v] = fma(C3 / 24.0, q[v], G[v]);
                if (TE && DEPTH == 3) { dF[v] = (C3 / 24.0) * r[v]; dG[v] = (C3 / 24.0) * q[v]; }
            }
            if (DEPTH >= 4) put(r, q);
        }
    }
    if (DEPTH >= 4) {
        __syncthreads();
        line_contract<N, C, false>(X, Y, tid);
        __syncthreads();
        // stage 4: utttt; f_tttt (dg_2d.jl:1140-1206)
        if (active) {
            double d[NV], f0[NV], g0[NV], r[NV], q[NV], f[NV], g[NV];
            node_sum<N, C>(X, Y, el, i, j, d);
            node_get<N, C>(F0X, F0Y, el, i, j, f0, g0);
            const double s = s0 * C3;
            double sk[NV];
            if (SRC) src_ttt_N34(sq, sk);   // s_ttt (dg_2d.jl:1148-1162)
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                d[v] *= s;
                if (SRC) {
                    Ssrc[v] = fma(1.0 / 24.0, sk[v], Ssrc[v]);
                    d[v] = fma(dt, sk[v], d[v]);
                }
                U[v] = fma(1.0 / 120.0, d[v], U[v]);
                um[v] = fma(1.0 / 24.0, d[v], um[v]);
                up[v] = fma(1.0 / 24.0, d[v], up[v]);
                umm[v] = fma(2.0 / 3.0, d[v], umm[v]);
                upp[v] = fma(2.0 / 3.0, d[v], upp[v]);
            }
            if (DSTORE) store_stage_derivative<nn>(a, 4, e, node, d);
            // raw4 = f(upp) - 4 f(up) + 6 f0 - 4 f(um) + f(umm)
            const Recip4 rc = TLW_VOL_ILP ? recip4(upp, up, um, umm) : Recip4{0.0, 0.0, 0.0, 0.0};
            flux(upp, rc.pp, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(6.0, f0[v], f[v]); q[v] = fma(6.0, g0[v], g[v]); }
            flux(up, rc.p, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-4.0, f[v], r[v]); q[v] = fma(-4.0, g[v], q[v]); }
            flux(um, rc.m, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-4.0, f[v], r[v]); q[v] = fma(-4.0, g[v], q[v]); }
            flux(umm, rc.mm, f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                r[v] += f[v];
                q[v] += g[v];
                F[v] = fma(C4 / 120.0, r[v], F[v]);
                if (TE) { dF[v] = (C4 / 120.0) * r[v]; dG[v] = (C4 / 120.0) * q[v]; }
                G[v] = fma(C4 / 120.0, q[v], G[v]);
            }
        }
    }
    // final: Dhat contraction of the time-averaged fluxes (every owner has read its node's results of
    // the last contraction before writing F, G over them: same address, same thread)
    if (SRC && active) {
        // the last stencil: depth 1 s_t / 2 (N12), 2 s_tt / 6 (N23), 3 s_ttt / 24, 4 s_tttt / 120
        // (dg_2d.jl:474-477, :651-654, :891-897, :1227-1233)
        double sk[NV];
        if (DEPTH == 1) src_t_N12(sq, sk);
        else if (DEPTH == 2) src_tt_N23(sq, sk);
        else if (DEPTH == 3) src_ttt_N34(sq, sk);
        else src_tttt_N4(sq, sk);
        const double c = DEPTH == 1 ? 0.5 : DEPTH == 2 ? 1.0 / 6.0 : DEPTH == 3 ? 1.0 / 24.0 : 1.0 / 120.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) Ssrc[v] = fma(c, sk[v], Ssrc[v]);
    }
    if (active) {
        if (CURVED) {
            if (a.tG) physical_flux_traces<n>(a, e, i, j, F, G);
            // the surface needs the normal fluxes: keep the contravariant time averages F~, G~ (their face
            // values are F . Ja^1 and F . Ja^2)
            double ft[NV], gt[NV];
            contravariant(Ja, F, G, ft, gt);
#pragma unroll
            for (int v = 0; v < NV; ++v) { F[v] = ft[v]; G[v] = gt[v]; }
            if (TE) {   // the last stage's term of F~, G~
                contravariant(Ja, dF, dG, ft, gt);
#pragma unroll
                for (int v = 0; v < NV; ++v) { dF[v] = ft[v]; dG[v] = gt[v]; }
            }
        }
        node_put<N, C>(X, Y, el, i, j, F, G);
        if (SC) {
            if constexpr (CURVED) sc_faces_curved<N, C, REC>(a, UU, VC, F0X, F0Y, UF, FVX, FVY, el, e, i, j, blended, muscl);
            else sc_faces<N, C>(UU, VC, F0X, F0Y, FVX, FVY, el, i, j, a.speed_kind);
        }
    }
    __syncthreads();
    line_contract<N, C, true>(X, Y, tid);
    __syncthreads();
    double l1 = 0.0, l2 = 0.0;
    if (active) {
        double acc[NV], o[NV];
        node_sum<N, C>(X, Y, el, i, j, acc);
        if (SC) {
            if constexpr (CURVED) sc_blend_curved<N, C>(a, FVX, FVY, el, e, i, j, alpha_e, blended, acc);
            else sc_blend<N, C>(a, FVX, FVY, el, e, i, j, __ldg(a.alpha + e), acc);
        }
        volume_epilogue<n, MODE>(a, e, i, j, node, ij, dt, acc, U, F, G, o, SRC ? Ssrc : nullptr);
        if (SLOTS && a.cfl_slots && i > 0 && i < n - 1 && j > 0 && j < n - 1) node_speeds(a.gamma, o, a.status, l1, l2);
    }
    if (SLOTS && a.cfl_slots) write_interior_slots<N, C>(a, X, active, el, i, j, tid, l1, l2);
    if (TE) {
        // lw_volume_kernel_4!'s error estimate (dg_2d.jl:1183-1265; curvilinear, with F~, G~ and the node's
        // J^{-1}: dgsem_structured/dg_2d.jl:1595-1682 at depth 3, :1983-2075 at depth 4): the strong-form volume
        // updates u_np1 = u - dt J^{-1} (D F + D G) and u_np1_low with F, G before the last stage's term;
        // temporal_errors[e] = sum over nodes and variables of ((u_np1 - u_np1_low) / (abstol + reltol max))^2
        double un[NV], err = 0.0;
        __syncthreads();
        if (active) node_put<N, C>(X, Y, el, i, j, F, G);
        __syncthreads();
        line_contract<N, C, false>(X, Y, tid);
        __syncthreads();
        if (active) {
            double dd[NV];
            node_sum<N, C>(X, Y, el, i, j, dd);
#pragma unroll
            for (int v = 0; v < NV; ++v) un[v] = fma(s0, dd[v], u0[v]);
        }
        __syncthreads();
        if (active) node_put<N, C>(X, Y, el, i, j, dF, dG);
        __syncthreads();
        line_contract<N, C, false>(X, Y, tid);
        __syncthreads();
        if (active) {
            double dd[NV];
            node_sum<N, C>(X, Y, el, i, j, dd);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const double lo = un[v] - s0 * dd[v];
                const double r = (un[v] - lo) / (a.abstol + a.reltol * fmax(fabs(un[v]), fabs(lo)));
                err = fma(r, r, err);
            }
        }
        __syncthreads();
        if (active) X[el * C::P + i + C::R * j] = err;
        __syncthreads();
        const int ee = blockIdx.x * EB + tid;
        if (tid < EB && ee < a.E) {
            double sum = 0.0;
            for (int jj = 0; jj < n; ++jj)
                for (int ii = 0; ii < n; ++ii) sum += X[tid * C::P + ii + C::R * jj];
            a.temporal_errors[ee] = sum;
        }
    }
}

// MDRK stage 1's stored sums from u^n and d = u_t: F2 = f + f_t/6, G2 = g + g_t/6, U2 = u + u_t/6 with f_t the
// 4-point stencil at u +- d, u +- 2d (multi_derivative_2d.jl:337-371), the operations of mdrk1_volume_kernel
__device__ __forceinline__ void mdrk_stage1_sums(double gm1, const double* uu, const double* d, double* F2v,
                                                 double* G2v, double* U2v) {
    double f0[NV], g0[NV], f[NV], g[NV], ft[NV], gt[NV], s[NV];
    euler_fluxes(gm1, uu[0], uu[1], uu[2], uu[3], f0, g0);
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = fma(2.0, d[v], uu[v]);
    euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
    for (int v = 0; v < NV; ++v) { ft[v] = -f[v]; gt[v] = -g[v]; s[v] = uu[v] + d[v]; }
    euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
    for (int v = 0; v < NV; ++v) { ft[v] = fma(8.0, f[v], ft[v]); gt[v] = fma(8.0, g[v], gt[v]); s[v] = uu[v] - d[v]; }
    euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
    for (int v = 0; v < NV; ++v) { ft[v] = fma(-8.0, f[v], ft[v]); gt[v] = fma(-8.0, g[v], gt[v]); s[v] = fma(-2.0, d[v], uu[v]); }
    euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        ft[v] = (ft[v] + f[v]) * (1.0 / 12.0);
        gt[v] = (gt[v] + g[v]) * (1.0 / 12.0);
        F2v[v] = fma(1.0 / 6.0, ft[v], f0[v]);
        G2v[v] = fma(1.0 / 6.0, gt[v], g0[v]);
        U2v[v] = fma(1.0 / 6.0, d[v], uu[v]);
    }
}

// ------------------------------------------------------------------------------------------------
// MDRK stage 1 (mdrk_kernel_1!, multi_derivative_2d.jl:263-421): F = f/2 + f_t/8, U = u/2 + u_t/8,
// F2 = f + f_t/6, U2 = u + u_t/6 (stored whole for stage 2).
// ------------------------------------------------------------------------------------------------
// CURVED (mdrk_kernel_1!, src/solvers/dgsem_structured/multi_derivative_2d.jl:82-243): the contractions take the
// contravariant fluxes, d carries the node's J^{-1}; F2, G2 stay physical, the traces are contravariant.
// SRC (FR volume integral): ut += dt s(u, t); S = s/2 + s_t/8 enters du, S2 = s + s_t/6 is stored for stage 2
// (multi_derivative_2d.jl:321-400; dgsem_structured/multi_derivative_2d.jl:151-239).
// COMPACT (the plain TreeMesh step): store only u_t (into a.U2) instead of U2 and F2; stage 2 recomputes them from
// u^n and u_t with this kernel's operations (64 instead of 192 bytes a node between the stages).
template <int N, int MODE, bool SC, bool CURVED = false, int REC = 0, bool SRC = false, bool COMPACT = false>
static __global__ void __launch_bounds__(VolCfg<N>::THREADS, (SC && CURVED) ? VolCfg<N>::SC_CURVED_MIN_BLOCKS
                                                                         : VolCfg<N>::MDRK_MIN_BLOCKS)
    mdrk1_volume_kernel(VolArgs a) {
    static_assert(REC == 0 || (SC && CURVED), "MUSCL subcells: curvilinear shock capturing");
    static_assert(!SRC || !SC, "source terms: the FR volume integral");
    static_assert(!COMPACT || (!SC && !CURVED && !SRC && MODE == MODE_STEP), "compact stages: the plain TreeMesh step");
    using C = VolCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB;
    extern __shared__ double smem_d[];
    double* X = smem_d;
    double* Y = X + C::PLANES;
    double* F0X = Y + C::PLANES;       // shock capturing only: fluxes, u, speeds at u^n, subcell fluxes
    double* F0Y = F0X + C::PLANES;
    double* UU = F0Y + C::PLANES;
    double* VC = UU + C::PLANES;
    double* FVX = VC + C::PLANES;
    double* FVY = FVX + C::PLANES;
    double* UF = FVY + C::PLANES;      // curvilinear MUSCL: face values, 4 regions (left, right, down, up)
    const int tid = threadIdx.x;
    const double gm1 = a.gamma - 1.0;
    const int el = tid / nn;
    const int node = tid - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    double alpha_e = 0.0;
    bool blended = false, muscl = false;
    if (SC && CURVED && active) {
        alpha_e = __ldg(a.alpha + e);
        blended = !(fabs(alpha_e) <= 1e-12);
        muscl = REC >= 1 && blended && !__ldg(a.atb + e);
    }
    // dt of this element's instance (batched form) or the single dt
    const double dt = a.inst ? a.dt[__ldg(a.inst + min(e, a.E - 1))] : *a.dt;
    double uu[NV], f0[NV], g0[NV], ij = 0.0, Ja[4] = {0.0, 0.0, 0.0, 0.0};
    // a flux pair into the contraction planes (contravariant on curvilinear meshes)
    auto put = [&](const double* f, const double* g) {
        if (CURVED) {
            double ft[NV], gt[NV];
            contravariant(Ja, f, g, ft, gt);
            node_put<N, C>(X, Y, el, i, j, ft, gt);
        } else {
            node_put<N, C>(X, Y, el, i, j, f, g);
        }
    };
    if (active) {
        load4(a.u + ((size_t)e * nn + node) * NV, uu);
        if (CURVED) {
            load4(a.metrics + ((size_t)e * nn + node) * 4, Ja);
            ij = __ldg(a.inv_jac_node + (size_t)e * nn + node);
        } else {
            ij = __ldg(a.inv_jac + e);
        }
        euler_fluxes(gm1, uu[0], uu[1], uu[2], uu[3], f0, g0);
        put(f0, g0);
        if (SC) {
            // the subcell FV part uses the instantaneous u^n (multi_derivative_2d.jl:205)
            node_put<N, C>(F0X, F0Y, el, i, j, f0, g0);
            sc_park<N, C>(UU, VC, el, i, j, uu, a.gamma, a.status);
        }
    }
    __syncthreads();
    // (the MUSCL face values are read by the neighbours after the next barrier)
    if (SC && CURVED && REC >= 1 && muscl) sc_muscl_faces<N, C, REC>(a, UU, UF, el, e, i, j, gm1, alpha_e, 0.5 * dt, ij);
    line_contract<N, C, false>(X, Y, tid);
    __syncthreads();
    double U[NV], F[NV], G[NV], Ssrc[NV] = {0.0, 0.0, 0.0, 0.0};
    if (active) {
        double d[NV], ft[NV], gt[NV], f[NV], g[NV], s[NV];
        node_sum<N, C>(X, Y, el, i, j, d);
        const double s0 = -dt * ij;
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v] *= s0;
        SrcNode sq{};
        double sn[NV];
        if (SRC) {
            const double* xn = a.xnode + 2 * ((size_t)e * nn + node);
            sq = SrcNode{__ldg(xn), __ldg(xn + 1), *a.tnow, dt, a.gamma};
            src_eval(sq, 0.0, sn);
#pragma unroll
            for (int v = 0; v < NV; ++v) d[v] = fma(dt, sn[v], d[v]);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = fma(2.0, d[v], uu[v]);
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { ft[v] = -f[v]; gt[v] = -g[v]; s[v] = uu[v] + d[v]; }
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { ft[v] = fma(8.0, f[v], ft[v]); gt[v] = fma(8.0, g[v], gt[v]); s[v] = uu[v] - d[v]; }
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { ft[v] = fma(-8.0, f[v], ft[v]); gt[v] = fma(-8.0, g[v], gt[v]); s[v] = fma(-2.0, d[v], uu[v]); }
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
        double U2v[NV], F2v[NV], G2v[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ft[v] = (ft[v] + f[v]) * (1.0 / 12.0);
            gt[v] = (gt[v] + g[v]) * (1.0 / 12.0);
            F[v] = fma(0.125, ft[v], 0.5 * f0[v]);
            G[v] = fma(0.125, gt[v], 0.5 * g0[v]);
            U[v] = fma(0.125, d[v], 0.5 * uu[v]);
            F2v[v] = fma(1.0 / 6.0, ft[v], f0[v]);
            G2v[v] = fma(1.0 / 6.0, gt[v], g0[v]);
            U2v[v] = fma(1.0 / 6.0, d[v], uu[v]);
        }
        const size_t off = ((size_t)e * nn + node);
        if (COMPACT) {
            store4(a.U2 + off * NV, d);
        } else {
            store4(a.U2 + off * NV, U2v);
            store4(a.F2 + off * 2 * NV, F2v);
            store4(a.F2 + off * 2 * NV + NV, G2v);
        }
        if (SRC) {
            double st[NV], S2v[NV];
            src_t_N34(sq, st);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Ssrc[v] = fma(0.125, st[v], 0.5 * sn[v]);
                S2v[v] = fma(1.0 / 6.0, st[v], sn[v]);
            }
            store4(a.S2 + off * NV, S2v);
        }
        if (CURVED) {
            double ft2[NV], gt2[NV];
            contravariant(Ja, F, G, ft2, gt2);
#pragma unroll
            for (int v = 0; v < NV; ++v) { F[v] = ft2[v]; G[v] = gt2[v]; }
        }
        node_put<N, C>(X, Y, el, i, j, F, G);
        if (SC) {
            if constexpr (CURVED) sc_faces_curved<N, C, REC>(a, UU, VC, F0X, F0Y, UF, FVX, FVY, el, e, i, j, blended, muscl);
            else sc_faces<N, C>(UU, VC, F0X, F0Y, FVX, FVY, el, i, j, a.speed_kind);
        }
    }
    __syncthreads();
    line_contract<N, C, true>(X, Y, tid);
    __syncthreads();
    if (active) {
        double acc[NV];
        node_sum<N, C>(X, Y, el, i, j, acc);
        if (SC) {
            if constexpr (CURVED) sc_blend_curved<N, C>(a, FVX, FVY, el, e, i, j, alpha_e, blended, acc);
            else sc_blend<N, C>(a, FVX, FVY, el, e, i, j, __ldg(a.alpha + e), acc);
        }
        double o[NV];
        volume_epilogue<n, MODE>(a, e, i, j, node, ij, dt, acc, U, F, G, o, SRC ? Ssrc : nullptr);
    }
}

// ------------------------------------------------------------------------------------------------
// MDRK stage 2 (mdrk_kernel_2!, multi_derivative_2d.jl:423-555): at u* = a.u,
// F = F2 + f_t(u*)/3, U = U2 + u*_t/3.
// ------------------------------------------------------------------------------------------------
// CURVED (mdrk_kernel_2!, src/solvers/dgsem_structured/multi_derivative_2d.jl:245-445): as in stage 1.
// SRC (FR volume integral): u*_t += dt s(u*); S = S2 + s_t(u*)/3 (multi_derivative_2d.jl:484-550), the source at
// t + dt/2 on the TreeMesh and at t on curvilinear meshes (dgsem_structured/multi_derivative_2d.jl:325-361).
// COMPACT: F2, G2, U2 recomputed from u^n (a.u_base) and stage 1's u_t (a.U2) at the start, parked in shared memory
// (three more planes) until the stage's own sums are formed.
template <int N, int MODE, bool SC, bool CURVED = false, int REC = 0, bool SRC = false, bool COMPACT = false>
static __global__ void __launch_bounds__(VolCfg<N>::THREADS, (SC && CURVED) ? VolCfg<N>::SC_CURVED_MIN_BLOCKS
                                                                         : VolCfg<N>::MDRK_MIN_BLOCKS)
    mdrk2_volume_kernel(VolArgs a) {
    static_assert(REC == 0 || (SC && CURVED), "MUSCL subcells: curvilinear shock capturing");
    static_assert(!SRC || !SC, "source terms: the FR volume integral");
    static_assert(!COMPACT || (!SC && !CURVED && !SRC && MODE == MODE_STEP), "compact stages: the plain TreeMesh step");
    using C = VolCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB;
    extern __shared__ double smem_d[];
    double* X = smem_d;
    double* Y = X + C::PLANES;
    double* F0X = Y + C::PLANES;       // shock capturing only: fluxes, u, speeds at u^n, subcell fluxes
    double* F0Y = F0X + C::PLANES;
    double* UU = F0Y + C::PLANES;
    double* VC = UU + C::PLANES;
    double* FVX = VC + C::PLANES;
    double* FVY = FVX + C::PLANES;
    double* UF = FVY + C::PLANES;      // curvilinear MUSCL: face values, 4 regions (left, right, down, up)
    const int tid = threadIdx.x;
    const double gm1 = a.gamma - 1.0;
    const int el = tid / nn;
    const int node = tid - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    double alpha_e = 0.0;
    bool blended = false, muscl = false;
    if (SC && CURVED && active) {
        alpha_e = __ldg(a.alpha + e);
        blended = !(fabs(alpha_e) <= 1e-12);
        muscl = REC >= 1 && blended && !__ldg(a.atb + e);
    }
    // dt of this element's instance (batched form) or the single dt
    const double dt = a.inst ? a.dt[__ldg(a.inst + min(e, a.E - 1))] : *a.dt;
    double us[NV], ij = 0.0, Ja[4] = {0.0, 0.0, 0.0, 0.0};
    if (active) {
        double f[NV], g[NV];
        load4(a.u + ((size_t)e * nn + node) * NV, us);
        if (CURVED) {
            load4(a.metrics + ((size_t)e * nn + node) * 4, Ja);
            ij = __ldg(a.inv_jac_node + (size_t)e * nn + node);
        } else {
            ij = __ldg(a.inv_jac + e);
        }
        euler_fluxes(gm1, us[0], us[1], us[2], us[3], f, g);
        if (CURVED) {
            double ft[NV], gt[NV];
            contravariant(Ja, f, g, ft, gt);
            node_put<N, C>(X, Y, el, i, j, ft, gt);
        } else {
            node_put<N, C>(X, Y, el, i, j, f, g);
        }
        if (COMPACT) {
            // stage 1's F2, G2 (into the F0X, F0Y planes) and U2 (the UU plane) from u^n and u_t
            double un[NV], dn[NV], F2v[NV], G2v[NV], U2v[NV];
            const size_t off = ((size_t)e * nn + node);
            load4(a.u_base + off * NV, un);
            load4(a.U2 + off * NV, dn);
            mdrk_stage1_sums(gm1, un, dn, F2v, G2v, U2v);
            node_put<N, C>(F0X, F0Y, el, i, j, F2v, G2v);
            node_put<N, C>(UU, UU, el, i, j, U2v, U2v);
        }
        if (SC) {
            // the subcell FV part uses the instantaneous u^n, not u* (multi_derivative_2d.jl:257)
            double un[NV], fn0[NV], gn0[NV];
            load4(a.u_base + ((size_t)e * nn + node) * NV, un);
            euler_fluxes(gm1, un[0], un[1], un[2], un[3], fn0, gn0);
            node_put<N, C>(F0X, F0Y, el, i, j, fn0, gn0);
            sc_park<N, C>(UU, VC, el, i, j, un, a.gamma, a.status);
        }
    }
    __syncthreads();
    // (the MUSCL face values are read by the neighbours after the next barrier)
    if (SC && CURVED && REC >= 1 && muscl) sc_muscl_faces<N, C, REC>(a, UU, UF, el, e, i, j, gm1, alpha_e, dt, ij);
    line_contract<N, C, false>(X, Y, tid);
    __syncthreads();
    double U[NV], F[NV], G[NV], Ssrc[NV] = {0.0, 0.0, 0.0, 0.0};
    if (active) {
        double d[NV], ft[NV], gt[NV], f[NV], g[NV], s[NV];
        node_sum<N, C>(X, Y, el, i, j, d);
        const double s0 = -dt * ij;
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v] *= s0;
        if (SRC) {
            const double* xn = a.xnode + 2 * ((size_t)e * nn + node);
            // at t + dt/2 on the TreeMesh (multi_derivative_2d.jl:484-495), at t on curvilinear meshes
            // (dgsem_structured/multi_derivative_2d.jl:336, 361)
            const SrcNode sq{__ldg(xn), __ldg(xn + 1), CURVED ? *a.tnow : *a.tnow + 0.5 * dt, dt, a.gamma};
            double sn[NV], st[NV];
            src_eval(sq, 0.0, sn);
#pragma unroll
            for (int v = 0; v < NV; ++v) d[v] = fma(dt, sn[v], d[v]);
            src_t_N34(sq, st);
            load4(a.S2 + ((size_t)e * nn + node) * NV, sn);
#pragma unroll
            for (int v = 0; v < NV; ++v) Ssrc[v] = fma(1.0 / 3.0, st[v], sn[v]);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = fma(2.0, d[v], us[v]);
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { ft[v] = -f[v]; gt[v] = -g[v]; s[v] = us[v] + d[v]; }
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { ft[v] = fma(8.0, f[v], ft[v]); gt[v] = fma(8.0, g[v], gt[v]); s[v] = us[v] - d[v]; }
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { ft[v] = fma(-8.0, f[v], ft[v]); gt[v] = fma(-8.0, g[v], gt[v]); s[v] = fma(-2.0, d[v], us[v]); }
        euler_fluxes(gm1, s[0], s[1], s[2], s[3], f, g);
        const size_t off = ((size_t)e * nn + node);
        double U2v[NV], F2v[NV], G2v[NV];
        if (COMPACT) {
            node_get<N, C>(F0X, F0Y, el, i, j, F2v, G2v);
            node_get<N, C>(UU, UU, el, i, j, U2v, U2v);
        } else {
            load4(a.U2 + off * NV, U2v);
            load4(a.F2 + off * 2 * NV, F2v);
            load4(a.F2 + off * 2 * NV + NV, G2v);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ft[v] = (ft[v] + f[v]) * (1.0 / 12.0);
            gt[v] = (gt[v] + g[v]) * (1.0 / 12.0);
            F[v] = fma(1.0 / 3.0, ft[v], F2v[v]);
            G[v] = fma(1.0 / 3.0, gt[v], G2v[v]);
            U[v] = fma(1.0 / 3.0, d[v], U2v[v]);
        }
        if (CURVED) {
            double ft2[NV], gt2[NV];
            contravariant(Ja, F, G, ft2, gt2);
#pragma unroll
            for (int v = 0; v < NV; ++v) { F[v] = ft2[v]; G[v] = gt2[v]; }
        }
        node_put<N, C>(X, Y, el, i, j, F, G);
        if (SC) {
            if constexpr (CURVED) sc_faces_curved<N, C, REC>(a, UU, VC, F0X, F0Y, UF, FVX, FVY, el, e, i, j, blended, muscl);
            else sc_faces<N, C>(UU, VC, F0X, F0Y, FVX, FVY, el, i, j, a.speed_kind);
        }
    }
    __syncthreads();
    line_contract<N, C, true>(X, Y, tid);
    __syncthreads();
    // the step's final values: per-element CFL slots as the LW kernel writes them (plain TreeMesh MDRK step)
    constexpr bool SLOTS = MODE == MODE_STEP && !SC && !CURVED;
    double l1 = 0.0, l2 = 0.0;
    if (active) {
        double acc[NV];
        node_sum<N, C>(X, Y, el, i, j, acc);
        if (SC) {
            if constexpr (CURVED) sc_blend_curved<N, C>(a, FVX, FVY, el, e, i, j, alpha_e, blended, acc);
            else sc_blend<N, C>(a, FVX, FVY, el, e, i, j, __ldg(a.alpha + e), acc);
        }
        double o[NV];
        volume_epilogue<n, MODE>(a, e, i, j, node, ij, dt, acc, U, F, G, o, SRC ? Ssrc : nullptr);
        if (SLOTS && a.cfl_slots && i > 0 && i < n - 1 && j > 0 && j < n - 1) node_speeds(a.gamma, o, a.status, l1, l2);
    }
    if (SLOTS && a.cfl_slots) write_interior_slots<N, C>(a, X, active, el, i, j, tid, l1, l2);
}

}  // namespace tlw
