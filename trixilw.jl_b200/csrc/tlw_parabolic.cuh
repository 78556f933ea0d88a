// tlw_parabolic.cuh -- compressible Navier-Stokes on a periodic TreeMesh{2} with the LW scheme
// (rhs! of SemidiscretizationHyperbolicParabolic, src/solvers/dgsem_tree/dg_2d_parabolic.jl:15-99):
//   grad_volume_kernel + grad_interface_kernel: BR1 gradients of the conservative variables
//     (Trixi calc_gradient!: J^{-1} (Dhat u + lifted interface averages (u_L + u_R) / 2));
//   par_volume_kernel: the LW procedure of lw_volume_kernel_3! / _4! (dg_2d_parabolic.jl:725-1860) with the
//     flux f(u) - f_v(u, grad u), the perturbed states carried with their gradients (grad d_m = J^{-1} D d_m),
//     advective and viscous time averages kept apart for the surface;
//   the interface kernel then subtracts the central viscous flux (Fv_L + Fv_R) / 2 from the LW surface flux
//     (calc_interface_flux_hyperbolic_parabolic!, dg_2d_parabolic.jl:1911-1949);
//   par_speed_kernel: the advective and viscous maxima of compute_dt (src/solvers/lwfr.jl:192-210) and the
//     parabolic max_dt (src/equations/compressible_navier_stokes_2d.jl:204-261).
// Viscous flux (Trixi CompressibleNavierStokesDiffusion2D with conservative gradient variables, T = p / rho):
//   primitive derivatives from the conservative gradients (convert_derivative_to_primitive,
//   compressible_navier_stokes_2d.jl:36-57), tau = mu (grad v + grad v^T - 2/3 div v I), q = mu kappa grad T,
//   kappa = gamma / ((gamma - 1) Pr).
#pragma once
#include "tlw_device.cuh"
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"
#include "tlw_curved.cuh"

namespace tlw {

struct NSParams {
    double gamma, mu, Pr, kappa;
};

__device__ __forceinline__ void ns_viscous_fluxes(const NSParams& p, const double* u, const double* gx,
                                                  const double* gy, double* fv, double* gv) {
    const double ir = nr_reciprocal(u[0]);
    const double v1 = u[1] * ir, v2 = u[2] * ir;
    const double pr = (p.gamma - 1.0) * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    const double T = pr * ir;
    const double kin = 0.5 * (v1 * v1 + v2 * v2);
    // primitive derivatives along one direction from the conservative gradient W
    auto prim = [&](const double* W, double& v1d, double& v2d, double& Td) {
        const double rd = W[0];
        v1d = (W[1] - rd * v1) * ir;
        v2d = (W[2] - rd * v2) * ir;
        const double pd = (W[3] - rd * kin - u[0] * (v1 * v1d + v2 * v2d)) * (p.gamma - 1.0);
        Td = (pd - rd * T) * ir;
    };
    double v1x, v2x, Tx, v1y, v2y, Ty;
    prim(gx, v1x, v2x, Tx);
    prim(gy, v1y, v2y, Ty);
    const double t11 = 4.0 / 3.0 * v1x - 2.0 / 3.0 * v2y;
    const double t12 = v1y + v2x;
    const double t22 = 4.0 / 3.0 * v2y - 2.0 / 3.0 * v1x;
    fv[0] = 0.0;
    fv[1] = t11 * p.mu;
    fv[2] = t12 * p.mu;
    fv[3] = (v1 * t11 + v2 * t12 + p.kappa * Tx) * p.mu;
    gv[0] = 0.0;
    gv[1] = t12 * p.mu;
    gv[2] = t22 * p.mu;
    gv[3] = (v1 * t12 + v2 * t22 + p.kappa * Ty) * p.mu;
}

template <int N>
struct ParCfg {
    static constexpr int n = N + 1;
    static constexpr int nn = n * n;
    static constexpr int EB = VolCfg<N>::EB;
    static constexpr int THREADS = VolCfg<N>::THREADS;
    static constexpr int DEPTH = N >= 4 ? 4 : 3;
    static constexpr int TILE = NV * EB * nn;   // 4 values per node of the CTA
    // D, Dhat; contraction tiles X, Y, W; perturbed states P (4) and their gradients GX, GY (4 + 4)
    static constexpr size_t smem_bytes() { return (size_t)(2 * nn + 15 * TILE) * sizeof(double); }
};

// gradient volume term: gx = J^{-1} Dhat u (along i), gy = J^{-1} Dhat u (along j); on a curvilinear mesh
// (metrics [4, i, j, e], inv_jac per node) the two reference derivatives r_xi, r_eta mix as
// gx = J^{-1} (Ja^1_1 r_xi + Ja^2_1 r_eta), gy = J^{-1} (Ja^1_2 r_xi + Ja^2_2 r_eta) (Trixi calc_gradient! for
// P4estMesh{2})
template <int N, bool CURVED = false>
static __global__ void __launch_bounds__(VolCfg<N>::THREADS) grad_volume_kernel(const double* __restrict__ u,
                                                                              const double* __restrict__ inv_jac,
                                                                              int E, double* gx, double* gy,
                                                                              const double* __restrict__ metrics = nullptr) {
    using C = ParCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB;
    __shared__ double sU[NV * EB * nn];
    __shared__ double sDh[nn];
    for (int k = threadIdx.x; k < nn; k += blockDim.x) sDh[k] = c_tlw_Dhat[N][k];
    const int el = threadIdx.x / nn, node = threadIdx.x - (threadIdx.x / nn) * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < E;
    if (active) {
        double x[NV];
        load4(u + ((size_t)e * nn + node) * NV, x);
#pragma unroll
        for (int v = 0; v < NV; ++v) sU[(v * EB + el) * nn + node] = x[v];
    }
    __syncthreads();
    if (!active) return;
    const double ij = CURVED ? __ldg(inv_jac + (size_t)e * nn + node) : __ldg(inv_jac + e);
    double J[4] = {1.0, 0.0, 0.0, 1.0};
    if (CURVED) load4(metrics + ((size_t)e * nn + node) * 4, J);
    double ox[NV], oy[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double* p = sU + (v * EB + el) * nn;
        double sx = 0.0, sy = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) {
            sx = fma(sDh[i * n + k], p[k + n * j], sx);
            sy = fma(sDh[j * n + k], p[i + n * k], sy);
        }
        if (CURVED) {
            ox[v] = ij * fma(J[0], sx, J[2] * sy);
            oy[v] = ij * fma(J[1], sx, J[3] * sy);
        } else {
            ox[v] = ij * sx;
            oy[v] = ij * sy;
        }
    }
    store4(gx + ((size_t)e * nn + node) * NV, ox);
    store4(gy + ((size_t)e * nn + node) * NV, oy);
}

// gradient interface term (BR1): x-interfaces lift into gx, y-interfaces into gy (one launch for both)
template <int N>
static __global__ void __launch_bounds__(128) grad_interface_kernel(const double* __restrict__ u, const int* xl,
                                                                    const int* xr, int nx, const int* yl,
                                                                    const int* yr, int ny,
                                                                    const double* __restrict__ inv_jac,
                                                                    double inv_w_first, double inv_w_last,
                                                                    double* gx, double* gy) {
    constexpr int n = N + 1, nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int k = t / n;
    const int l = t - k * n;
    int o = 1;
    if (k >= nx) {
        k -= nx;
        o = 2;
        if (k >= ny) return;
    }
    const int le = o == 1 ? __ldg(xl + k) : __ldg(yl + k);
    const int re = o == 1 ? __ldg(xr + k) : __ldg(yr + k);
    const int nL = o == 1 ? (n - 1) + n * l : l + n * (n - 1);
    const int nR = o == 1 ? n * l : l;
    double uL[NV], uR[NV], x[NV];
    load4(u + ((size_t)le * nn + nL) * NV, uL);
    load4(u + ((size_t)re * nn + nR) * NV, uR);
    double* g = o == 1 ? gx : gy;
    const double cL = __ldg(inv_jac + le) * inv_w_last, cR = -__ldg(inv_jac + re) * inv_w_first;
    double* pL = g + ((size_t)le * nn + nL) * NV;
    double* pR = g + ((size_t)re * nn + nR) * NV;
    load4_rw(pL, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(cL, 0.5 * (uL[v] + uR[v]), x[v]);
    store4(pL, x);
    load4_rw(pR, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(cR, 0.5 * (uL[v] + uR[v]), x[v]);
    store4(pR, x);
}

// gradient boundary term (Trixi calc_boundary_flux_by_direction_gradient!): the wall value of
// BoundaryConditionNavierStokesWall(NoSlip(v), Adiabatic | Isothermal) (compressible_navier_stokes_2d.jl:92-124),
// prim2cons(rho_inner, v_wall, p) with p the inner pressure (adiabatic) or rho_inner T_wall (isothermal), is the
// flux itself; x-boundaries lift into gx, y-boundaries into gy
template <int N>
static __global__ void __launch_bounds__(128) grad_boundary_kernel(const double* __restrict__ u, const int* element,
                                                                   const int* direction, const int* wall_kind,
                                                                   const double* __restrict__ wall, int B,
                                                                   const double* __restrict__ inv_jac, double gamma,
                                                                   double inv_w_first, double inv_w_last, double* gx,
                                                                   double* gy) {
    constexpr int n = N + 1, nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n;
    const int l = t - k * n;
    if (k >= B) return;
    const int e = __ldg(element + k), dir = __ldg(direction + k);
    const int node = dir == 1 ? n * l : dir == 2 ? (n - 1) + n * l : dir == 3 ? l : l + n * (n - 1);
    double ui[NV], x[NV];
    load4(u + ((size_t)e * nn + node) * NV, ui);
    const double* w = wall + 3 * ((size_t)k * n + l);
    const double v1 = __ldg(w), v2 = __ldg(w + 1);
    const double rho = ui[0];
    const double p = __ldg(wall_kind + k) == WALL_ADIABATIC
                         ? (gamma - 1.0) * (ui[3] - 0.5 * (ui[1] * ui[1] + ui[2] * ui[2]) / rho)
                         : rho * __ldg(w + 2);
    const double uo[NV] = {rho, rho * v1, rho * v2, p / (gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2)};
    double* g = (dir <= 2 ? gx : gy) + ((size_t)e * nn + node) * NV;
    const double c = (dir % 2 == 0 ? inv_w_last : -inv_w_first) * __ldg(inv_jac + e);
    load4_rw(g, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(c, uo[v], x[v]);
    store4(g, x);
}

// gradient surface terms on a curvilinear mesh: the face value u* times the element's own outward normal and
// 1 / w, scaled by J^{-1} of the node, into both gx and gy (interfaces of one colour per launch, so that no
// launch touches a corner node twice)
__device__ __forceinline__ void curved_grad_lift(const double* __restrict__ metrics, const double* __restrict__ inv_jac,
                                                 int n, int e, int f, int node, const double* us, double iw,
                                                 double* gx, double* gy) {
    const int nn = n * n;
    double J[4], x[NV], y[NV];
    load4(metrics + ((size_t)e * nn + node) * 4, J);
    const double sg = (f & 1) ? 1.0 : -1.0;
    const double c = iw * __ldg(inv_jac + (size_t)e * nn + node);
    const double n0 = sg * (f < 2 ? J[0] : J[2]) * c, n1 = sg * (f < 2 ? J[1] : J[3]) * c;
    double* px = gx + ((size_t)e * nn + node) * NV;
    double* py = gy + ((size_t)e * nn + node) * NV;
    load4_rw(px, x);
    load4_rw(py, y);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        x[v] = fma(n0, us[v], x[v]);
        y[v] = fma(n1, us[v], y[v]);
    }
    store4(px, x);
    store4(py, y);
}

template <int N>
static __global__ void __launch_bounds__(128) curved_grad_interface_kernel(
    const double* __restrict__ u, const int* p_elem, const int* s_elem, const int* faces, int count,
    const double* __restrict__ metrics, const double* __restrict__ inv_jac, double inv_w_first, double inv_w_last,
    double* gx, double* gy) {
    constexpr int n = N + 1, nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n;
    const int l = t - k * n;
    if (k >= count) return;
    const int pe = __ldg(p_elem + k), se = __ldg(s_elem + k), code = __ldg(faces + k);
    const int pf = code & 3, sf = (code >> 2) & 3;
    const int ls = (code >> 4) & 1 ? n - 1 - l : l;
    const int np = face_node_index(n, pf, l), ns = face_node_index(n, sf, ls);
    double uP[NV], uS[NV], us[NV];
    load4(u + ((size_t)pe * nn + np) * NV, uP);
    load4(u + ((size_t)se * nn + ns) * NV, uS);
#pragma unroll
    for (int v = 0; v < NV; ++v) us[v] = 0.5 * (uP[v] + uS[v]);
    curved_grad_lift(metrics, inv_jac, n, pe, pf, np, us, (pf & 1) ? inv_w_last : inv_w_first, gx, gy);
    curved_grad_lift(metrics, inv_jac, n, se, sf, ns, us, (sf & 1) ? inv_w_last : inv_w_first, gx, gy);
}

template <int N>
static __global__ void __launch_bounds__(128) curved_grad_boundary_kernel(
    const double* __restrict__ u, const int* elem, const int* face, const int* index, int count, const int* wall_kind,
    const double* __restrict__ wall, const double* __restrict__ metrics, const double* __restrict__ inv_jac,
    double gamma, double inv_w_first, double inv_w_last, double* gx, double* gy) {
    constexpr int n = N + 1, nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n;
    const int l = t - k * n;
    if (k >= count) return;
    const int e = __ldg(elem + k), f = __ldg(face + k), b = __ldg(index + k);
    const int node = face_node_index(n, f, l);
    double ui[NV];
    load4(u + ((size_t)e * nn + node) * NV, ui);
    const double* w = wall + 3 * ((size_t)b * n + l);
    const double v1 = __ldg(w), v2 = __ldg(w + 1);
    const double rho = ui[0];
    const double p = __ldg(wall_kind + b) == WALL_ADIABATIC
                         ? (gamma - 1.0) * (ui[3] - 0.5 * (ui[1] * ui[1] + ui[2] * ui[2]) / rho)
                         : rho * __ldg(w + 2);
    const double uo[NV] = {rho, rho * v1, rho * v2, p / (gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2)};
    curved_grad_lift(metrics, inv_jac, n, e, f, node, uo, (f & 1) ? inv_w_last : inv_w_first, gx, gy);
}

struct ParArgs {
    const double* u;
    const double* gx;
    const double* gy;
    double* out;
    double* tU;
    double* tF;      // advective normal flux traces
    double* tFv;     // viscous normal flux traces
    const double* inv_jac;
    const double* dt;
    int E;
    NSParams ns;
    const double* metrics;   // curvilinear: [4, i, j, e] (inv_jac is then per node)
};

template <int DEPTH>
struct ParLW {
    static __device__ __forceinline__ constexpr double tw(int s) {
        return s == 1 ? 0.5 : s == 2 ? 1.0 / 6.0 : s == 3 ? 1.0 / 24.0 : 1.0 / 120.0;
    }
    static __device__ __forceinline__ constexpr double a(int q, int m) {
        return q == 0 ? (m == 1 ? -1.0 : m == 2 ? 0.5 : m == 3 ? -1.0 / 6.0 : 1.0 / 24.0)
             : q == 1 ? (m == 1 ? 1.0 : m == 2 ? 0.5 : m == 3 ? 1.0 / 6.0 : 1.0 / 24.0)
             : q == 2 ? (m == 1 ? -2.0 : m == 2 ? 2.0 : m == 3 ? -4.0 / 3.0 : 2.0 / 3.0)
                      : (m == 1 ? 2.0 : m == 2 ? 2.0 : m == 3 ? 4.0 / 3.0 : 2.0 / 3.0);
    }
    static __device__ __forceinline__ constexpr double w(int s, int k) {
        return s == 1 ? (k == 0 ? 0.0 : k == 1 ? -8.0 / 12.0 : k == 2 ? 8.0 / 12.0 : k == 3 ? 1.0 / 12.0 : -1.0 / 12.0)
             : s == 2 ? (DEPTH == 4 ? (k == 0 ? -30.0 / 12.0 : k <= 2 ? 16.0 / 12.0 : -1.0 / 12.0)
                                    : (k == 0 ? -2.0 : k <= 2 ? 1.0 : 0.0))
             : s == 3 ? (k == 0 ? 0.0 : k == 1 ? 1.0 : k == 2 ? -1.0 : k == 3 ? -0.5 : 0.5)
                      : (k == 0 ? 3.0 : k <= 2 ? -2.0 : 0.5);
    }
};

// CURVED: the stage fluxes are the contravariant ones (Ja^1 . (f_a - f_v, g_a - g_v), Ja^2 . (...)), d_m carries
// the node's J^{-1} and its gradient J^{-1} (Ja^1_d D_xi d_m + Ja^2_d D_eta d_m) (src/solvers/dgsem_p4est/
// dg_2d_parabolic.jl:51-104, 641-1787); the face traces are the contravariant fluxes along the face direction.
template <int N, int MODE, bool CURVED = false>
static __global__ void __launch_bounds__(ParCfg<N>::THREADS, 1) par_volume_kernel(ParArgs a) {
    using C = ParCfg<N>;
    using K = ParLW<C::DEPTH>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, DEPTH = C::DEPTH, TILE = C::TILE;
    extern __shared__ double sm[];
    double* sD = sm;
    double* sDh = sm + nn;
    double* X = sm + 2 * nn;
    double* Y = X + TILE;
    double* W = Y + TILE;
    double* P = W + TILE;          // [q][v] planes: P + q * TILE
    double* GX = P + 4 * TILE;
    double* GY = GX + 4 * TILE;
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        sD[k] = c_tlw_D[N][k];
        sDh[k] = c_tlw_Dhat[N][k];
    }
    const int el = threadIdx.x / nn;
    const int node = threadIdx.x - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    const bool in_tile = el < EB;
    const int slot = in_tile ? el : 0;
    auto at = [&](double* T, int v) -> double* { return T + (v * EB + slot) * nn + node; };
    auto put = [&](double* T, int v, double x) {
        if (in_tile) *at(T, v) = x;
    };
    auto cx = [&](const double* M, const double* F, int v) {
        const double* p = F + (v * EB + slot) * nn + n * j;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[i * n + k], p[k], s);
        return s;
    };
    auto cy = [&](const double* M, const double* F, int v) {
        const double* p = F + (v * EB + slot) * nn + i;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[j * n + k], p[n * k], s);
        return s;
    };
    double u[NV] = {1.0, 0.0, 0.0, 2.5}, gx[NV] = {0, 0, 0, 0}, gy[NV] = {0, 0, 0, 0};
    double ij = 1.0, J[4] = {1.0, 0.0, 0.0, 1.0};
    if (active) {
        load4(a.u + ((size_t)e * nn + node) * NV, u);
        load4(a.gx + ((size_t)e * nn + node) * NV, gx);
        load4(a.gy + ((size_t)e * nn + node) * NV, gy);
        if (CURVED) {
            ij = __ldg(a.inv_jac + (size_t)e * nn + node);
            load4(a.metrics + ((size_t)e * nn + node) * 4, J);
        } else {
            ij = __ldg(a.inv_jac + e);
        }
    }
    // the flux pair along the reference coordinates
    auto contra = [&](double f, double g, double& cf, double& cg) {
        if (CURVED) {
            cf = fma(J[0], f, J[1] * g);
            cg = fma(J[2], f, J[3] * g);
        } else {
            cf = f;
            cg = g;
        }
    };
    auto put_pair = [&](int v, double f, double g) {
        double cf, cg;
        contra(f, g, cf, cg);
        put(X, v, cf);
        put(Y, v, cg);
    };
    const double dt = *a.dt;
    const double sc = -dt * ij;
    const double gm1 = a.ns.gamma - 1.0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            put(P + q * TILE, v, u[v]);
            put(GX + q * TILE, v, gx[v]);
            put(GY + q * TILE, v, gy[v]);
        }
    double Fa[NV], Ga[NV], Fv[NV], Gv[NV], U[NV];
    {
        double fv[NV], gv[NV];
        euler_fluxes(gm1, u[0], u[1], u[2], u[3], Fa, Ga);
        ns_viscous_fluxes(a.ns, u, gx, gy, fv, gv);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            Fv[v] = fv[v]; Gv[v] = gv[v]; U[v] = u[v];
            put_pair(v, Fa[v] - fv[v], Ga[v] - gv[v]);
        }
    }
    // d and its gradient from the stage fluxes in X, Y
    double d[NV], dx[NV], dy[NV];
    auto derive = [&]() {
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v] = sc * (cx(sD, X, v) + cy(sD, Y, v));
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) put(W, v, d[v]);
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double r1 = cx(sD, W, v), r2 = cy(sD, W, v);
            if (CURVED) {
                dx[v] = ij * fma(J[0], r1, J[2] * r2);
                dy[v] = ij * fma(J[1], r1, J[3] * r2);
            } else {
                dx[v] = ij * r1;
                dy[v] = ij * r2;
            }
        }
        __syncthreads();
    };
    derive();
#pragma unroll
    for (int s = 1; s <= DEPTH; ++s) {
        double sfa[NV] = {0, 0, 0, 0}, sga[NV] = {0, 0, 0, 0}, sfv[NV] = {0, 0, 0, 0}, sgv[NV] = {0, 0, 0, 0};
#pragma unroll
        for (int v = 0; v < NV; ++v) U[v] = fma(K::tw(s), d[v], U[v]);
        if (K::w(s, 0) != 0.0) {
            double fa[NV], ga[NV], fv[NV], gv[NV];
            euler_fluxes(gm1, u[0], u[1], u[2], u[3], fa, ga);
            ns_viscous_fluxes(a.ns, u, gx, gy, fv, gv);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                sfa[v] = K::w(s, 0) * fa[v]; sga[v] = K::w(s, 0) * ga[v];
                sfv[v] = K::w(s, 0) * fv[v]; sgv[v] = K::w(s, 0) * gv[v];
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            // advance state q (and its gradients) by the newest derivative
            double Pq[NV], Xq[NV], Yq[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Pq[v] = fma(K::a(q, s), d[v], *at(P + q * TILE, v));
                Xq[v] = fma(K::a(q, s), dx[v], *at(GX + q * TILE, v));
                Yq[v] = fma(K::a(q, s), dy[v], *at(GY + q * TILE, v));
                put(P + q * TILE, v, Pq[v]);
                put(GX + q * TILE, v, Xq[v]);
                put(GY + q * TILE, v, Yq[v]);
            }
            if (K::w(s, 1 + q) == 0.0) continue;
            double fa[NV], ga[NV], fv[NV], gv[NV];
            euler_fluxes(gm1, Pq[0], Pq[1], Pq[2], Pq[3], fa, ga);
            ns_viscous_fluxes(a.ns, Pq, Xq, Yq, fv, gv);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                sfa[v] = fma(K::w(s, 1 + q), fa[v], sfa[v]); sga[v] = fma(K::w(s, 1 + q), ga[v], sga[v]);
                sfv[v] = fma(K::w(s, 1 + q), fv[v], sfv[v]); sgv[v] = fma(K::w(s, 1 + q), gv[v], sgv[v]);
            }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            Fa[v] = fma(K::tw(s), sfa[v], Fa[v]); Ga[v] = fma(K::tw(s), sga[v], Ga[v]);
            Fv[v] = fma(K::tw(s), sfv[v], Fv[v]); Gv[v] = fma(K::tw(s), sgv[v], Gv[v]);
        }
        if (s < DEPTH) {
#pragma unroll
            for (int v = 0; v < NV; ++v) put_pair(v, sfa[v] - sfv[v], sga[v] - sgv[v]);
            derive();
        }
    }
    // du = Dhat (Fa - Fv) + Dhat (Ga - Gv) (contravariant on a curvilinear mesh)
#pragma unroll
    for (int v = 0; v < NV; ++v) put_pair(v, Fa[v] - Fv[v], Ga[v] - Gv[v]);
    __syncthreads();
    if (!active) return;
    double acc[NV], o[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = cx(sDh, X, v) + cy(sDh, Y, v);
    const size_t off = ((size_t)e * nn + node) * NV;
    if (MODE == MODE_RHS) {
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = -ij * acc[v];
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = fma(sc, acc[v], u[v]);
    }
    store4(a.out + off, o);
    if (CURVED) {
        // traces: the fluxes along the face's reference direction
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double cf, cg;
            contra(Fa[v], Ga[v], cf, cg);
            Fa[v] = cf;
            Ga[v] = cg;
            contra(Fv[v], Gv[v], cf, cg);
            Fv[v] = cf;
            Gv[v] = cg;
        }
    }
    const size_t tb = (size_t)e * 4 * n * NV;
    if (i == 0) { store4(a.tU + tb + (0 * n + j) * NV, U); store4(a.tF + tb + (0 * n + j) * NV, Fa); store4(a.tFv + tb + (0 * n + j) * NV, Fv); }
    if (i == n - 1) { store4(a.tU + tb + (1 * n + j) * NV, U); store4(a.tF + tb + (1 * n + j) * NV, Fa); store4(a.tFv + tb + (1 * n + j) * NV, Fv); }
    if (j == 0) { store4(a.tU + tb + (2 * n + i) * NV, U); store4(a.tF + tb + (2 * n + i) * NV, Ga); store4(a.tFv + tb + (2 * n + i) * NV, Gv); }
    if (j == n - 1) { store4(a.tU + tb + (3 * n + i) * NV, U); store4(a.tF + tb + (3 * n + i) * NV, Ga); store4(a.tFv + tb + (3 * n + i) * NV, Gv); }
}

// advective and viscous maxima for the parabolic dt: max_bits <- max_e J^{-1} (l1 + l2),
// visc_bits <- max_nodes J^{-2} max(4 mu / (3 rho), mu kappa / (rho Pr))
// (on a curvilinear mesh inv_jac is the per-node array and element e reads its e-th entry, which is how the
// reference's parabolic max_dt indexes cache.elements.inverse_jacobian[element] on a P4estMesh; adv_bits then
// receives this TreeMesh-style advective maximum, the CFL one comes from curved_max_speed_kernel)
template <int N>
static __global__ void __launch_bounds__(MS_THREADS) par_speed_kernel(const double* __restrict__ u,
                                                                      const double* __restrict__ inv_jac, int E,
                                                                      NSParams ns, StepState* s,
                                                                      unsigned long long* visc_bits,
                                                                      unsigned long long* adv_bits) {
    constexpr int n = N + 1, nn = n * n;
    constexpr int ELEMS = MsCfg<N>::ELEMS;
    __shared__ double l1s[ELEMS * nn], l2s[ELEMS * nn];
    __shared__ double wmax[MS_THREADS / 32], wvis[MS_THREADS / 32];
    const int e0 = blockIdx.x * ELEMS;
    const int ne = min(ELEMS, E - e0);
    const double gm1 = ns.gamma - 1.0;
    double vis = 0.0;
    for (int k = threadIdx.x; k < ne * nn; k += MS_THREADS) {
        double x[NV];
        load4(u + ((size_t)e0 * nn + k) * NV, x);
        const double ir = 1.0 / x[0];
        const double v1 = x[1] * ir, v2 = x[2] * ir;
        const double p = gm1 * (x[3] - 0.5 * (x[1] * v1 + x[2] * v2));
        const double c = checked_sqrt(ns.gamma * p * ir, &s->status);
        l1s[k] = fabs(v1) + c;
        l2s[k] = fabs(v2) + c;
        const double ij = __ldg(inv_jac + e0 + k / nn);
        vis = fmax(vis, ij * ij * fmax(4.0 * ns.mu / (3.0 * x[0]), ns.mu * ns.kappa / (x[0] * ns.Pr)));
    }
    __syncthreads();
    double m = 0.0;
    if (threadIdx.x < ne) {
        double ml1 = 0.0, ml2 = 0.0;
        for (int k = 0; k < nn; ++k) {
            ml1 = fmax(ml1, l1s[threadIdx.x * nn + k]);
            ml2 = fmax(ml2, l2s[threadIdx.x * nn + k]);
        }
        m = __ldg(inv_jac + e0 + threadIdx.x) * (ml1 + ml2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        vis = fmax(vis, __shfl_xor_sync(0xffffffffu, vis, o));
    }
    if ((threadIdx.x & 31) == 0) {
        wmax[threadIdx.x >> 5] = m;
        wvis[threadIdx.x >> 5] = vis;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmax[0], bv = wvis[0];
        for (int w = 1; w < MS_THREADS / 32; ++w) {
            b = fmax(b, wmax[w]);
            bv = fmax(bv, wvis[w]);
        }
        if (b > 0.0) atomicMax(adv_bits, (unsigned long long)__double_as_longlong(b));
        if (bv > 0.0) atomicMax(visc_bits, (unsigned long long)__double_as_longlong(bv));
    }
}

// Curvilinear Navier-Stokes: curved_max_speed_kernel's CFL maximum (into s->max_bits) and par_speed_kernel's
// parabolic maxima (adv_bits, visc_bits; inv_jac_lin read by the element-linear index, as that kernel reads it)
// in one pass over u, with the same operations for each.
template <int N>
static __global__ void __launch_bounds__(MS_THREADS) curved_par_speed_kernel(const double* __restrict__ u,
                                                                             const double* __restrict__ metrics,
                                                                             const double* __restrict__ inv_jac,
                                                                             int E, NSParams ns, StepState* s,
                                                                             unsigned long long* visc_bits,
                                                                             unsigned long long* adv_bits) {
    constexpr int n = N + 1, nn = n * n;
    constexpr int ELEMS = MsCfg<N>::ELEMS;
    __shared__ double c1s[ELEMS * nn], c2s[ELEMS * nn], l1s[ELEMS * nn], l2s[ELEMS * nn];
    __shared__ double wmax[MS_THREADS / 32], wadv[MS_THREADS / 32], wvis[MS_THREADS / 32];
    const int e0 = blockIdx.x * ELEMS;
    const int ne = min(ELEMS, E - e0);
    const double gm1 = ns.gamma - 1.0;
    double vis = 0.0;
    for (int k = threadIdx.x; k < ne * nn; k += MS_THREADS) {
        const size_t node = (size_t)e0 * nn + k;
        double x[NV], J[4];
        load4w(u + node * NV, x);
        load4w(metrics + node * 4, J);
        const double ir = 1.0 / x[0];
        const double v1 = x[1] * ir, v2 = x[2] * ir;
        const double p = gm1 * (x[3] - 0.5 * (x[1] * v1 + x[2] * v2));
        const double c = checked_sqrt(ns.gamma * p * ir, &s->status);
        const double l1 = fabs(v1) + c, l2 = fabs(v2) + c;
        const double ijn = fabs(__ldg(inv_jac + node));
        c1s[k] = fabs(J[0] * l1 + J[1] * l2) * ijn;
        c2s[k] = fabs(J[2] * l1 + J[3] * l2) * ijn;
        l1s[k] = l1;
        l2s[k] = l2;
        const double ij = __ldg(inv_jac + e0 + k / nn);
        vis = fmax(vis, ij * ij * fmax(4.0 * ns.mu / (3.0 * x[0]), ns.mu * ns.kappa / (x[0] * ns.Pr)));
    }
    __syncthreads();
    double m = 0.0, ma = 0.0;
    if (threadIdx.x < ne) {
        double m1 = 0.0, m2 = 0.0, ml1 = 0.0, ml2 = 0.0;
        for (int k = 0; k < nn; ++k) {
            m1 = fmax(m1, c1s[threadIdx.x * nn + k]);
            m2 = fmax(m2, c2s[threadIdx.x * nn + k]);
            ml1 = fmax(ml1, l1s[threadIdx.x * nn + k]);
            ml2 = fmax(ml2, l2s[threadIdx.x * nn + k]);
        }
        m = m1 + m2;
        ma = __ldg(inv_jac + e0 + threadIdx.x) * (ml1 + ml2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
        vis = fmax(vis, __shfl_xor_sync(0xffffffffu, vis, o));
    }
    if ((threadIdx.x & 31) == 0) {
        wmax[threadIdx.x >> 5] = m;
        wadv[threadIdx.x >> 5] = ma;
        wvis[threadIdx.x >> 5] = vis;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmax[0], ba = wadv[0], bv = wvis[0];
        for (int w = 1; w < MS_THREADS / 32; ++w) {
            b = fmax(b, wmax[w]);
            ba = fmax(ba, wadv[w]);
            bv = fmax(bv, wvis[w]);
        }
        if (b > 0.0) atomicMax(&s->max_bits, (unsigned long long)__double_as_longlong(b));
        if (ba > 0.0) atomicMax(adv_bits, (unsigned long long)__double_as_longlong(ba));
        if (bv > 0.0) atomicMax(visc_bits, (unsigned long long)__double_as_longlong(bv));
    }
}

// dt = min(cfl 2 / (n lam_a), cfl / ((lam_a' + 2 (2N + 1) lam_v) 2 (2N + 1))), then the set_dt! clamp;
// lam_a' = lam_a on a TreeMesh, visc_bits[1] (the parabolic max_dt's own advective maximum) when curved
static __global__ void par_finalize_dt_kernel(StepState* s, unsigned long long* visc_bits, int N, int curved = 0) {
    const double tiny = 4.9406564584124654e-324;
    double la = __longlong_as_double((long long)s->max_bits);
    double lv = __longlong_as_double((long long)visc_bits[0]);
    double lq = curved ? __longlong_as_double((long long)visc_bits[1]) : la;
    if (!(la > tiny)) la = tiny;
    if (!(lv > tiny)) lv = tiny;
    if (!(lq > tiny)) lq = tiny;
    const double k = 2.0 * (2.0 * N + 1.0);
    const double dt_adv = s->cfl * (2.0 / ((N + 1) * la));
    const double dt_visc = s->cfl / ((lq + lv * k) * k);
    double dt = s->fixed_dt > 0.0 ? s->fixed_dt : fmin(dt_adv, dt_visc);
    const double t = s->t, te = s->t_end;
    const bool finished = run_finished(t, te);
    if (finished) dt = 0.0;
    else if (t + dt > te) dt = te - t;
    s->dt = dt;
    s->t = finished ? t : t + dt;
    if (!finished) s->steps += 1;
    s->max_bits = 0ull;
    visc_bits[0] = 0ull;
    if (curved) visc_bits[1] = 0ull;
}

}  // namespace tlw
