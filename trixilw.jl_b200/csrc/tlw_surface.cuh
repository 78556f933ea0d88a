// tlw_surface.cuh -- interface and boundary LW fluxes fused with the weak-form surface lift and the
// Jacobian (FP64, sm_100a), plus the CFL time-step reduction.
//
// Restates (TreeMesh{2}):
//   prolong2interfaces!   src/solvers/dgsem_tree/dg_2d.jl:1269-1326 (traces read where they lie)
//   calc_interface_flux!  src/solvers/dgsem_tree/dg_2d.jl:1903-1946 (plain FR: compute_alp = 0)
//   prolong2boundaries!   src/solvers/dgsem_tree/dg_2d.jl:1328-1376
//   calc_boundary_flux!   src/solvers/dgsem_tree/dg_2d.jl:1385-1454 + time-averaged Dirichlet
//                         src/equations/equations.jl:6-37
//   Trixi calc_surface_integral! (weak form: du[1] -= Fn/w_1, du[n] += Fn/w_n) and apply_jacobian!
//   (du *= -J^{-1}), folded into a read-modify-write of the face nodes only.
//   Trixi max_dt (TreeMesh{2}, CompressibleEulerEquations2D) * cfl, src/solvers/lwfr.jl:176-190, with
//   set_dt! clamping (src/solvers/lwfr.jl:76-90).
//
// One thread per (interface, face node). x- and y-oriented interfaces are launched separately: inside
// one orientation no two threads touch the same node, so the read-modify-writes need no atomics and
// the result is deterministic.
#pragma once
#include "tlw_device.cuh"

namespace tlw {

struct SurfArgs {
    const double* u;         // instantaneous state u^n (jumps)            [v,i,j,e]
    double* out;             // du (mode 0) or the updated state (mode 1)  [v,i,j,e]
    const double* tU;        // [v, l, face, e]
    const double* tF;        // [v, l, face, e]
    const int* left;         // interfaces of this orientation
    const int* right;
    int count;
    int orientation;         // 1 = x, 2 = y
    const double* inv_jac;
    const double* dt;
    int step_mode;           // 1: scale the lift by dt (state update)
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
    // shock capturing (compute_alp, src/solvers/dgsem_tree/dg_2d.jl:1879-1901)
    int shock_capturing;
    const double* alpha;     // [e]
    const double* tFn;       // first-order subcell flux next to each face [v, l, face, e]
    double jac_first;        // J^{-1} used by the admissibility test (element 1's on TreeMesh)
    double w_first, w_last;  // GLL weights w_1, w_n
    const int* inst;         // batched form: instance of each element (dt indexed by it); null otherwise
    const double* tFv;      // compressible Navier-Stokes: viscous normal flux traces (null otherwise)
    unsigned long long* cfl_slots;   // plain LW step: per-element CFL slots of the nodes finalised here
    const int* nbr;          // surface_kernel: the element across each face [4, e] (-x, +x, -y, +y)
    int E;                   // surface_kernel: number of elements
};

__device__ __forceinline__ bool admissible(double gm1, const double* u) {
    // is_admissible (src/equations/compressible_euler_2d.jl:4-7): rho > 0 and p > 0
    const double v1 = u[1] / u[0], v2 = u[2] / u[0];
    const double p = gm1 * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    return u[0] > 0.0 && p > 0.0;
}

// Fn <- alp fn + (1 - alp) Fn with compute_alp (dg_2d.jl:1879-1901, 1929-1937): fn is the first-order
// flux at the instantaneous u, alp = (alpha_L + alpha_R)/2, or 1 when the low-order update of either face
// subcell (subcell flux next to the face, fil / fir, lambda = 1/2) is not admissible. jac is the J^{-1} the
// reference takes for the test (element 1's on TreeMesh), wf / wl the GLL weights w_1 / w_n.
__device__ __forceinline__ void blend_flux_values(double gamma, int speed_kind, unsigned* status, double jac,
                                                  double wf, double wl, int orientation, const double* uL,
                                                  const double* uR, double alphaL, double alphaR, const double* fil,
                                                  const double* fir, double dt, double* Fn) {
    const double gm1 = gamma - 1.0;
    double fl[NV], fr[NV], fn[NV];
    euler_flux_dir(gm1, uL, orientation, fl);
    euler_flux_dir(gm1, uR, orientation, fr);
    const double lam = max_abs_speed(gamma, uL, uR, orientation, speed_kind, status);
#pragma unroll
    for (int v = 0; v < NV; ++v) fn[v] = 0.5 * (fl[v] + fr[v]) + (-0.5 * lam * (uR[v] - uL[v]));
    double alp = 0.5 * (alphaL + alphaR);
    double Fb[NV], low[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) Fb[v] = (1.0 - alp) * Fn[v] + alp * fn[v];
    const double lamx = 0.5;
#pragma unroll
    for (int v = 0; v < NV; ++v) low[v] = uL[v] - dt * jac / (wl * lamx) * (Fb[v] - fil[v]);
    if (!admissible(gm1, low)) {
        alp = 1.0;
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) low[v] = uR[v] - dt * jac / (wf * lamx) * (fir[v] - Fb[v]);
        if (!admissible(gm1, low)) alp = 1.0;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) Fn[v] = alp * fn[v] + (1.0 - alp) * Fn[v];
}

template <int N>
__device__ __forceinline__ void blend_interface_flux(const SurfArgs& a, int orientation, int le, int re, int faceL,
                                                     int faceR, int l, const double* uL, const double* uR, double dt,
                                                     double* Fn) {
    constexpr int n = N + 1;
    double fil[NV], fir[NV];
    load4(a.tFn + (((size_t)le * 4 + faceL) * n + l) * NV, fil);
    load4(a.tFn + (((size_t)re * 4 + faceR) * n + l) * NV, fir);
    blend_flux_values(a.gamma, a.speed_kind, a.status, a.jac_first, a.w_first, a.w_last, orientation, uL, uR,
                      __ldg(a.alpha + le), __ldg(a.alpha + re), fil, fir, dt, Fn);
}

// The LW flux at node l of the interface (le, re) of one orientation, with the blending and the viscous
// flux where they apply: calc_interface_flux! (dg_2d.jl:1903-1946) at one node.
// WIDE: 256-bit loads of the node records (the element-centric surface pass; 32-byte aligned arrays)
template <int N, bool SC = true, bool WIDE = false>
__device__ __forceinline__ void interface_node_flux(const SurfArgs& a, int orientation, int le, int re, int l,
                                                    double dt, double* Fn) {
    constexpr int n = N + 1;
    int nodeL, nodeR, faceL, faceR;
    if (orientation == 1) { nodeL = (n - 1) + n * l; nodeR = n * l; faceL = 1; faceR = 0; }
    else { nodeL = l + n * (n - 1); nodeR = l; faceL = 3; faceR = 2; }
    double uL[NV], uR[NV], UL[NV], UR[NV], FL[NV], FR[NV];
    auto ld = [](const double* p, double* x) {
        if (WIDE) load4w(p, x);
        else load4(p, x);
    };
    ld(a.u + ((size_t)le * n * n + nodeL) * NV, uL);
    ld(a.u + ((size_t)re * n * n + nodeR) * NV, uR);
    ld(a.tU + (((size_t)le * 4 + faceL) * n + l) * NV, UL);
    ld(a.tU + (((size_t)re * 4 + faceR) * n + l) * NV, UR);
    ld(a.tF + (((size_t)le * 4 + faceL) * n + l) * NV, FL);
    ld(a.tF + (((size_t)re * 4 + faceR) * n + l) * NV, FR);
    // TreeMesh argument order: surface_flux(f_ll, f_rr, U_ll, U_rr, u_ll, u_rr) (dg_2d.jl:1928)
    lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, FL, FR, UL, UR, uL, uR, orientation, Fn, a.status);
    if (SC && a.shock_capturing) blend_interface_flux<N>(a, orientation, le, re, faceL, faceR, l, uL, uR, dt, Fn);
    if (a.tFv) {
        // compressible Navier-Stokes: minus the central viscous flux (Fv_L + Fv_R) / 2
        double vL[NV], vR[NV];
        load4(a.tFv + (((size_t)le * 4 + faceL) * n + l) * NV, vL);
        load4(a.tFv + (((size_t)re * 4 + faceR) * n + l) * NV, vR);
#pragma unroll
        for (int v = 0; v < NV; ++v) Fn[v] -= 0.5 * (vL[v] + vR[v]);
    }
}

template <int N>
static __global__ void __launch_bounds__(256) interface_kernel(SurfArgs a) {
    constexpr int n = N + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n;
    const int l = t - k * n;
    if (k >= a.count) return;
    const int le = __ldg(a.left + k), re = __ldg(a.right + k);
    const int nodeL = a.orientation == 1 ? (n - 1) + n * l : l + n * (n - 1);
    const int nodeR = a.orientation == 1 ? n * l : l;
    const double dt = a.inst ? a.dt[__ldg(a.inst + le)] : *a.dt;
    double Fn[NV];
    interface_node_flux<N, true, true>(a, a.orientation, le, re, l, dt, Fn);
    const double dts = a.step_mode ? dt : 1.0;
    const double sL = -__ldg(a.inv_jac + le) * a.inv_w_last * dts;
    const double sR = __ldg(a.inv_jac + re) * a.inv_w_first * dts;
    double* oL = a.out + ((size_t)le * n * n + nodeL) * NV;
    double* oR = a.out + ((size_t)re * n * n + nodeR) * NV;
    // x faces finalise their non-corner nodes, y faces all of theirs (the y launch runs after the x launch)
    const bool slots = a.cfl_slots && (a.orientation == 2 || (l > 0 && l < n - 1));
    const int sL_slot = a.orientation == 1 ? 2 : 4, sR_slot = a.orientation == 1 ? 1 : 3;
    double x[NV], l1, l2;
    load4w_rw(oL, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(sL, Fn[v], x[v]);
    store4w(oL, x);
    if (slots) {
        node_speeds(a.gamma, x, a.status, l1, l2);
        atomicMax(a.cfl_slots + (size_t)le * CFL_SLOTS + 2 * sL_slot, (unsigned long long)__double_as_longlong(l1));
        atomicMax(a.cfl_slots + (size_t)le * CFL_SLOTS + 2 * sL_slot + 1, (unsigned long long)__double_as_longlong(l2));
    }
    load4w_rw(oR, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(sR, Fn[v], x[v]);
    store4w(oR, x);
    if (slots) {
        node_speeds(a.gamma, x, a.status, l1, l2);
        atomicMax(a.cfl_slots + (size_t)re * CFL_SLOTS + 2 * sR_slot, (unsigned long long)__double_as_longlong(l1));
        atomicMax(a.cfl_slots + (size_t)re * CFL_SLOTS + 2 * sR_slot + 1, (unsigned long long)__double_as_longlong(l2));
    }
}

struct BndArgs {
    const double* u;
    double* out;
    const double* tU;
    const double* tF;
    const int* bidx;         // boundaries of this orientation (0-based ids into the arrays below)
    const int* element;      // [B] element of each boundary
    const int* direction;    // [B] Trixi direction 1..4 (1: -x face of the element, 2: +x, 3: -y, 4: +y)
    const double* levels;    // exterior state at the n time levels [v, q, l, B]
    const double* now;       // exterior state at t                 [v, l, B]
    int count;
    int orientation;
    const double* inv_jac;
    const double* dt;
    int step_mode;
    double scaling_factor;   // 1, or 0.5 for MDRK stage 1 (multi_derivative_2d.jl:34)
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    const double* weights;   // GLL weights (device)
    unsigned* status;
    const int* kind;         // [B] BC_* per boundary, or null (all Dirichlet)
    // compressible Navier-Stokes walls: the viscous normal flux traces, the wall kind and data [3, l, B]
    const double* tFv;       // or null
    const int* wall_kind;
    const double* wall;
};

// boundary conditions of the advective part (the parabolic walls are WALL_*)
constexpr int BC_DIRICHLET = 0, BC_SLIP_WALL_VERTICAL = 1, BC_SLIP_WALL_HORIZONTAL = 2;
constexpr int WALL_NONE = 0, WALL_ADIABATIC = 1, WALL_ISOTHERMAL = 2;

// boundary_condition_slip_wall_vertical / _horizontal (src/equations/equations.jl:95-135): the exterior
// normal flux, U and u are the inner ones mirrored in the wall's normal momentum
__device__ __forceinline__ void slip_wall_exterior(int kind, const double* Fi, const double* Ui, const double* ui,
                                                   double* Fo, double* Uo, double* uo) {
    const bool vert = kind == BC_SLIP_WALL_VERTICAL;
    Fo[0] = -Fi[0]; Fo[1] = vert ? Fi[1] : -Fi[1]; Fo[2] = vert ? -Fi[2] : Fi[2]; Fo[3] = -Fi[3];
    Uo[0] = Ui[0]; Uo[1] = vert ? -Ui[1] : Ui[1]; Uo[2] = vert ? Ui[2] : -Ui[2]; Uo[3] = Ui[3];
    uo[0] = ui[0]; uo[1] = vert ? -ui[1] : ui[1]; uo[2] = vert ? ui[2] : -ui[2]; uo[3] = ui[3];
}

// The LW flux at node l of boundary k (element e, Trixi direction dir): calc_boundary_flux! (dg_2d.jl:1385-1454)
// with the time-averaged Dirichlet data or a slip wall, and the Navier-Stokes wall's viscous flux.
template <int N>
__device__ __forceinline__ void boundary_node_flux(const BndArgs& a, int k, int e, int dir, int l, double* Fn) {
    constexpr int n = N + 1;
    const int orientation = dir <= 2 ? 1 : 2;
    int node, face;
    switch (dir) {
        case 1: node = n * l; face = 0; break;
        case 2: node = (n - 1) + n * l; face = 1; break;
        case 3: node = l; face = 2; break;
        default: node = l + n * (n - 1); face = 3; break;
    }
    const double gm1 = a.gamma - 1.0;
    double ui[NV], Ui[NV], Fi[NV], Uo[NV] = {0, 0, 0, 0}, Fo[NV] = {0, 0, 0, 0}, uo[NV];
    load4(a.u + ((size_t)e * n * n + node) * NV, ui);
    load4(a.tU + (((size_t)e * 4 + face) * n + l) * NV, Ui);
    load4(a.tF + (((size_t)e * 4 + face) * n + l) * NV, Fi);
    const int kind = a.kind ? __ldg(a.kind + k) : BC_DIRICHLET;
    if (kind == BC_DIRICHLET) {
        for (int q = 0; q < n; ++q) {
            double ub[NV], fb[NV];
            load4(a.levels + (((size_t)k * n + l) * n + q) * NV, ub);
            euler_flux_dir(gm1, ub, orientation, fb);
            const double w = 0.5 * a.scaling_factor;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                Uo[v] += w * ub[v] * a.weights[q];
                Fo[v] += w * fb[v] * a.weights[q];
            }
        }
        load4(a.now + ((size_t)k * n + l) * NV, uo);
    } else {
        slip_wall_exterior(kind, Fi, Ui, ui, Fo, Uo, uo);
    }
    if (dir % 2 == 0)
        lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, Fi, Fo, Ui, Uo, ui, uo, orientation, Fn, a.status);
    else
        lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, Fo, Fi, Uo, Ui, uo, ui, orientation, Fn, a.status);
    if (a.tFv) {
        // minus the wall's viscous flux (calc_boundary_flux_divergence_lw!, dg_2d_parabolic.jl:2005-2084;
        // BoundaryConditionNavierStokesWall, compressible_navier_stokes_2d.jl:81-108)
        double fv[NV];
        load4(a.tFv + (((size_t)e * 4 + face) * n + l) * NV, fv);
        if (__ldg(a.wall_kind + k) == WALL_ADIABATIC) {
            const double* w = a.wall + 3 * ((size_t)k * n + l);
            fv[3] = fma(__ldg(w), fv[1], fma(__ldg(w + 1), fv[2], __ldg(w + 2)));
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) Fn[v] -= fv[v];
    }
}

template <int N>
static __global__ void __launch_bounds__(128) boundary_kernel(BndArgs a) {
    constexpr int n = N + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int kk = t / n;
    const int l = t - kk * n;
    if (kk >= a.count) return;
    const int k = __ldg(a.bidx + kk);
    const int e = __ldg(a.element + k);
    const int dir = __ldg(a.direction + k);
    const int node = dir == 1 ? n * l : dir == 2 ? (n - 1) + n * l : dir == 3 ? l : l + n * (n - 1);
    double Fn[NV];
    boundary_node_flux<N>(a, k, e, dir, l, Fn);
    const double dts = a.step_mode ? *a.dt : 1.0;
    const double ij = __ldg(a.inv_jac + e);
    const double s = (dir % 2 == 0) ? -ij * a.inv_w_last * dts : ij * a.inv_w_first * dts;
    double* o = a.out + ((size_t)e * n * n + node) * NV;
    double x[NV];
    load4_rw(o, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(s, Fn[v], x[v]);
    store4(o, x);
}

// surface_kernel launch shape: about TLW_SURF_THREADS threads a CTA (4n flux threads per element); the plain
// kernel (no boundaries, no blending) capped to TLW_SURF_MINB resident CTAs' registers when the CTA has at most
// 128 threads (7 x 128 threads: 72 registers, no spills), 5 otherwise; TLW_SURF_PREFETCH 1 loads the output face
// node before the flux phase (more registers). Measured on the 512 x 512, N = 4 vortex with one 256-bit access
// per node record: 0.1836 ms with (120, 7, 0), 0.187 ms with (160, 5, 0), 0.1996 ms with (120, 6, 0); before
// the wide accesses: 0.205 ms with (160, 5, 0), 0.232 ms with (160, 1, 1) at 90 registers, 0.236 ms with
// (320, 3, 0) and (240, 3, 0), 0.216 ms with (120, 6, 0), 0.224 ms with (160, 6, 0); an asynchronous copy of the
// output face nodes into shared memory during the flux phase: 0.222 ms. The x / y sweeps took 0.236 ms.
#ifndef TLW_SURF_THREADS
#define TLW_SURF_THREADS 120
#endif
#ifndef TLW_SURF_MINB
#define TLW_SURF_MINB 7
#endif
#ifndef TLW_SURF_PREFETCH
#define TLW_SURF_PREFETCH 0
#endif
#ifndef TLW_SURF_REVERSE
#define TLW_SURF_REVERSE 1
#endif
// Elements per CTA of surface_kernel: 4n flux threads per element, about TLW_SURF_THREADS threads a CTA.
template <int N> struct SurfCfg {
    static constexpr int n = N + 1;
    static constexpr int EB = (TLW_SURF_THREADS + 4 * n - 1) / (4 * n);
    // whole warps (the face-node maxima are reduced by warp shuffles over full masks)
    static constexpr int THREADS = (EB * 4 * n + 31) / 32 * 32;
    static constexpr int MIN_BLOCKS = THREADS <= 128 ? TLW_SURF_MINB : 5;
};

// All four faces of each element in one pass, for a mesh whose every face is a conforming interface or a
// boundary: nbr[4e + f] (f = -x, +x, -y, +y) is the element across face f, or -(k + 1) for boundary k of the
// boundary arguments. Phase 1: one thread per (element, face, node) evaluates that face's flux exactly as
// interface_kernel / boundary_kernel do (an interface with its own (left, right) arguments, so both elements get
// the same bits) into shared memory. Phase 2: one thread per face node of the element applies the x face's lift
// and then the y face's (the order of the x and y launches), with the Jacobian and dt, and reduces the element's
// face-node CFL speeds. Each interface is evaluated twice and each element's face nodes are read and written once:
// no strided x sweep, no atomics.
#ifndef TLW_SURF_MINB_SC
#define TLW_SURF_MINB_SC 1
#endif
template <int N, bool BND, bool SC>
static __global__ void __launch_bounds__(SurfCfg<N>::THREADS, (BND || SC) ? TLW_SURF_MINB_SC : SurfCfg<N>::MIN_BLOCKS)
    surface_kernel(SurfArgs a, BndArgs bnd) {
    using C = SurfCfg<N>;
    constexpr int n = N + 1, EB = C::EB, NB = 4 * (n - 1);
    __shared__ double sF[EB * 4 * n * NV];
    const int tid = threadIdx.x;
    // TLW_SURF_REVERSE: the CTAs take the elements from the last one down, so that the first ones read the traces
    // and face nodes the volume kernel wrote last (still in L2), and the next volume kernel, which starts from the
    // first element, finds the face nodes written last (512^2, N = 4: 0.2034 against 0.2051 ms a launch, LW step
    // 0.7145 against 0.7173 ms, MDRK step 0.978 against 0.983 ms)
    const int e0 = (TLW_SURF_REVERSE ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x) * EB;
    // phase-2 thread: element el2, boundary node b (bottom row, top row, left column, right column)
    const int el2 = tid / NB, b = tid - el2 * NB, e2 = e0 + el2;
    const bool has2 = el2 < EB && e2 < a.E;
    int i2, j2;
    if (b < n) { i2 = b; j2 = 0; }
    else if (b < 2 * n) { i2 = b - n; j2 = n - 1; }
    else if (b < 3 * n - 2) { i2 = 0; j2 = b - 2 * n + 1; }
    else { i2 = n - 1; j2 = b - 3 * n + 3; }
    double* o2 = a.out + ((size_t)e2 * n * n + i2 + n * j2) * NV;
    double x[NV];
    if (TLW_SURF_PREFETCH && has2) load4w_rw(o2, x);
    {
        const int el = tid / (4 * n), r = tid - el * 4 * n, f = r / n, l = r - f * n, e = e0 + el;
        if (el < EB && e < a.E) {
            const double dt = a.inst ? a.dt[__ldg(a.inst + e)] : *a.dt;   // (batched form: the instance's dt)
            const int nb = __ldg(a.nbr + 4 * e + f);
            const bool plus = f & 1;   // this element is the interface's left (lower) element
            double Fn[NV];
            if (!BND || nb >= 0)
                interface_node_flux<N, SC, true>(a, f < 2 ? 1 : 2, plus ? e : nb, plus ? nb : e, l, dt, Fn);
            else boundary_node_flux<N>(bnd, -nb - 1, e, f + 1, l, Fn);
#pragma unroll
            for (int v = 0; v < NV; ++v) sF[tid * NV + v] = Fn[v];
        }
    }
    __syncthreads();
    double l1 = 0.0, l2 = 0.0;
    if (has2) {
        if (!TLW_SURF_PREFETCH) load4w_rw(o2, x);
        const double dt = a.inst ? a.dt[__ldg(a.inst + e2)] : *a.dt;
        const double dts = a.step_mode ? dt : 1.0;
        const double ij = __ldg(a.inv_jac + e2);
        const double sMinus = ij * a.inv_w_first * dts;   // the element is the right (upper) one of the interface
        const double sPlus = -ij * a.inv_w_last * dts;    // the element is the left (lower) one
        const double* F = sF + el2 * 4 * n * NV;
        if (i2 == 0 || i2 == n - 1) {
            const double s = i2 == 0 ? sMinus : sPlus;
            const double* p = F + ((i2 == 0 ? 0 : 1) * n + j2) * NV;
#pragma unroll
            for (int v = 0; v < NV; ++v) x[v] = fma(s, p[v], x[v]);
        }
        if (j2 == 0 || j2 == n - 1) {
            const double s = j2 == 0 ? sMinus : sPlus;
            const double* p = F + ((j2 == 0 ? 2 : 3) * n + i2) * NV;
#pragma unroll
            for (int v = 0; v < NV; ++v) x[v] = fma(s, p[v], x[v]);
        }
        store4w(o2, x);
        if (a.cfl_slots) node_speeds(a.gamma, x, a.status, l1, l2);
    }
    if (a.cfl_slots && 32 % NB == 0) {
        // the element's NB phase-2 threads are NB aligned consecutive lanes of one warp: reduce by shuffles
#pragma unroll
        for (int o = NB / 2; o > 0; o >>= 1) {
            l1 = fmax(l1, __shfl_xor_sync(0xffffffffu, l1, o));
            l2 = fmax(l2, __shfl_xor_sync(0xffffffffu, l2, o));
        }
        if (has2 && b < 2)
            a.cfl_slots[(size_t)e2 * CFL_SLOTS + 2 + b] = (unsigned long long)__double_as_longlong(b ? l2 : l1);
    } else if (a.cfl_slots) {
        // the element's face-node maxima through shared memory (NB consecutive threads per element)
        __syncthreads();
        if (has2) {
            sF[tid] = l1;
            sF[EB * NB + tid] = l2;
        }
        __syncthreads();
        if (has2 && b < 2) {
            const double* p = sF + b * EB * NB + el2 * NB;
            double m = 0.0;
#pragma unroll
            for (int k = 0; k < NB; ++k) m = fmax(m, p[k]);
            a.cfl_slots[(size_t)e2 * CFL_SLOTS + 2 + b] = (unsigned long long)__double_as_longlong(m);
        }
    }
}


// ------------------------------------------------------------------------------------------------
// CFL time step on the device.
// ------------------------------------------------------------------------------------------------
struct StepState {
    unsigned long long max_bits;   // bits of max_e J^{-1}(lambda1 + lambda2) (non-negative doubles order as ints)
    double dt;                     // time step used by the current step
    double t;                      // time at the start of the next step
    double t_end;
    double cfl;
    double fixed_dt;               // > 0: use this dt instead of the CFL estimate
    long long steps;               // accepted steps
    unsigned status;               // STATUS_* bits
    int pad;
    double dt_call;                // dt for the rhs entry points (set from the host)
    double t_step;                 // time at the start of the current step (source terms)
    double t_call;                 // t of the rhs entry points (set from the host; source terms)
};

constexpr int MS_THREADS = 256;
template <int N>
struct MsCfg {
    static constexpr int n = N + 1, nn = n * n;
    static constexpr int ELEMS = N >= 6 ? 16 : 32;   // elements per CTA (shared memory: 4 x ELEMS x nn doubles)
};

struct IndicatorArgs {
    double* alpha_raw;       // [e] indicator before smoothing
    double* alpha;           // [e] blending factor (smoothed afterwards)
    double alpha_max, alpha_min, threshold, parameter_s;
    // curvilinear meshes: the CFL speeds of the same pass take the node's metrics and J^{-1} (null on a TreeMesh)
    const double* metrics;
    const double* inv_jac_node;
};

// One pass over u for the CFL reduction (SPEED) and/or the Hennemann-Gassner indicator (IND).
// The CTA reads its elements' nodes in order (coalesced 32-byte node records) into shared memory.
//  SPEED: per element max over nodes of |v1|+c and |v2|+c, times J^{-1}; max over elements (atomic).
//  IND:   Trixi IndicatorHennemannGassner with variable density_pressure: modal = Vinv ind Vinv^T by
//         eight threads per element (constant-memory Vinv), energy fractions of the highest modes,
//         logistic map, alpha_min / alpha_max clipping (Hennemann et al., J. Comput. Phys. 426 (2021)).
// batched form: per-instance maxima instead of the single StepState one
struct BatchSpeedArgs {
    const int* inst;                // instance of each element, or null
    unsigned long long* inst_max;   // [instance] bits of the max scaled speed
};

// CSPEED (curvilinear meshes): the speeds of curved_max_speed_kernel, |Ja^d . (l1, l2)| |J^{-1}| per node, and the
// element's value max l1 + max l2 without the element J^{-1}
template <int N, bool SPEED, bool IND, bool CSPEED = false>
static __global__ void __launch_bounds__(MS_THREADS) max_speed_kernel(const double* __restrict__ u,
                                                               const double* __restrict__ inv_jac, int E,
                                                               double gamma, StepState* s, IndicatorArgs ia,
                                                               BatchSpeedArgs bs) {
    constexpr int n = N + 1;
    constexpr int nn = n * n;
    constexpr int ELEMS = MsCfg<N>::ELEMS;
    __shared__ double l1s[SPEED ? ELEMS * nn : 1], l2s[SPEED ? ELEMS * nn : 1];
    __shared__ double inds[IND ? ELEMS * nn : 1], tmps[IND ? ELEMS * nn : 1];
    __shared__ double wmax[MS_THREADS / 32];
    const int e0 = blockIdx.x * ELEMS;
    const int ne = min(ELEMS, E - e0);
    const double gm1 = gamma - 1.0;
    for (int k = threadIdx.x; k < ne * nn; k += MS_THREADS) {
        double x[NV];
        load4w(u + ((size_t)e0 * nn + k) * NV, x);
        if (SPEED && CSPEED) {
            const size_t node = (size_t)e0 * nn + k;
            double J[4], l1, l2;
            load4w(ia.metrics + node * 4, J);
            node_speeds(gamma, x, &s->status, l1, l2);
            const double ij = fabs(__ldg(ia.inv_jac_node + node));
            l1s[k] = fabs(J[0] * l1 + J[1] * l2) * ij;
            l2s[k] = fabs(J[2] * l1 + J[3] * l2) * ij;
        } else if (SPEED) {
            node_speeds(gamma, x, &s->status, l1s[k], l2s[k]);
        }
        // indicator variable density_pressure = (gamma - 1)(rho rho_e - |rho v|^2 / 2)
        if (IND) inds[k] = gm1 * (x[0] * x[3] - 0.5 * (x[1] * x[1] + x[2] * x[2]));
    }
    __syncthreads();
    double m = 0.0;
    if (SPEED && threadIdx.x < ne) {
        double ml1 = 0.0, ml2 = 0.0;
        for (int k = 0; k < nn; ++k) {
            ml1 = fmax(ml1, l1s[threadIdx.x * nn + k]);
            ml2 = fmax(ml2, l2s[threadIdx.x * nn + k]);
        }
        m = CSPEED ? ml1 + ml2 : __ldg(inv_jac + e0 + threadIdx.x) * (ml1 + ml2);
    }
    if (IND) {
        const int el = threadIdx.x >> 3, q = threadIdx.x & 7;
        const double* Vi = c_tlw_Vinv[N];
        // tmp = Vinv ind (column q of the element)
        if (el < ne && q < n) {
#pragma unroll
            for (int i = 0; i < n; ++i) {
                double r = 0.0;
#pragma unroll
                for (int a = 0; a < n; ++a) r += Vi[i * n + a] * inds[el * nn + a + n * q];
                tmps[el * nn + i + n * q] = r;
            }
        }
        __syncthreads();
        // modal row q: modal[q][j] = sum_c Vinv[j][c] tmp[q][c]; partial energies of the three sums
        double tot = 0.0, c1 = 0.0, c2 = 0.0;
        if (el < ne && q < n) {
#pragma unroll
            for (int j = 0; j < n; ++j) {
                double r = 0.0;
#pragma unroll
                for (int c = 0; c < n; ++c) r += Vi[j * n + c] * tmps[el * nn + q + n * c];
                const double r2 = r * r;
                tot += r2;
                if (q < n - 1 && j < n - 1) c1 += r2;
                if (q < n - 2 && j < n - 2) c2 += r2;
            }
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
            c1 += __shfl_xor_sync(0xffffffffu, c1, o);
            c2 += __shfl_xor_sync(0xffffffffu, c2, o);
        }
        if (el < ne && q == 0) {
            const double f1 = tot != 0.0 ? (tot - c1) / tot : 0.0;
            const double f2 = c1 != 0.0 ? (c1 - c2) / c1 : 0.0;
            const double energy = fmax(f1, f2);
            double al = 1.0 / (1.0 + exp(-ia.parameter_s / ia.threshold * (energy - ia.threshold)));
            if (al < ia.alpha_min) al = 0.0;
            if (al > 1.0 - ia.alpha_min) al = 1.0;
            al = fmin(ia.alpha_max, al);
            ia.alpha_raw[e0 + el] = al;
            ia.alpha[e0 + el] = al;
        }
    }
    if (SPEED && bs.inst) {
        // batched: the (<= 32) element values sit in warp 0; one atomic per instance present
        if (threadIdx.x < 32) {
            const int last = min(ne, 32) - 1;
            const int my = threadIdx.x <= last ? __ldg(bs.inst + e0 + threadIdx.x) : -1;
            const int first_inst = __shfl_sync(0xffffffffu, my, 0);
            const int last_inst = __shfl_sync(0xffffffffu, my, last);
            if (first_inst == last_inst) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
                if (threadIdx.x == 0 && m > 0.0)
                    atomicMax(bs.inst_max + first_inst, (unsigned long long)__double_as_longlong(m));
            } else if (threadIdx.x <= last && m > 0.0) {
                atomicMax(bs.inst_max + my, (unsigned long long)__double_as_longlong(m));
            }
        }
    } else if (SPEED) {
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
}

// batched form: dt of every instance from its max scaled speed (finalize_dt_kernel per instance)
// isfinished: t ≈ t_end (src/solvers/lwfr.jl:146-148) with Julia's isapprox (rtol = sqrt(eps(Float64)),
// never true against an infinite t_end unless equal); t >= t_end cannot happen after the set_dt! clamp and
// only guards against an endless run.
__device__ __forceinline__ bool run_finished(double t, double te) {
    if (t == te) return true;
    if (!isfinite(t) || !isfinite(te)) return false;
    return fabs(t - te) <= 1.4901161193847656e-8 * fmax(fabs(t), fabs(te)) || t >= te;
}

struct BatchTime {
    unsigned long long* max_bits;
    double* dt;
    double* t;
    const double* t_end;
    const double* cfl;
    long long* steps;
    const int* nnodes;
    int count;
};

static __global__ void batch_finalize_dt_kernel(BatchTime b) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= b.count) return;
    double maxs = __longlong_as_double((long long)b.max_bits[k]);
    const double tiny = 4.9406564584124654e-324;
    if (!(maxs > tiny)) maxs = tiny;
    double dt = b.cfl[k] * (2.0 / (b.nnodes[k] * maxs));
    const double t = b.t[k], te = b.t_end[k];
    const bool finished = run_finished(t, te);
    if (finished) dt = 0.0;
    else if (t + dt > te) dt = te - t;
    b.dt[k] = dt;
    b.t[k] = finished ? t : t + dt;
    if (!finished) b.steps[k] += 1;
    b.max_bits[k] = 0ull;
}

// Trixi apply_smoothing! (TreeMesh{2}): alpha_e = max(alpha_e, alpha_raw_nb / 2) over the interfaces,
// independent of the order (max over non-negative doubles = max over their bit patterns)
static __global__ void alpha_smooth_kernel(const int* __restrict__ left, const int* __restrict__ right, int count,
                                    const double* __restrict__ alpha_raw, double* alpha) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int l = __ldg(left + k), r = __ldg(right + k);
    unsigned long long* ab = reinterpret_cast<unsigned long long*>(alpha);
    atomicMax(ab + l, (unsigned long long)__double_as_longlong(0.5 * __ldg(alpha_raw + r)));
    atomicMax(ab + r, (unsigned long long)__double_as_longlong(0.5 * __ldg(alpha_raw + l)));
}

// dt = cfl * 2 / (n * max_scaled_speed), clamped so that t + dt <= t_end; a finished run gets dt = 0
// (the remaining launches of a captured step are then exact no-ops on the state).
static __global__ void finalize_dt_kernel(StepState* s, int n) {
    double maxs = __longlong_as_double((long long)s->max_bits);
    const double tiny = 4.9406564584124654e-324;   // nextfloat(0.0)
    if (!(maxs > tiny)) maxs = tiny;
    double dt = s->fixed_dt > 0.0 ? s->fixed_dt : s->cfl * (2.0 / (n * maxs));
    const double t = s->t, te = s->t_end;
    const bool finished = run_finished(t, te);
    if (finished) dt = 0.0;
    else if (t + dt > te) dt = te - t;
    s->t_step = t;
    s->dt = dt;
    s->t = finished ? t : t + dt;
    if (!finished) s->steps += 1;
    s->max_bits = 0ull;
}

// the next step's CFL maximum from the per-element slots: max_e J^{-1} (max_s l1 + max_s l2)
static __global__ void __launch_bounds__(256) cfl_slots_reduce_kernel(const unsigned long long* __restrict__ slots,
                                                                      const double* __restrict__ inv_jac, int E,
                                                                      StepState* s) {
    __shared__ double wmax[8];
    double m = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        const unsigned long long* sl = slots + (size_t)e * CFL_SLOTS;
        unsigned long long b1 = 0ull, b2 = 0ull;
#pragma unroll
        for (int k = 0; k < CFL_SLOTS / 2; ++k) {
            b1 = max(b1, __ldg(sl + 2 * k));
            b2 = max(b2, __ldg(sl + 2 * k + 1));
        }
        m = fmax(m, __ldg(inv_jac + e) * (__longlong_as_double((long long)b1) + __longlong_as_double((long long)b2)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmax[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, wmax[w]);
        if (b > 0.0) atomicMax(&s->max_bits, (unsigned long long)__double_as_longlong(b));
    }
}


// Adaptive step control: partial sums of the per-element temporal errors (fixed order within a block) and
// admissibility (is_admissible, src/equations/compressible_euler_2d.jl:4-7) of every node of the trial state
static __global__ void __launch_bounds__(256) adaptive_check_kernel(const double* __restrict__ te, int E,
                                                                    const double* __restrict__ u, long long nodes,
                                                                    double gamma, double* partial, unsigned* bad) {
    __shared__ double red[256];
    double s = 0.0;
    for (int e = blockIdx.x * 256 + threadIdx.x; e < E; e += gridDim.x * 256) s += te[e];
    red[threadIdx.x] = s;
    bool ok = true;
    for (long long k = (long long)blockIdx.x * 256 + threadIdx.x; k < nodes; k += (long long)gridDim.x * 256) {
        double x[NV];
        load4(u + k * NV, x);
        const double v1 = x[1] / x[0], v2 = x[2] / x[0];
        const double p = (gamma - 1.0) * (x[3] - 0.5 * (x[1] * v1 + x[2] * v2));
        ok = ok && x[0] > 0.0 && p > 0.0;
    }
    if (!ok) atomicOr(bad, 1u);
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

static __global__ void adaptive_sum_kernel(const double* partial, int count, double* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < count; ++k) s += partial[k];
        *out = s;
    }
}

// accept the trial step: t += dt, one more accepted step
static __global__ void adaptive_accept_kernel(StepState* s, double dt) {
    s->dt = dt;
    s->t += dt;
    s->steps += 1;
}

// The controller of perform_step!(..., ::Adaptive, ::LW) (src/solvers/adaptive.jl:101-172) on the device, so
// that trials run back to back without a host round trip: the epsilon history of load_temporal_errors!
// (:47-61; shifted only on the first try of a step, a non-finite error keeps the previous estimate),
// dt_factor (:100-105) with the controller (beta1, beta2, beta3) of lwfr.jl:162, rejection when the trial is
// not admissible or factor <= 0.81 (retry at min(factor, 0.95) dt), acceptance otherwise (next dt
// min(factor, 1.5) dt), both clamped by set_dt! to end at t_end. The reference retries without a limit; here a
// run whose next dt falls to ADAPTIVE_DT_FLOOR |t| or below (t + dt no longer moves t) stops as stalled, and the
// host reports it as a non-admissible state instead of enqueuing trials for ever.
constexpr double ADAPTIVE_DT_FLOOR = 1e-14;
struct AdaptiveState {
    double eps[3];          // epsilon[-1], epsilon[0], epsilon[1]
    double beta[3];
    double dt;              // dt of the next trial
    double t_end;
    double k;               // nnodes
    double ndofs;
    double factor;
    long long n_fail, nreject, trials;
    int accept;             // the last trial was accepted
    int finished;
    int stalled;            // dt fell to the floor after repeated rejections: no further trials
};

__device__ __forceinline__ bool adaptive_finished(double t, double te) {
    // isapprox(t, t_end) with the default rtol sqrt(eps(Float64))
    return t == te || fabs(t - te) <= 1.4901161193847656e-08 * fmax(fabs(t), fabs(te));
}

static __global__ void adaptive_prepare_kernel(StepState* s, AdaptiveState* a) {
    a->finished = (a->stalled || adaptive_finished(s->t, a->t_end)) ? 1 : 0;
    s->dt_call = a->finished ? 0.0 : a->dt;
}

static __global__ void adaptive_judge_kernel(StepState* s, AdaptiveState* a, const double* sum, unsigned* bad) {
    a->accept = 0;
    const bool ok = *bad == 0 && s->status == 0;
    *bad = 0;
    s->status = 0;   // test_rhs! catches the DomainError: the trial is only inadmissible
    if (a->finished) return;
    const double err = sqrt(*sum / a->ndofs);
    if (a->n_fail == 0) {
        a->eps[0] = a->eps[1];
        a->eps[1] = a->eps[2];
    }
    if (isfinite(err)) a->eps[2] = 1.0 / (err + 1e-12);
    const double f = pow(a->eps[2], a->beta[0] / a->k) * pow(a->eps[1], a->beta[1] / a->k) *
                     pow(a->eps[0], a->beta[2] / a->k);
    const double factor = 1.0 + atan(f - 1.0);
    a->factor = factor;
    a->trials += 1;
    double nd;
    if (ok && !(factor <= 0.81)) {
        a->nreject += a->n_fail;
        a->n_fail = 0;
        s->dt = a->dt;
        s->t += a->dt;
        s->steps += 1;
        a->accept = 1;
        nd = fmin(factor, 1.5) * a->dt;
    } else {
        a->n_fail += 1;
        nd = fmin(factor, 0.95) * a->dt;
    }
    a->dt = s->t + nd > a->t_end ? a->t_end - s->t : nd;
    if (!(a->dt > ADAPTIVE_DT_FLOOR * fmax(fabs(s->t), fabs(a->t_end))) && !adaptive_finished(s->t, a->t_end))
        a->stalled = 1;
}

// an accepted trial becomes the current state
static __global__ void __launch_bounds__(256) adaptive_commit_kernel(const AdaptiveState* a, const double* __restrict__ trial,
                                                                     double* __restrict__ u, long long count) {
    if (!a->accept) return;
    for (long long k = (long long)blockIdx.x * 256 + threadIdx.x; k < count; k += (long long)gridDim.x * 256)
        u[k] = trial[k];
}

}  // namespace tlw
