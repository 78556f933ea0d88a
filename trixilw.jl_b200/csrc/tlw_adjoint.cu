// tlw_adjoint.cu -- the differentiable form: a hand-written discrete adjoint (vector-Jacobian product) of
// the full Lax-Wendroff step on a periodic TreeMesh{2}, and a checkpointed reverse sweep over a whole run.
//
// What is differentiated is the forward map of one step at a fixed dt,
//   u_new = u + dt * rhs(u)    (src/solvers/dgsem_tree/dg_2d.jl:28-83, perform_step! src/solvers/lwfr.jl:212-230)
// with the LW volume procedure of depth 3 (N = 3, dg_2d.jl:674-916) or 4 (N >= 4, dg_2d.jl:918-1267), the
// Rusanov interface flux in the TreeMesh argument order (dg_2d.jl:1903-1946: speed from the time-averaged
// U, jump in the instantaneous u), the weak-form surface lift and apply_jacobian. The reference has no
// adjoint; the step sizes of the forward run are recorded and held fixed in the reverse sweep, so the
// gradient is that of the discrete solution map at the recorded dt sequence.
//
// Notation: d_1 = ut, d_2 = utt, ... are the dt-scaled time derivatives; C(x, y) = -dt J^{-1} (D x + D y)
// produces the next one from the stage fluxes; the perturbed states of stage s are P_q = u + sum_{m<=s}
// a[q][m] d_m, q in {-, +, --, ++}; ft_s = w_s[0] f(u) + sum_q w_s[q] f(P_q); the time averages are
// F = f(u) + sum_s tw_s ft_s and U = u + sum_s tw_s d_s.
//
// Kernels (one adjoint step = two launches after a forward recompute that leaves the U traces):
//   adj_interface_kernel<N>: per interface node, the adjoint of Fn = (F_L + F_R)/2 - lambda(U_L, U_R) (u_R - u_L)/2
//     with the lift weights and -dt J^{-1}: adjoint face traces of F, U and u for both elements.
//   adj_volume_kernel<N>: per element (one thread per node), recomputes d_1..d_depth, then runs the LW
//     procedure backwards with the Euler flux Jacobians transposed at every perturbed state, the transposed
//     contractions through shared memory, and writes lam_out = lam_in + (du_new/du)^T lam_in.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tlw.h"
#include "tlw_basis.h"
#include "tlw_handle.h"
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"

using namespace tlw;

namespace {

// The adjoint kernels read and write the library's own arrays (segment states and traces, the adjoint states, the
// face-trace adjoints), whose node records are 32-byte aligned: one 256-bit access per record.
#ifndef TLW_ADJ_WIDE
#define TLW_ADJ_WIDE 1
#endif
__device__ __forceinline__ void aload4(const double* p, double* x) {
    if (TLW_ADJ_WIDE) load4w(p, x);
    else load4(p, x);
}
__device__ __forceinline__ void astore4(double* p, const double* x) {
    if (TLW_ADJ_WIDE) store4w(p, x);
    else store4(p, x);
}

int afail(tlw_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

#define TLW_ACUDA(h, call)                                                                       \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return afail(h, TLW_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

// ---- LW stencil constants (compile-time after unrolling) ------------------------------------------
template <int DEPTH>
struct LWC {
    // Taylor weight of stage s = 1..4
    static __device__ __forceinline__ constexpr double tw(int s) {
        return s == 1 ? 0.5 : s == 2 ? 1.0 / 6.0 : s == 3 ? 1.0 / 24.0 : 1.0 / 120.0;
    }
    // perturbation coefficient of d_m in state q (0: -, 1: +, 2: --, 3: ++)
    static __device__ __forceinline__ constexpr double a(int q, int m) {
        return q == 0 ? (m == 1 ? -1.0 : m == 2 ? 0.5 : m == 3 ? -1.0 / 6.0 : 1.0 / 24.0)
             : q == 1 ? (m == 1 ? 1.0 : m == 2 ? 0.5 : m == 3 ? 1.0 / 6.0 : 1.0 / 24.0)
             : q == 2 ? (m == 1 ? -2.0 : m == 2 ? 2.0 : m == 3 ? -4.0 / 3.0 : 2.0 / 3.0)
                      : (m == 1 ? 2.0 : m == 2 ? 2.0 : m == 3 ? 4.0 / 3.0 : 2.0 / 3.0);
    }
    // stencil weight of stage s: k = 0 -> f(u), k = 1 + q -> f(P_q)
    static __device__ __forceinline__ constexpr double w(int s, int k) {
        // stage 1: (-fpp + 8 fp - 8 fm + fmm) / 12
        return s == 1 ? (k == 0 ? 0.0 : k == 1 ? -8.0 / 12.0 : k == 2 ? 8.0 / 12.0 : k == 3 ? 1.0 / 12.0 : -1.0 / 12.0)
             // stage 2: depth 4 (-fpp + 16 fp - 30 f + 16 fm - fmm) / 12; depth 3 fp - 2 f + fm
             : s == 2 ? (DEPTH == 4 ? (k == 0 ? -30.0 / 12.0 : k <= 2 ? 16.0 / 12.0 : -1.0 / 12.0)
                                    : (k == 0 ? -2.0 : k <= 2 ? 1.0 : 0.0))
             // stage 3: (fpp - 2 fp + 2 fm - fmm) / 2
             : s == 3 ? (k == 0 ? 0.0 : k == 1 ? 1.0 : k == 2 ? -1.0 : k == 3 ? -0.5 : 0.5)
             // stage 4: (fpp - 4 fp + 6 f - 4 fm + fmm) / 2
                      : (k == 0 ? 3.0 : k <= 2 ? -2.0 : 0.5);
    }
};

// out += Jf(u)^T wf + Jg(u)^T wg for the Euler fluxes (conservative variables)
__device__ __forceinline__ void euler_flux_vjp(double gamma, const double* u, const double* wf, const double* wg,
                                               double* out) {
    const double gm1 = gamma - 1.0;
    const double ir = nr_reciprocal(u[0]);
    const double v1 = u[1] * ir, v2 = u[2] * ir;
    const double q = 0.5 * (v1 * v1 + v2 * v2);
    const double p = gm1 * (u[3] - u[0] * q);
    const double H = (u[3] + p) * ir;
    const double gq = gm1 * q, v12 = v1 * v2;
    out[0] += wf[1] * (gq - v1 * v1) - (wf[2] + wg[1]) * v12 + wf[3] * v1 * (gq - H) + wg[2] * (gq - v2 * v2) +
              wg[3] * v2 * (gq - H);
    out[1] += wf[0] + wf[1] * (2.0 - gm1) * v1 + wf[2] * v2 + wf[3] * (H - gm1 * v1 * v1) + wg[1] * v2 -
              wg[2] * gm1 * v1 - wg[3] * gm1 * v12;
    out[2] += -wf[1] * gm1 * v2 + wf[2] * v1 - wf[3] * gm1 * v12 + wg[0] + wg[1] * v1 + wg[2] * (2.0 - gm1) * v2 +
              wg[3] * (H - gm1 * v2 * v2);
    out[3] += (wf[1] + wg[2]) * gm1 + gamma * (wf[3] * v1 + wg[3] * v2);
}

// gradients of |v_d| and c = sqrt(gamma p / rho) with respect to the conservative state; returns |v_d|, c
__device__ __forceinline__ void speed_partials(double gamma, const double* u, int orientation, double* dv,
                                               double* dc, double* absv, double* c, unsigned* status) {
    const double gm1 = gamma - 1.0;
    const double ir = 1.0 / u[0];
    const double v1 = u[1] * ir, v2 = u[2] * ir;
    const double q = 0.5 * (v1 * v1 + v2 * v2);
    const double p = gm1 * (u[3] - 0.5 * (u[1] * v1 + u[2] * v2));
    const double cc = checked_sqrt(gamma * p * ir, status);
    const double vd = orientation == 1 ? v1 : v2;
    const double sg = (vd > 0.0) - (vd < 0.0);
    dv[0] = -sg * vd * ir;
    dv[1] = orientation == 1 ? sg * ir : 0.0;
    dv[2] = orientation == 2 ? sg * ir : 0.0;
    dv[3] = 0.0;
    const double k = gamma / (2.0 * cc * u[0]);
    dc[0] = k * (gm1 * q - p * ir);
    dc[1] = -k * gm1 * v1;
    dc[2] = -k * gm1 * v2;
    dc[3] = k * gm1;
    *absv = fabs(vd);
    *c = cc;
}

struct AdjSurfArgs {
    const double* u;        // state of the step [v, i, j, e]
    const double* tU;       // forward time-averaged U traces of the step [v, l, face, e]
    const double* lam;      // adjoint of u_new [v, i, j, e]
    double* bF;             // out: adjoint of the normal flux trace   [v, l, face, e]
    double* bU;             // out: adjoint of the U trace             [v, l, face, e]
    double* bu;             // out: direct adjoint of the u face value [v, l, face, e]
    const int *xl, *xr, *yl, *yr;
    int nx, ny;
    const double* inv_jac;
    const double* dt;
    double gamma;
    int speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
};

template <int N>
static __global__ void __launch_bounds__(128) adj_interface_kernel(AdjSurfArgs a) {
    constexpr int n = N + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int k = t / n;
    const int l = t - k * n;
    int orientation = 1;
    if (k >= a.nx) {
        k -= a.nx;
        orientation = 2;
        if (k >= a.ny) return;
    }
    const int le = orientation == 1 ? __ldg(a.xl + k) : __ldg(a.yl + k);
    const int re = orientation == 1 ? __ldg(a.xr + k) : __ldg(a.yr + k);
    int nodeL, nodeR, faceL, faceR;
    if (orientation == 1) { nodeL = (n - 1) + n * l; nodeR = n * l; faceL = 1; faceR = 0; }
    else { nodeL = l + n * (n - 1); nodeR = l; faceL = 3; faceR = 2; }
    double uL[NV], uR[NV], UL[NV], UR[NV], lL[NV], lR[NV];
    aload4(a.u + ((size_t)le * n * n + nodeL) * NV, uL);
    aload4(a.u + ((size_t)re * n * n + nodeR) * NV, uR);
    aload4(a.tU + (((size_t)le * 4 + faceL) * n + l) * NV, UL);
    aload4(a.tU + (((size_t)re * 4 + faceR) * n + l) * NV, UR);
    aload4(a.lam + ((size_t)le * n * n + nodeL) * NV, lL);
    aload4(a.lam + ((size_t)re * n * n + nodeR) * NV, lR);
    const double dt = *a.dt;
    const double sL = -dt * __ldg(a.inv_jac + le) * a.inv_w_last;
    const double sR = dt * __ldg(a.inv_jac + re) * a.inv_w_first;
    double bFn[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) bFn[v] = sL * lL[v] + sR * lR[v];
    double dvL[NV], dcL[NV], dvR[NV], dcR[NV], vl, cl, vr, cr;
    speed_partials(a.gamma, UL, orientation, dvL, dcL, &vl, &cl, a.status);
    speed_partials(a.gamma, UR, orientation, dvR, dcR, &vr, &cr, a.status);
    const double lambda = a.speed_kind == 0 ? fmax(vl, vr) + fmax(cl, cr) : fmax(vl + cl, vr + cr);
    double blam = 0.0;
    double o[NV];
    const size_t tl = (((size_t)le * 4 + faceL) * n + l) * NV, tr = (((size_t)re * 4 + faceR) * n + l) * NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        blam -= 0.5 * bFn[v] * (uR[v] - uL[v]);
        o[v] = 0.5 * bFn[v];
    }
    astore4(a.bF + tl, o);
    astore4(a.bF + tr, o);
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = 0.5 * lambda * bFn[v];
    astore4(a.bu + tl, o);
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = -o[v];
    astore4(a.bu + tr, o);
    // speed adjoint goes to the side whose |v| (and c) the max selected; the left argument wins ties
    double gL[NV], gR[NV];
    if (a.speed_kind == 0) {
        // max(|v_L|, |v_R|) + max(c_L, c_R)
        const double wvL = vl >= vr ? blam : 0.0, wvR = blam - wvL;
        const double wcL = cl >= cr ? blam : 0.0, wcR = blam - wcL;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            gL[v] = wvL * dvL[v] + wcL * dcL[v];
            gR[v] = wvR * dvR[v] + wcR * dcR[v];
        }
    } else {
        // max(|v_L| + c_L, |v_R| + c_R)
        const double wL = vl + cl >= vr + cr ? blam : 0.0, wR = blam - wL;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            gL[v] = wL * (dvL[v] + dcL[v]);
            gR[v] = wR * (dvR[v] + dcR[v]);
        }
    }
    astore4(a.bU + tl, gL);
    astore4(a.bU + tr, gR);
}

template <int N>
struct AdjCfg {
    static constexpr int n = N + 1;
    static constexpr int nn = n * n;
    static constexpr int EB = VolCfg<N>::EB;
    static constexpr int THREADS = VolCfg<N>::THREADS;
    static constexpr int DEPTH = N >= 4 ? 4 : 3;
    // resident CTAs per SM the register budget must allow (stage derivatives and their adjoints live in
    // shared memory, so the per-thread state is small)
    static constexpr int MIN_BLOCKS = THREADS <= 128 ? 3 : 1;
    // shared memory: D, Dhat, the two contraction tiles X, Y, the stage derivatives d_m and their adjoints
    static constexpr int TILE = NV * EB * nn;
    static constexpr size_t smem_bytes() { return (size_t)(2 * nn + (2 + 2 * DEPTH) * TILE) * sizeof(double); }
    // adj_volume_reg_kernel: D, Dhat, X, Y and the d_m (their adjoints are in registers)
    static constexpr size_t reg_smem_bytes() { return (size_t)(2 * nn + (2 + DEPTH) * TILE) * sizeof(double); }
};

struct AdjVolArgs {
    const double* u;        // state of the step
    const double* lam;      // adjoint of u_new
    double* lam_out;        // adjoint of u
    const double* bF;       // adjoint face traces from adj_interface_kernel
    const double* bU;
    const double* bu;
    const double* inv_jac;
    const double* dt;
    int E;
    double gamma;
    const double* dstore;   // the step's stage derivatives d_1..d_depth [m][e][v][node], from the recompute
};

template <int N>
static __global__ void __launch_bounds__(AdjCfg<N>::THREADS, AdjCfg<N>::MIN_BLOCKS) adj_volume_kernel(AdjVolArgs a) {
    using C = AdjCfg<N>;
    using K = LWC<C::DEPTH>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, DEPTH = C::DEPTH, TILE = C::TILE;
    extern __shared__ double sm[];
    double* sD = sm;
    double* sDh = sm + nn;
    double* X = sm + 2 * nn;
    double* Y = X + TILE;
    double* Dm = Y + TILE;             // d_m,     m = 1..DEPTH at Dm + (m - 1) * TILE
    double* Bm = Dm + DEPTH * TILE;    // bar d_m, same layout
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        sD[k] = c_tlw_D[N][k];
        sDh[k] = c_tlw_Dhat[N][k];
    }
    const int el = threadIdx.x / nn;
    const int node = threadIdx.x - el * nn;
    const int i = node % n, j = node / n;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    // threads past the last element slot of the CTA take part in the barriers only: they read slot 0 and
    // write nothing to shared memory
    const bool in_tile = el < EB;
    const int slot = in_tile ? el : 0;
    const int me = slot * nn + node;   // this node's offset inside a variable plane of a tile
    auto at = [&](double* T, int v) -> double* { return T + v * EB * nn + me; };
    auto put = [&](double* T, int v, double x) {
        if (in_tile) *at(T, v) = x;
    };
    double u[NV] = {1.0, 0.0, 0.0, 2.5};
    double ij = 1.0;
    if (active) {
        aload4(a.u + ((size_t)e * nn + node) * NV, u);
        ij = __ldg(a.inv_jac + e);
    }
    const double dt = *a.dt;
    const double sc = -dt * ij;
    const double gm1 = a.gamma - 1.0;
    // x / y contraction of a shared tile at this node: sum_k M[i][k] F[k, j] and sum_k M[j][k] F[i, k]
    auto cx = [&](const double* M, const double* F, int v) {
        const double* p = F + v * EB * nn + slot * nn + n * j;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[i * n + k], p[k], s);
        return s;
    };
    auto cy = [&](const double* M, const double* F, int v) {
        const double* p = F + v * EB * nn + slot * nn + i;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[j * n + k], p[n * k], s);
        return s;
    };
    // transposed: sum_k M[k][i] W[k, j] and sum_k M[k][j] W[i, k]
    auto cxt = [&](const double* M, const double* W, int v) {
        const double* p = W + v * EB * nn + slot * nn + n * j;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[k * n + i], p[k], s);
        return s;
    };
    auto cyt = [&](const double* M, const double* W, int v) {
        const double* p = W + v * EB * nn + slot * nn + i;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[k * n + j], p[n * k], s);
        return s;
    };
    // perturbed state q of stage s at this node
    auto state = [&](int s, int q, double* P) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double x = u[v];
#pragma unroll
            for (int m = 1; m <= s; ++m) x = fma(K::a(q, m), *at(Dm + (m - 1) * TILE, v), x);
            P[v] = x;
        }
    };

    // ---- d_1 .. d_DEPTH into shared memory
    {
        double f[NV], g[NV];
        euler_fluxes(gm1, u[0], u[1], u[2], u[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { put(X, v, f[v]); put(Y, v, g[v]); }
    }
    __syncthreads();
    {
        double d1[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) d1[v] = sc * (cx(sD, X, v) + cy(sD, Y, v));
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) put(Dm, v, d1[v]);
    }
#pragma unroll
    for (int s = 1; s < DEPTH; ++s) {
        double ft[NV] = {0.0, 0.0, 0.0, 0.0}, gt[NV] = {0.0, 0.0, 0.0, 0.0};
        if (K::w(s, 0) != 0.0) {
            double f[NV], g[NV];
            euler_fluxes(gm1, u[0], u[1], u[2], u[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { ft[v] = K::w(s, 0) * f[v]; gt[v] = K::w(s, 0) * g[v]; }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (K::w(s, 1 + q) == 0.0) continue;
            double P[NV], f[NV], g[NV];
            state(s, q, P);
            euler_fluxes(gm1, P[0], P[1], P[2], P[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { ft[v] = fma(K::w(s, 1 + q), f[v], ft[v]); gt[v] = fma(K::w(s, 1 + q), g[v], gt[v]); }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) { put(X, v, ft[v]); put(Y, v, gt[v]); }
        __syncthreads();
        double dn[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) dn[v] = sc * (cx(sD, X, v) + cy(sD, Y, v));
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) put(Dm + s * TILE, v, dn[v]);
    }

    // ---- adjoint inputs: volume term u_new += sc (Dhat F + Dhat G), then the face traces
    double bF[NV], bG[NV], bU[NV] = {0.0, 0.0, 0.0, 0.0}, bud[NV] = {0.0, 0.0, 0.0, 0.0};
    {
        double lam[NV] = {0.0, 0.0, 0.0, 0.0};
        if (active) aload4(a.lam + ((size_t)e * nn + node) * NV, lam);
#pragma unroll
        for (int v = 0; v < NV; ++v) put(X, v, sc * lam[v]);
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) { bF[v] = cxt(sDh, X, v); bG[v] = cyt(sDh, X, v); }
    if (active) {
        auto face = [&](int f, int l, double* tgt) {
            const size_t t = (((size_t)e * 4 + f) * n + l) * NV;
            double x[NV];
            aload4(a.bF + t, x);
#pragma unroll
            for (int v = 0; v < NV; ++v) tgt[v] += x[v];
            aload4(a.bU + t, x);
#pragma unroll
            for (int v = 0; v < NV; ++v) bU[v] += x[v];
            aload4(a.bu + t, x);
#pragma unroll
            for (int v = 0; v < NV; ++v) bud[v] += x[v];
        };
        if (i == 0) face(0, j, bF);
        if (i == n - 1) face(1, j, bF);
        if (j == 0) face(2, i, bG);
        if (j == n - 1) face(3, i, bG);
    }

    // ---- reverse sweep (bar d_m accumulate in shared memory, each thread on its own node)
    double bu[NV], bf0[NV], bg0[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int m = 0; m < DEPTH; ++m) put(Bm + m * TILE, v, K::tw(m + 1) * bU[v]);
        bu[v] = bU[v];
        bf0[v] = bF[v];
        bg0[v] = bG[v];
    }
#pragma unroll
    for (int s = DEPTH; s >= 1; --s) {
        double bfx[NV], bgy[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) { bfx[v] = K::tw(s) * bF[v]; bgy[v] = K::tw(s) * bG[v]; }
        if (s < DEPTH) {
            // d_{s+1} = C(ft_s, gt_s): its adjoint is complete (stages > s are done)
            __syncthreads();
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                bfx[v] = fma(sc, cxt(sD, Bm + s * TILE, v), bfx[v]);
                bgy[v] = fma(sc, cyt(sD, Bm + s * TILE, v), bgy[v]);
            }
        }
        if (K::w(s, 0) != 0.0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) { bf0[v] = fma(K::w(s, 0), bfx[v], bf0[v]); bg0[v] = fma(K::w(s, 0), bgy[v], bg0[v]); }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (K::w(s, 1 + q) == 0.0) continue;
            double P[NV], wf[NV], wg[NV], bP[NV] = {0.0, 0.0, 0.0, 0.0};
            state(s, q, P);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                wf[v] = K::w(s, 1 + q) * bfx[v];
                wg[v] = K::w(s, 1 + q) * bgy[v];
            }
            euler_flux_vjp(a.gamma, P, wf, wg, bP);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                bu[v] += bP[v];
                if (in_tile) {
#pragma unroll
                    for (int m = 1; m <= s; ++m) *at(Bm + (m - 1) * TILE, v) = fma(K::a(q, m), bP[v], *at(Bm + (m - 1) * TILE, v));
                }
            }
        }
    }
    // d_1 = C(f(u), g(u))
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) { bf0[v] = fma(sc, cxt(sD, Bm, v), bf0[v]); bg0[v] = fma(sc, cyt(sD, Bm, v), bg0[v]); }
    euler_flux_vjp(a.gamma, u, bf0, bg0, bu);
    if (active) {
        double lam[NV], o[NV];
        aload4(a.lam + ((size_t)e * nn + node) * NV, lam);
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = lam[v] + bu[v] + bud[v];
        astore4(a.lam_out + ((size_t)e * nn + node) * NV, o);
    }
}

// adj_volume_kernel with the stage derivatives stored by the segment recompute, held in registers with their
// adjoints: each thread reads and accumulates only its own node's d_m and bar d_m, so only the transposed
// contractions go through shared memory (one tile per stage, alternating between X and Y so that one barrier a
// stage separates a tile's reads from its next writes). Same operations in the same order as the LOADD kernel.
// DREG: the d_m in registers too; otherwise in shared memory, where each thread reads back only what it wrote.
template <int N, int MINB, bool DREG = false>
static __global__ void __launch_bounds__(AdjCfg<N>::THREADS, MINB) adj_volume_reg_kernel(AdjVolArgs a) {
    using C = AdjCfg<N>;
    using K = LWC<C::DEPTH>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, DEPTH = C::DEPTH, TILE = C::TILE;
    extern __shared__ double sm[];
    double* sD = sm;
    double* sDh = sm + nn;
    double* X = sm + 2 * nn;
    double* Y = X + TILE;
    double* Dt = Y + TILE;   // d_m at Dt + (m - 1) * TILE (!DREG)
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        sD[k] = c_tlw_D[N][k];
        sDh[k] = c_tlw_Dhat[N][k];
    }
    const int el = threadIdx.x / nn;
    const int node = threadIdx.x - el * nn;
    const int i = node % n, j = node / n;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    const bool in_tile = el < EB;
    const int slot = in_tile ? el : 0;
    const int me = slot * nn + node;
    auto put = [&](double* T, int v, double x) {
        if (in_tile) T[v * EB * nn + me] = x;
    };
    double u[NV] = {1.0, 0.0, 0.0, 2.5};
    double ij = 1.0;
    double dm[DREG ? DEPTH : 1][NV];
#pragma unroll
    for (int m = 0; m < (DREG ? DEPTH : 1); ++m)
#pragma unroll
        for (int v = 0; v < NV; ++v) dm[m][v] = 0.0;
    double lam[NV] = {0.0, 0.0, 0.0, 0.0};
    if (active) {
        aload4(a.u + ((size_t)e * nn + node) * NV, u);
        ij = __ldg(a.inv_jac + e);
        if (DREG) {
#pragma unroll
            for (int m = 0; m < DEPTH; ++m)
                for (int v = 0; v < NV; ++v) dm[DREG ? m : 0][v] = a.dstore[((size_t)m * a.E + e) * NV * nn + v * nn + node];
        }
        aload4(a.lam + ((size_t)e * nn + node) * NV, lam);
    }
    if (!DREG) {
#pragma unroll
        for (int m = 0; m < DEPTH; ++m) {
            double d[NV] = {0.0, 0.0, 0.0, 0.0};
            if (active) {
#pragma unroll
                for (int v = 0; v < NV; ++v) d[v] = a.dstore[((size_t)m * a.E + e) * NV * nn + v * nn + node];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) put(Dt + m * TILE, v, d[v]);
        }
    }
    // d_m of this node, m = 1..DEPTH (a thread outside the tile reads zeros)
    auto dget = [&](int m, int v) -> double {
        if (DREG) return dm[DREG ? m - 1 : 0][v];
        return in_tile ? Dt[(m - 1) * TILE + v * EB * nn + me] : 0.0;
    };
    const double dt = *a.dt;
    const double sc = -dt * ij;
    auto cxt = [&](const double* M, const double* W, int v) {
        const double* p = W + v * EB * nn + slot * nn + n * j;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[k * n + i], p[k], s);
        return s;
    };
    auto cyt = [&](const double* M, const double* W, int v) {
        const double* p = W + v * EB * nn + slot * nn + i;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[k * n + j], p[n * k], s);
        return s;
    };

    // ---- adjoint inputs: volume term u_new += sc (Dhat F + Dhat G), then the face traces
    double bF[NV], bG[NV], bU[NV] = {0.0, 0.0, 0.0, 0.0}, bud[NV] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int v = 0; v < NV; ++v) put(X, v, sc * lam[v]);
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) { bF[v] = cxt(sDh, X, v); bG[v] = cyt(sDh, X, v); }
    if (active) {
        auto face = [&](int f, int l, double* tgt) {
            const size_t t = (((size_t)e * 4 + f) * n + l) * NV;
            double x[NV];
            aload4(a.bF + t, x);
#pragma unroll
            for (int v = 0; v < NV; ++v) tgt[v] += x[v];
            aload4(a.bU + t, x);
#pragma unroll
            for (int v = 0; v < NV; ++v) bU[v] += x[v];
            aload4(a.bu + t, x);
#pragma unroll
            for (int v = 0; v < NV; ++v) bud[v] += x[v];
        };
        if (i == 0) face(0, j, bF);
        if (i == n - 1) face(1, j, bF);
        if (j == 0) face(2, i, bG);
        if (j == n - 1) face(3, i, bG);
    }

    // ---- reverse sweep
    double bd[DEPTH][NV], bu[NV], bf0[NV], bg0[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int m = 0; m < DEPTH; ++m) bd[m][v] = K::tw(m + 1) * bU[v];
        bu[v] = bU[v];
        bf0[v] = bF[v];
        bg0[v] = bG[v];
    }
#pragma unroll
    for (int s = DEPTH; s >= 1; --s) {
        double bfx[NV], bgy[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) { bfx[v] = K::tw(s) * bF[v]; bgy[v] = K::tw(s) * bG[v]; }
        if (s < DEPTH) {
            // d_{s+1} = C(ft_s, gt_s): its adjoint is complete (stages > s are done)
            double* T = ((DEPTH - s) & 1) ? Y : X;
#pragma unroll
            for (int v = 0; v < NV; ++v) put(T, v, bd[s][v]);
            __syncthreads();
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                bfx[v] = fma(sc, cxt(sD, T, v), bfx[v]);
                bgy[v] = fma(sc, cyt(sD, T, v), bgy[v]);
            }
        }
        if (K::w(s, 0) != 0.0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) { bf0[v] = fma(K::w(s, 0), bfx[v], bf0[v]); bg0[v] = fma(K::w(s, 0), bgy[v], bg0[v]); }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (K::w(s, 1 + q) == 0.0) continue;
            double P[NV], wf[NV], wg[NV], bP[NV] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double x = u[v];
#pragma unroll
                for (int m = 1; m <= s; ++m) x = fma(K::a(q, m), dget(m, v), x);
                P[v] = x;
                wf[v] = K::w(s, 1 + q) * bfx[v];
                wg[v] = K::w(s, 1 + q) * bgy[v];
            }
            euler_flux_vjp(a.gamma, P, wf, wg, bP);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                bu[v] += bP[v];
#pragma unroll
                for (int m = 1; m <= s; ++m) bd[m - 1][v] = fma(K::a(q, m), bP[v], bd[m - 1][v]);
            }
        }
    }
    // d_1 = C(f(u), g(u))
    {
        double* T = (DEPTH & 1) ? Y : X;
#pragma unroll
        for (int v = 0; v < NV; ++v) put(T, v, bd[0][v]);
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NV; ++v) { bf0[v] = fma(sc, cxt(sD, T, v), bf0[v]); bg0[v] = fma(sc, cyt(sD, T, v), bg0[v]); }
    }
    euler_flux_vjp(a.gamma, u, bf0, bg0, bu);
    if (active) {
        double o[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = lam[v] + bu[v] + bud[v];
        astore4(a.lam_out + ((size_t)e * nn + node) * NV, o);
    }
}

// ---- the two-stage MDRK step (mdrk.jl:1-29, rhs_mdrk1! / rhs_mdrk2!, src/solvers/dgsem_tree/multi_derivative_2d.jl)
// Stage 1 at u: d = C(f(u)), P_q = u + a_q d (a = -1, +1, -2, +2), f_t = sum_q w_q f(P_q) (w = -8/12, 8/12, 1/12,
// -1/12); Fh = f/2 + f_t/8, Uh = u/2 + d/8 feed the surface, F2 = f + f_t/6, U2 = u + d/6 go to stage 2;
// u* = u + dt rhs_1. Stage 2 at u*: the same procedure, F = F2 + f*_t/3, U = U2 + d*/3, interfaces with the jump in
// u^n; u_new = u + dt rhs_2. Both stages have the LW step's form x_out = u + dt rhs(.), so adj_interface_kernel
// gives each stage's face adjoints (stage 2: U traces of stage 2, adjoint lam; stage 1: Uh traces, adjoint of u*).
// adj_mdrk_volume_kernel<N, 2> turns lam into the adjoint of u* (out), of (F2, G2) and U2 (to stage 1), and
// lam + the jump's direct term (lam_acc); adj_mdrk_volume_kernel<N, 1> takes the adjoint of u* as its lam and
// writes lam_out = lam_acc + lam + (du*/du)^T-part of stage 1.
struct AdjMdrkArgs {
    const double* x;        // the stage's state: u^n (stage 1) or u* (stage 2)
    const double* lam;      // adjoint of the stage's output: u_new (stage 2) or u* (stage 1)
    const double* bF;       // face adjoints from adj_interface_kernel [v, l, face, e]
    const double* bU;
    const double* bu;
    double* bF2;            // adjoint of (F2, G2) [v, d, node]: written by stage 2, read by stage 1
    double* bU2;            // adjoint of U2 [v, node]
    double* lam_acc;        // stage 2 writes lam + the jump's direct term; stage 1 adds it
    double* out;            // stage 2: adjoint of u*; stage 1: the adjoint of u^n
    const double* inv_jac;
    const double* dt;
    int E;
    double gamma;
};

template <int N>
struct AdjMdrkCfg {
    static constexpr int n = N + 1, nn = n * n;
    static constexpr int EB = VolCfg<N>::EB;
    static constexpr int THREADS = VolCfg<N>::THREADS;
    static constexpr int MIN_BLOCKS = THREADS <= 128 ? 3 : 1;
    static constexpr int TILE = NV * EB * nn;
    // D, Dhat and three tiles (X, Y, the adjoint of d)
    static constexpr size_t smem_bytes() { return (size_t)(2 * nn + 3 * TILE) * sizeof(double); }
};

template <int N, int STAGE>
static __global__ void __launch_bounds__(AdjMdrkCfg<N>::THREADS, AdjMdrkCfg<N>::MIN_BLOCKS)
    adj_mdrk_volume_kernel(AdjMdrkArgs a) {
    using C = AdjMdrkCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, TILE = C::TILE;
    constexpr double A[4] = {-1.0, 1.0, -2.0, 2.0};
    constexpr double W[4] = {-8.0 / 12.0, 8.0 / 12.0, 1.0 / 12.0, -1.0 / 12.0};
    extern __shared__ double sm[];
    double* sD = sm;
    double* sDh = sm + nn;
    double* X = sm + 2 * nn;
    double* Y = X + TILE;
    double* Bd = Y + TILE;
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        sD[k] = c_tlw_D[N][k];
        sDh[k] = c_tlw_Dhat[N][k];
    }
    const int el = threadIdx.x / nn;
    const int node = threadIdx.x - el * nn;
    const int i = node % n, j = node / n;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    const bool in_tile = el < EB;
    const int slot = in_tile ? el : 0;
    const int me = slot * nn + node;
    auto at = [&](double* T, int v) -> double* { return T + v * EB * nn + me; };
    auto put = [&](double* T, int v, double x) {
        if (in_tile) *at(T, v) = x;
    };
    auto cx = [&](const double* M, const double* F, int v) {
        const double* p = F + v * EB * nn + slot * nn + n * j;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[i * n + k], p[k], s);
        return s;
    };
    auto cy = [&](const double* M, const double* F, int v) {
        const double* p = F + v * EB * nn + slot * nn + i;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[j * n + k], p[n * k], s);
        return s;
    };
    auto cxt = [&](const double* M, const double* W_, int v) {
        const double* p = W_ + v * EB * nn + slot * nn + n * j;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[k * n + i], p[k], s);
        return s;
    };
    auto cyt = [&](const double* M, const double* W_, int v) {
        const double* p = W_ + v * EB * nn + slot * nn + i;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < n; ++k) s = fma(M[k * n + j], p[n * k], s);
        return s;
    };
    double x[NV] = {1.0, 0.0, 0.0, 2.5};
    double ij = 1.0;
    const size_t off = (size_t)e * nn + node;
    if (active) {
        aload4(a.x + off * NV, x);
        ij = __ldg(a.inv_jac + e);
    }
    const double dt = *a.dt;
    const double sc = -dt * ij;
    const double gm1 = a.gamma - 1.0;
    // forward: d = C(f(x), g(x))
    {
        double f[NV], g[NV];
        euler_fluxes(gm1, x[0], x[1], x[2], x[3], f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) { put(X, v, f[v]); put(Y, v, g[v]); }
    }
    __syncthreads();
    double d[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) d[v] = sc * (cx(sD, X, v) + cy(sD, Y, v));
    __syncthreads();
    // adjoint of the volume term sc (Dhat F + Dhat G), then the face traces
    double lam[NV] = {0.0, 0.0, 0.0, 0.0};
    if (active) aload4(a.lam + off * NV, lam);
#pragma unroll
    for (int v = 0; v < NV; ++v) put(X, v, sc * lam[v]);
    __syncthreads();
    double bF[NV], bG[NV], bU[NV] = {0.0, 0.0, 0.0, 0.0}, bud[NV] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int v = 0; v < NV; ++v) { bF[v] = cxt(sDh, X, v); bG[v] = cyt(sDh, X, v); }
    if (active) {
        auto face = [&](int f, int l, double* tgt) {
            const size_t t = (((size_t)e * 4 + f) * n + l) * NV;
            double y[NV];
            aload4(a.bF + t, y);
#pragma unroll
            for (int v = 0; v < NV; ++v) tgt[v] += y[v];
            aload4(a.bU + t, y);
#pragma unroll
            for (int v = 0; v < NV; ++v) bU[v] += y[v];
            aload4(a.bu + t, y);
#pragma unroll
            for (int v = 0; v < NV; ++v) bud[v] += y[v];
        };
        if (i == 0) face(0, j, bF);
        if (i == n - 1) face(1, j, bF);
        if (j == 0) face(2, i, bG);
        if (j == n - 1) face(3, i, bG);
    }
    // the stage's combination of f(x), f_t, x, d into its outputs
    double bft[NV], bgt[NV], bf0[NV], bg0[NV], bx[NV], bd[NV];
    if (STAGE == 2) {
        // F = F2 + f_t / 3, U = U2 + d / 3
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            bft[v] = bF[v] * (1.0 / 3.0);
            bgt[v] = bG[v] * (1.0 / 3.0);
            bd[v] = bU[v] * (1.0 / 3.0);
            bf0[v] = bg0[v] = bx[v] = 0.0;
        }
        if (active) {
            astore4(a.bF2 + off * 2 * NV, bF);
            astore4(a.bF2 + off * 2 * NV + NV, bG);
            astore4(a.bU2 + off * NV, bU);
            double acc[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) acc[v] = lam[v] + bud[v];
            astore4(a.lam_acc + off * NV, acc);
        }
    } else {
        // Fh = f/2 + f_t/8, Uh = x/2 + d/8; F2 = f + f_t/6, U2 = x + d/6
        double b2f[NV] = {0.0, 0.0, 0.0, 0.0}, b2g[NV] = {0.0, 0.0, 0.0, 0.0}, b2u[NV] = {0.0, 0.0, 0.0, 0.0};
        if (active) {
            aload4(a.bF2 + off * 2 * NV, b2f);
            aload4(a.bF2 + off * 2 * NV + NV, b2g);
            aload4(a.bU2 + off * NV, b2u);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            bf0[v] = fma(0.5, bF[v], b2f[v]);
            bg0[v] = fma(0.5, bG[v], b2g[v]);
            bft[v] = fma(0.125, bF[v], b2f[v] * (1.0 / 6.0));
            bgt[v] = fma(0.125, bG[v], b2g[v] * (1.0 / 6.0));
            bx[v] = fma(0.5, bU[v], b2u[v]);
            bd[v] = fma(0.125, bU[v], b2u[v] * (1.0 / 6.0));
        }
    }
    // f_t = sum_q W_q f(x + A_q d)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double P[NV], wf[NV], wg[NV], bP[NV] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            P[v] = fma(A[q], d[v], x[v]);
            wf[v] = W[q] * bft[v];
            wg[v] = W[q] * bgt[v];
        }
        euler_flux_vjp(a.gamma, P, wf, wg, bP);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            bx[v] += bP[v];
            bd[v] = fma(A[q], bP[v], bd[v]);
        }
    }
    // d = C(f(x), g(x))
#pragma unroll
    for (int v = 0; v < NV; ++v) put(Bd, v, bd[v]);
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) { bf0[v] = fma(sc, cxt(sD, Bd, v), bf0[v]); bg0[v] = fma(sc, cyt(sD, Bd, v), bg0[v]); }
    euler_flux_vjp(a.gamma, x, bf0, bg0, bx);
    if (active) {
        double o[NV];
        if (STAGE == 2) {
#pragma unroll
            for (int v = 0; v < NV; ++v) o[v] = bx[v];
        } else {
            double acc[NV];
            aload4(a.lam_acc + off * NV, acc);
#pragma unroll
            for (int v = 0; v < NV; ++v) o[v] = acc[v] + lam[v] + bx[v] + bud[v];
        }
        astore4(a.out + off * NV, o);
    }
}

// J = 1/2 sum_nodes (rho - rho_target)^2: per-block partial sums (fixed order) and the seed lam = (rho - rho_t, 0, 0, 0)
constexpr int OBJ_THREADS = 256;
static __global__ void __launch_bounds__(OBJ_THREADS) objective_kernel(const double* u, const double* target,
                                                                       long long nodes, double* partial, double* lam) {
    __shared__ double red[OBJ_THREADS];
    const long long k = (long long)blockIdx.x * OBJ_THREADS + threadIdx.x;
    double r = 0.0;
    if (k < nodes) {
        r = u[k * NV] - target[k];
        double o[NV] = {r, 0.0, 0.0, 0.0};
        astore4(lam + k * NV, o);
    }
    red[threadIdx.x] = 0.5 * r * r;
    __syncthreads();
    for (int w = OBJ_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

static __global__ void __launch_bounds__(OBJ_THREADS) sum_kernel(const double* partial, int count, double* out) {
    __shared__ double red[OBJ_THREADS];
    double s = 0.0;
    for (int k = threadIdx.x; k < count; k += OBJ_THREADS) s += partial[k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = OBJ_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// ---- launches ---------------------------------------------------------------------------------------
template <int N>
struct AL {
    static void set_attributes() {
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VolCfg<N>::smem_bytes(4));
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VolCfg<N>::smem_bytes(4));
        cudaFuncSetAttribute(adj_volume_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)AdjCfg<N>::smem_bytes());
        cudaFuncSetAttribute(adj_volume_reg_kernel<N, AdjCfg<N>::MIN_BLOCKS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)AdjCfg<N>::reg_smem_bytes());
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false, 0, false, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VolCfg<N>::smem_bytes(4));
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, false, 0, false, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VolCfg<N>::smem_bytes(4));
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_STEP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VolCfg<N>::smem_bytes(2));
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VolCfg<N>::smem_bytes(2));
        cudaFuncSetAttribute(adj_mdrk_volume_kernel<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)AdjMdrkCfg<N>::smem_bytes());
        cudaFuncSetAttribute(adj_mdrk_volume_kernel<N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)AdjMdrkCfg<N>::smem_bytes());
    }
    // the forward MDRK stages (stage 1: u -> u*, stage 2: u* -> u_new with u_base = u^n)
    static void forward_mdrk_volume(cudaStream_t s, int stage, const VolArgs& va) {
        using C = VolCfg<N>;
        const int grid = (int)((va.E + C::EB - 1) / C::EB);
        if (stage == 1) mdrk1_volume_kernel<N, MODE_STEP, false><<<grid, C::THREADS, C::smem_bytes(2), s>>>(va);
        else mdrk2_volume_kernel<N, MODE_STEP, false><<<grid, C::THREADS, C::smem_bytes(2), s>>>(va);
    }
    static void adjoint_mdrk(cudaStream_t s, int stage, const AdjSurfArgs& sa, const AdjMdrkArgs& ma) {
        const long long th = (long long)(sa.nx + sa.ny) * (N + 1);
        if (th) adj_interface_kernel<N><<<(unsigned)((th + 127) / 128), 128, 0, s>>>(sa);
        using C = AdjMdrkCfg<N>;
        const int grid = (ma.E + C::EB - 1) / C::EB;
        if (stage == 2) adj_mdrk_volume_kernel<N, 2><<<grid, C::THREADS, C::smem_bytes(), s>>>(ma);
        else adj_mdrk_volume_kernel<N, 1><<<grid, C::THREADS, C::smem_bytes(), s>>>(ma);
    }
    // with va.dstore: also store the stage derivatives for the adjoint
    static void forward_volume(cudaStream_t s, int mode, const VolArgs& va) {
        using C = VolCfg<N>;
        const int grid = (int)((va.E + C::EB - 1) / C::EB);
        const size_t sm = C::smem_bytes(4);
        if (va.dstore) {
            if (mode == MODE_STEP) lw_volume_kernel<N, MODE_STEP, false, 0, false, false, true><<<grid, C::THREADS, sm, s>>>(va);
            else lw_volume_kernel<N, MODE_RHS, false, 0, false, false, true><<<grid, C::THREADS, sm, s>>>(va);
        } else {
            if (mode == MODE_STEP) lw_volume_kernel<N, MODE_STEP, false><<<grid, C::THREADS, sm, s>>>(va);
            else lw_volume_kernel<N, MODE_RHS, false><<<grid, C::THREADS, sm, s>>>(va);
        }
    }
    static void forward_interfaces(cudaStream_t s, SurfArgs sa, const tlw_handle* h) {
        if (h->d_nbr && h->nb == 0 && h->nmx + h->nmy == 0 && h->nh == 0) {
            // the element-centric pass the plain step uses on a periodic mesh (same bits)
            sa.nbr = h->d_nbr;
            sa.E = (int)h->E;
            using C = SurfCfg<N>;
            surface_kernel<N, false, false><<<(unsigned)((sa.E + C::EB - 1) / C::EB), C::THREADS, 0, s>>>(sa, BndArgs{});
            return;
        }
        sa.left = h->d_xl; sa.right = h->d_xr; sa.count = h->nx; sa.orientation = 1;
        long long th = (long long)sa.count * (N + 1);
        if (th) interface_kernel<N><<<(unsigned)((th + 127) / 128), 128, 0, s>>>(sa);
        sa.left = h->d_yl; sa.right = h->d_yr; sa.count = h->ny; sa.orientation = 2;
        th = (long long)sa.count * (N + 1);
        if (th) interface_kernel<N><<<(unsigned)((th + 127) / 128), 128, 0, s>>>(sa);
    }
    static void speed(cudaStream_t s, const tlw_handle* h, const double* u) {
        const int E = (int)h->E;
        const int grid = (E + MsCfg<N>::ELEMS - 1) / MsCfg<N>::ELEMS;
        max_speed_kernel<N, true, false><<<grid, MS_THREADS, 0, s>>>(u, h->d_inv_jac, E, h->opts.gamma, h->d_step,
                                                                     IndicatorArgs{}, BatchSpeedArgs{});
    }
    static void adjoint(cudaStream_t s, const AdjSurfArgs& sa, const AdjVolArgs& va) {
        const long long th = (long long)(sa.nx + sa.ny) * (N + 1);
        if (th) adj_interface_kernel<N><<<(unsigned)((th + 127) / 128), 128, 0, s>>>(sa);
        using C = AdjCfg<N>;
        const int grid = (va.E + C::EB - 1) / C::EB;
        if (va.dstore) {
            adj_volume_reg_kernel<N, C::MIN_BLOCKS><<<grid, C::THREADS, C::reg_smem_bytes(), s>>>(va);
        } else {
            adj_volume_kernel<N><<<grid, C::THREADS, C::smem_bytes(), s>>>(va);
        }
    }
};

template <class F>
bool adj_degree(int N, F&& f) {
    switch (N) {
        case 3: f(std::integral_constant<int, 3>{}); return true;
        case 4: f(std::integral_constant<int, 4>{}); return true;
        case 5: f(std::integral_constant<int, 5>{}); return true;
        default: return false;
    }
}

size_t nstate(const tlw_handle* h) { return (size_t)NV * h->nn * h->E; }
size_t ntrace(const tlw_handle* h) { return (size_t)NV * h->n * 4 * h->E; }
// stages of the volume procedure: 3 for N = 3, 4 for N >= 4
int depth(const tlw_handle* h) { return h->N >= 4 ? 4 : 3; }

// segment buffer b (0 or 1): step j's input state (j = len: the segment's output, or scratch), U traces and
// stage derivatives
double* seg_state(tlw_handle* h, int b, int j) {
    return h->adj.d_seg + ((size_t)b * (h->adj.capacity_states + 1) + j) * nstate(h);
}
double* seg_trace(tlw_handle* h, int b, int j) {
    return h->adj.d_segU + ((size_t)b * h->adj.capacity_states + j) * ntrace(h);
}
double* seg_D(tlw_handle* h, int b, int j) {
    return h->adj.d_segD ? h->adj.d_segD + ((size_t)b * h->adj.capacity_states + j) * depth(h) * nstate(h) : nullptr;
}
bool is_mdrk(const tlw_handle* h) { return h->opts.time_discretization == TLW_MDRK; }
// MDRK: step j's stage state u* and stage-2 U traces (null for LW)
double* seg_ustar(tlw_handle* h, int b, int j) {
    return h->adj.d_segS ? h->adj.d_segS + ((size_t)b * h->adj.capacity_states + j) * nstate(h) : nullptr;
}
double* seg_trace2(tlw_handle* h, int b, int j) {
    return h->adj.d_segU2 ? h->adj.d_segU2 + ((size_t)b * h->adj.capacity_states + j) * ntrace(h) : nullptr;
}

int adj_ready(tlw_handle* h) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh) return afail(h, TLW_E_STATE, "no mesh: call tlw_set_tree_mesh first");
    if (h->sc || h->opts.surface_flux != TLW_FLUX_RUSANOV || h->nb > 0 || h->curved || h->N < 3 || h->N > 5 ||
        h->nmx + h->nmy > 0 || h->parabolic || h->lim_count > 0)
        return afail(h, TLW_E_UNSUPPORTED,
                     "adjoint: LW or MDRK, FR volume integral, Rusanov flux, periodic conforming TreeMesh, Euler, "
                     "N = 3..5, no positivity limiter");
    TLW_ACUDA(h, cudaSetDevice(h->device));
    AdjointBuffers& A = h->adj;
    if (!A.const_uploaded) {
        Basis all[8];
        std::memset(&all[0], 0, sizeof(all[0]));
        for (int N = 1; N <= 7; ++N) host_build_basis(N, all[N]);
        TLW_ACUDA(h, upload_const_basis(all));
        adj_degree(h->N, [&](auto Nc) { AL<decltype(Nc)::value>::set_attributes(); });
        A.const_uploaded = true;
    }
    if (A.E != h->E) {
        const bool keep = A.const_uploaded;
        free_adjoint(A);
        A.const_uploaded = keep;
        A.E = h->E;
    }
    if (!A.d_lam[0]) {
        TLW_ACUDA(h, cudaMalloc(&A.d_lam[0], nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_lam[1], nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_bF, ntrace(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_bU, ntrace(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_bu, ntrace(h) * sizeof(double)));
        const size_t blocks = ((size_t)h->nn * h->E + OBJ_THREADS - 1) / OBJ_THREADS;
        TLW_ACUDA(h, cudaMalloc(&A.d_work, (blocks + 8) * sizeof(double)));
    }
    if (is_mdrk(h) && !A.d_bus) {
        TLW_ACUDA(h, cudaMalloc(&A.d_mus, nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_mtU2, ntrace(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_bus, nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_bF2, 2 * nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_bU2, nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_lamacc, nstate(h) * sizeof(double)));
    }
    if (!A.s_rec) {
        // the reverse sweep's two streams: the adjoint chain (the critical path) above the recomputation in
        // priority
        int least = 0, greatest = 0;
        TLW_ACUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
        TLW_ACUDA(h, cudaStreamCreateWithPriority(&A.s_rec, cudaStreamNonBlocking, least));
        TLW_ACUDA(h, cudaStreamCreateWithPriority(&A.s_adj, cudaStreamNonBlocking, greatest));
        for (cudaEvent_t* ev : {&A.ev_fork, &A.ev_join, &A.ev_join2, &A.ev_ready[0], &A.ev_ready[1], &A.ev_free[0],
                                &A.ev_free[1]})
            TLW_ACUDA(h, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    }
    return TLW_OK;
}

int ensure_steps(tlw_handle* h, int nsteps, int ck) {
    AdjointBuffers& A = h->adj;
    // captured sweeps hold the buffer addresses: drop them when a buffer is replaced
    auto drop = [&]() {
        if (A.g_fwd) cudaGraphExecDestroy(A.g_fwd);
        if (A.g_rev) cudaGraphExecDestroy(A.g_rev);
        A.g_fwd = A.g_rev = nullptr;
    };
    // a run of one segment needs one segment buffer, otherwise two (recompute and adjoint alternate)
    const int nbuf = nsteps > ck ? 2 : 1;
    if (A.capacity_steps < nsteps || A.capacity_ckpt < (nsteps + ck - 1) / ck || A.capacity_states < ck ||
        A.capacity_buffers < nbuf)
        drop();
    if (A.capacity_steps < nsteps) {
        dfree(A.d_dts);
        TLW_ACUDA(h, cudaMalloc(&A.d_dts, (size_t)std::max(nsteps, 1) * sizeof(double)));
        A.capacity_steps = std::max(nsteps, 1);
    }
    const int nck = (nsteps + ck - 1) / ck;
    if (A.capacity_ckpt < nck) {
        dfree(A.d_ckpt);
        TLW_ACUDA(h, cudaMalloc(&A.d_ckpt, (size_t)std::max(nck, 1) * nstate(h) * sizeof(double)));
        A.capacity_ckpt = std::max(nck, 1);
    }
    if (A.capacity_states < ck || A.capacity_buffers < nbuf) {
        dfree(A.d_seg);
        dfree(A.d_segU);
        dfree(A.d_segD);
        dfree(A.d_segS);
        dfree(A.d_segU2);
        A.capacity_states = A.capacity_buffers = 0;
        A.last_resident = false;
        TLW_ACUDA(h, cudaMalloc(&A.d_seg, nbuf * (size_t)(ck + 1) * nstate(h) * sizeof(double)));
        TLW_ACUDA(h, cudaMalloc(&A.d_segU, nbuf * (size_t)ck * ntrace(h) * sizeof(double)));
        if (is_mdrk(h)) {
            // the MDRK adjoint recomputes the stage derivatives; it keeps u* and the stage-2 U traces instead
            TLW_ACUDA(h, cudaMalloc(&A.d_segS, nbuf * (size_t)ck * nstate(h) * sizeof(double)));
            TLW_ACUDA(h, cudaMalloc(&A.d_segU2, nbuf * (size_t)ck * ntrace(h) * sizeof(double)));
        } else {
            TLW_ACUDA(h, cudaMalloc(&A.d_segD, nbuf * (size_t)ck * depth(h) * nstate(h) * sizeof(double)));
        }
        A.capacity_states = ck;
        A.capacity_buffers = nbuf;
    }
    return TLW_OK;
}

// caller-given dt sequences (tlw_solve_dts, tlw_adjoint_step) live apart from the recorded one
int ensure_given_dts(tlw_handle* h, int nsteps) {
    AdjointBuffers& A = h->adj;
    if (A.capacity_given < nsteps) {
        dfree(A.d_dts_given);
        TLW_ACUDA(h, cudaMalloc(&A.d_dts_given, (size_t)nsteps * sizeof(double)));
        A.capacity_given = nsteps;
    }
    return TLW_OK;
}

VolArgs fwd_vol_args(tlw_handle* h, const double* u, double* out, double* tU, const double* dtp) {
    VolArgs va{};
    va.u = u;
    va.u_base = u;
    va.out = out;
    va.tU = tU;
    va.tF = h->d_tF;
    va.inv_jac = h->d_inv_jac;
    va.dt = dtp;
    va.basis = h->d_basis;
    va.E = (int)h->E;
    va.gamma = h->opts.gamma;
    va.status = &h->d_step->status;
    va.speed_kind = h->opts.max_speed;
    return va;
}

SurfArgs fwd_surf_args(tlw_handle* h, const double* u, double* out, const double* tU, const double* dtp, int step) {
    SurfArgs sa{};
    sa.u = u;
    sa.out = out;
    sa.tU = tU;
    sa.tF = h->d_tF;
    sa.inv_jac = h->d_inv_jac;
    sa.dt = dtp;
    sa.step_mode = step;
    sa.gamma = h->opts.gamma;
    sa.flux_kind = h->opts.surface_flux;
    sa.speed_kind = h->opts.max_speed;
    sa.inv_w_first = h->h_basis.inv_w_first;
    sa.inv_w_last = h->h_basis.inv_w_last;
    sa.status = &h->d_step->status;
    return sa;
}

// one forward step on stream s at the dt stored at dtp. LW: U traces into tU, stage derivatives into dstore. MDRK:
// the stage state u* into us and the stage-1 / stage-2 U traces into tU / tU2 (scratch when null)
void enqueue_fixed_step(tlw_handle* h, cudaStream_t s, const double* u, double* unew, double* tU, const double* dtp,
                        double* dstore = nullptr, double* us = nullptr, double* tU2 = nullptr) {
    if (is_mdrk(h)) {
        if (!us) us = h->adj.d_mus;
        if (!tU2) tU2 = h->adj.d_mtU2;
        VolArgs v1 = fwd_vol_args(h, u, us, tU, dtp);
        v1.U2 = h->d_U2;
        v1.F2 = h->d_F2;
        VolArgs v2 = fwd_vol_args(h, us, unew, tU2, dtp);
        v2.u_base = u;
        v2.U2 = h->d_U2;
        v2.F2 = h->d_F2;
        adj_degree(h->N, [&](auto Nc) {
            constexpr int N = decltype(Nc)::value;
            AL<N>::forward_mdrk_volume(s, 1, v1);
            AL<N>::forward_interfaces(s, fwd_surf_args(h, u, us, tU, dtp, 1), h);
            AL<N>::forward_mdrk_volume(s, 2, v2);
            AL<N>::forward_interfaces(s, fwd_surf_args(h, u, unew, tU2, dtp, 1), h);
        });
        return;
    }
    VolArgs va = fwd_vol_args(h, u, unew, tU, dtp);
    va.dstore = dstore;
    const SurfArgs sa = fwd_surf_args(h, u, unew, tU, dtp, 1);
    adj_degree(h->N, [&](auto Nc) {
        constexpr int N = decltype(Nc)::value;
        AL<N>::forward_volume(s, MODE_STEP, va);
        AL<N>::forward_interfaces(s, sa, h);
    });
}

// lam_out = (du_new/du)^T lam_in for the step from u at dt (*dtp); tU = that step's forward U traces (MDRK: its
// stage-1 traces, with us = u* and tU2 = the stage-2 traces)
void enqueue_adjoint_step(tlw_handle* h, const double* u, const double* tU, const double* dtp, const double* lam_in,
                          double* lam_out, const double* dstore = nullptr, cudaStream_t s = nullptr,
                          const double* us = nullptr, const double* tU2 = nullptr) {
    AdjointBuffers& A = h->adj;
    if (is_mdrk(h)) {
        AdjSurfArgs sa{};
        sa.u = u;   // both stages' jumps are in u^n
        sa.bF = A.d_bF;
        sa.bU = A.d_bU;
        sa.bu = A.d_bu;
        sa.xl = h->d_xl; sa.xr = h->d_xr; sa.yl = h->d_yl; sa.yr = h->d_yr;
        sa.nx = h->nx; sa.ny = h->ny;
        sa.inv_jac = h->d_inv_jac;
        sa.dt = dtp;
        sa.gamma = h->opts.gamma;
        sa.speed_kind = h->opts.max_speed;
        sa.inv_w_first = h->h_basis.inv_w_first;
        sa.inv_w_last = h->h_basis.inv_w_last;
        sa.status = &h->d_step->status;
        AdjMdrkArgs ma{};
        ma.bF = A.d_bF;
        ma.bU = A.d_bU;
        ma.bu = A.d_bu;
        ma.bF2 = A.d_bF2;
        ma.bU2 = A.d_bU2;
        ma.lam_acc = A.d_lamacc;
        ma.inv_jac = h->d_inv_jac;
        ma.dt = dtp;
        ma.E = (int)h->E;
        ma.gamma = h->opts.gamma;
        adj_degree(h->N, [&](auto Nc) {
            constexpr int N = decltype(Nc)::value;
            cudaStream_t st = s ? s : h->stream;
            // stage 2: lam -> adjoint of u*, (F2, G2), U2, lam + jump term
            AdjSurfArgs s2 = sa;
            s2.tU = tU2;
            s2.lam = lam_in;
            AdjMdrkArgs m2 = ma;
            m2.x = us;
            m2.lam = lam_in;
            m2.out = A.d_bus;
            AL<N>::adjoint_mdrk(st, 2, s2, m2);
            // stage 1: the adjoint of u* -> the adjoint of u^n
            AdjSurfArgs s1 = sa;
            s1.tU = tU;
            s1.lam = A.d_bus;
            AdjMdrkArgs m1 = ma;
            m1.x = u;
            m1.lam = A.d_bus;
            m1.out = lam_out;
            AL<N>::adjoint_mdrk(st, 1, s1, m1);
        });
        return;
    }
    AdjSurfArgs sa{};
    sa.u = u;
    sa.tU = tU;
    sa.lam = lam_in;
    sa.bF = A.d_bF;
    sa.bU = A.d_bU;
    sa.bu = A.d_bu;
    sa.xl = h->d_xl; sa.xr = h->d_xr; sa.yl = h->d_yl; sa.yr = h->d_yr;
    sa.nx = h->nx; sa.ny = h->ny;
    sa.inv_jac = h->d_inv_jac;
    sa.dt = dtp;
    sa.gamma = h->opts.gamma;
    sa.speed_kind = h->opts.max_speed;
    sa.inv_w_first = h->h_basis.inv_w_first;
    sa.inv_w_last = h->h_basis.inv_w_last;
    sa.status = &h->d_step->status;
    AdjVolArgs va{};
    va.u = u;
    va.lam = lam_in;
    va.lam_out = lam_out;
    va.bF = A.d_bF;
    va.bU = A.d_bU;
    va.bu = A.d_bu;
    va.inv_jac = h->d_inv_jac;
    va.dt = dtp;
    va.E = (int)h->E;
    va.gamma = h->opts.gamma;
    va.dstore = dstore;
    adj_degree(h->N, [&](auto Nc) { AL<decltype(Nc)::value>::adjoint(s ? s : h->stream, sa, va); });
}

int adj_status(tlw_handle* h) {
    TLW_ACUDA(h, cudaGetLastError());
    unsigned st = 0;
    TLW_ACUDA(h, cudaMemcpyAsync(&st, &h->d_step->status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    TLW_ACUDA(h, cudaStreamSynchronize(h->stream));
    if (st) {
        const unsigned zero = 0;
        TLW_ACUDA(h, upload_on(h->stream, &h->d_step->status, &zero, sizeof(zero)));
        return afail(h, TLW_E_NONADMISSIBLE, "non-admissible state: square root of a negative number (DomainError)");
    }
    return TLW_OK;
}

// copies n doubles from a caller pointer (host or device) into device memory on the handle's stream
int copy_in(tlw_handle* h, double* dst, const double* src, size_t n, int where) {
    TLW_ACUDA(h, cudaMemcpyAsync(dst, src, n * sizeof(double),
                                 where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 h->stream));
    return TLW_OK;
}
int copy_out(tlw_handle* h, double* dst, const double* src, size_t n, int where) {
    TLW_ACUDA(h, cudaMemcpyAsync(dst, src, n * sizeof(double),
                                 where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                 h->stream));
    return TLW_OK;
}

// captures what body() enqueues on the handle's stream into exec (replaced if present)
template <class F>
int capture_graph(tlw_handle* h, cudaGraphExec_t& exec, F&& body, unsigned long long flags = 0) {
    if (exec) {
        cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    TLW_ACUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return afail(h, TLW_E_CUDA, std::string("adjoint graph capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&exec, g, flags);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
        exec = nullptr;
        return afail(h, TLW_E_CUDA, std::string("adjoint graph instantiate: ") + cudaGetErrorString(e2));
    }
    return TLW_OK;
}

}  // namespace

extern "C" {

int tlw_adjoint_step(tlw_handle* h, double* lam_out, const double* lam_in, const double* u, double dt,
                     int32_t where) {
    int rc = adj_ready(h);
    if (rc) return rc;
    if (!lam_out || !lam_in || !u) return afail(h, TLW_E_ARG, "null array");
    AdjointBuffers& A = h->adj;
    if ((rc = ensure_steps(h, 1, 1))) return rc;
    A.last_resident = false;   // segment buffer 0 is reused here
    const size_t ns = nstate(h);
    // u -> seg[0], lam_in -> lam[0], dt -> dts[0]
    if ((rc = ensure_given_dts(h, 1))) return rc;
    if ((rc = copy_in(h, A.d_seg, u, ns, where)) || (rc = copy_in(h, A.d_lam[0], lam_in, ns, where))) return rc;
    TLW_ACUDA(h, cudaMemcpyAsync(A.d_dts_given, &dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    // forward rhs for the U traces (du into lam[1] as scratch), then the adjoint; MDRK: the whole step (u*, both
    // stages' U traces)
    if (is_mdrk(h)) {
        enqueue_fixed_step(h, h->stream, A.d_seg, A.d_lam[1], A.d_segU, A.d_dts_given, nullptr, seg_ustar(h, 0, 0),
                           seg_trace2(h, 0, 0));
        enqueue_adjoint_step(h, A.d_seg, A.d_segU, A.d_dts_given, A.d_lam[0], A.d_lam[1], nullptr, nullptr,
                             seg_ustar(h, 0, 0), seg_trace2(h, 0, 0));
    } else {
        const VolArgs va = fwd_vol_args(h, A.d_seg, A.d_lam[1], A.d_segU, A.d_dts_given);
        adj_degree(h->N, [&](auto Nc) { AL<decltype(Nc)::value>::forward_volume(h->stream, MODE_RHS, va); });
        enqueue_adjoint_step(h, A.d_seg, A.d_segU, A.d_dts_given, A.d_lam[0], A.d_lam[1]);
    }
    if ((rc = copy_out(h, lam_out, A.d_lam[1], ns, where))) return rc;
    return adj_status(h);
}

int tlw_solve_dts(tlw_handle* h, const double* u0, int32_t nsteps, const double* dts, double* uT_out,
                  int32_t where) {
    int rc = adj_ready(h);
    if (rc) return rc;
    if (!u0 || !uT_out || (nsteps > 0 && !dts) || nsteps < 0) return afail(h, TLW_E_ARG, "arguments");
    // dt array of nsteps, one trace buffer; no checkpoints
    if ((rc = ensure_steps(h, 1, 1))) return rc;
    AdjointBuffers& A = h->adj;
    A.last_resident = false;   // segment buffer 0's first trace is reused here
    if ((rc = ensure_given_dts(h, nsteps))) return rc;
    const size_t ns = nstate(h);
    if ((rc = copy_in(h, A.d_lam[0], u0, ns, where))) return rc;
    if (nsteps) TLW_ACUDA(h, cudaMemcpyAsync(A.d_dts_given, dts, nsteps * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    int cur = 0;
    for (int k = 0; k < nsteps; ++k) {
        enqueue_fixed_step(h, h->stream, A.d_lam[cur], A.d_lam[1 - cur], A.d_segU, A.d_dts_given + k);
        cur ^= 1;
    }
    if ((rc = copy_out(h, uT_out, A.d_lam[cur], ns, where))) return rc;
    return adj_status(h);
}

int tlw_forward_record(tlw_handle* h, const double* u0, int32_t nsteps, double cfl, int32_t checkpoint_every,
                       double* uT_out, int32_t where) {
    int rc = adj_ready(h);
    if (rc) return rc;
    if (!u0 || nsteps < 1 || checkpoint_every < 1 || !(cfl > 0.0)) return afail(h, TLW_E_ARG, "arguments");
    const int ck = std::min<int>(checkpoint_every, nsteps);
    if ((rc = ensure_steps(h, nsteps, ck))) return rc;
    AdjointBuffers& A = h->adj;
    A.rec_steps = 0;
    A.last_resident = false;
    const size_t ns = nstate(h);
    const int nseg = (nsteps + ck - 1) / ck;
    const int last = (nseg - 1) * ck, bl = (nseg - 1) & 1;
    // CFL dt recorded per step, checkpoints every ck steps; runs in the handle's two state buffers, except the
    // last segment, whose states, U traces and stage derivatives go straight into its segment buffer (the
    // reverse sweep starts there without recomputing it)
    StepState st{};
    st.t = 0.0;
    st.t_end = INFINITY;
    st.cfl = cfl;
    TLW_ACUDA(h, cudaMemcpyAsync(h->d_step, &st, sizeof(st), cudaMemcpyHostToDevice, h->stream));
    if ((rc = copy_in(h, last == 0 ? seg_state(h, bl, 0) : h->d_state[0], u0, ns, where))) return rc;
    h->slots_valid = false;   // the handle's state buffers are reused here
    // the whole sweep is one CUDA graph, captured once per (nsteps, checkpoint interval, buffers)
    auto body = [&]() -> int {
        double* s0 = h->d_state[0];
        double* s1 = h->d_state[1];
        for (int k = 0; k < nsteps; ++k) {
            const bool in_last = k >= last;
            const int j = k - last;
            double* u = in_last ? seg_state(h, bl, j) : s0;
            if (k % ck == 0)
                TLW_ACUDA(h, cudaMemcpyAsync(A.d_ckpt + (size_t)(k / ck) * ns, u, ns * sizeof(double),
                                             cudaMemcpyDeviceToDevice, h->stream));
            adj_degree(h->N, [&](auto Nc) { AL<decltype(Nc)::value>::speed(h->stream, h, u); });
            finalize_dt_kernel<<<1, 1, 0, h->stream>>>(h->d_step, h->n);
            TLW_ACUDA(h, cudaMemcpyAsync(A.d_dts + k, &h->d_step->dt, sizeof(double), cudaMemcpyDeviceToDevice,
                                         h->stream));
            if (in_last) {
                enqueue_fixed_step(h, h->stream, u, seg_state(h, bl, j + 1), seg_trace(h, bl, j), A.d_dts + k,
                                   seg_D(h, bl, j), seg_ustar(h, bl, j), seg_trace2(h, bl, j));
            } else {
                enqueue_fixed_step(h, h->stream, s0, k + 1 == last ? seg_state(h, bl, 0) : s1, h->d_tU, A.d_dts + k);
                std::swap(s0, s1);
            }
        }
        return TLW_OK;
    };
    const long long key = (long long)nsteps * 100003 + ck;
    if (!A.g_fwd || A.g_fwd_key != key) {
        if ((rc = capture_graph(h, A.g_fwd, body))) return rc;
        A.g_fwd_key = key;
    }
    TLW_ACUDA(h, cudaGraphLaunch(A.g_fwd, h->stream));
    A.d_final = seg_state(h, bl, nsteps - last);
    if (uT_out && (rc = copy_out(h, uT_out, A.d_final, ns, where))) return rc;
    if ((rc = adj_status(h))) return rc;
    A.rec_steps = nsteps;
    A.rec_ck = ck;
    A.last_resident = true;
    return TLW_OK;
}

namespace {

// reverse sweep of the recorded run, starting from the adjoint in A.d_lam[cur]; cur ends at the buffer
// that holds the gradient
int reverse_sweep_enqueue(tlw_handle* h, int& cur, double* phase_ms);

int reverse_sweep(tlw_handle* h, int& cur, double* phase_ms) {
    AdjointBuffers& A = h->adj;
    const int nseg = (A.rec_steps + A.rec_ck - 1) / A.rec_ck;
    int rc = TLW_OK;
    if (phase_ms) {
        rc = reverse_sweep_enqueue(h, cur, phase_ms);
    } else {
        const long long key = ((long long)A.rec_steps * 100003 + A.rec_ck) * 2 + (A.last_resident ? 1 : 0);
        if (cur != 0) return afail(h, TLW_E_ARG, "internal: sweep start buffer");
        if (!A.g_rev || A.g_rev_key != key) {
            int c = 0;
            // the kernels keep the priorities of the streams they were captured from
            rc = capture_graph(h, A.g_rev, [&]() { return reverse_sweep_enqueue(h, c, nullptr); },
                               cudaGraphInstantiateFlagUseNodePriority);
            if (rc) return rc;
            A.g_rev_key = key;
        }
        TLW_ACUDA(h, cudaGraphLaunch(A.g_rev, h->stream));
        cur = A.rec_steps % 2;
    }
    // with three or more segments the sweep has reused the last segment's buffer
    if (nseg > 2) A.last_resident = false;
    return rc;
}

// The segments from last to first: segment k's states, U traces and stage derivatives are recomputed from
// its checkpoint into buffer k & 1, then its adjoint steps run backwards over them. Without phase timing the
// recomputations run on their own stream (s_rec), one segment ahead of the adjoint chain (s_adj, highest
// priority), both forked from and joined back into the handle's stream: "ready" events order each segment's
// adjoint after its recompute and "free" events each buffer's reuse after the adjoint that read it. With phase
// timing everything runs in the same order on the handle's stream.
int reverse_sweep_enqueue(tlw_handle* h, int& cur, double* phase_ms) {
    AdjointBuffers& A = h->adj;
    const int nsteps = A.rec_steps, ck = A.rec_ck;
    const int nseg = (nsteps + ck - 1) / ck;
    const bool overlap = phase_ms == nullptr;
    const bool resident = A.last_resident;
    cudaStream_t sa = overlap ? A.s_adj : h->stream, sr = overlap ? A.s_rec : h->stream;
    cudaEvent_t ev[2] = {};
    if (!overlap)
        for (auto& x : ev) TLW_ACUDA(h, cudaEventCreate(&x));
    float rec_ms = 0.0f, adj_ms = 0.0f;
    auto timed = [&](float& acc, auto&& enqueue) -> int {
        if (overlap) return enqueue();
        cudaEventRecord(ev[0], sa);
        const int rc = enqueue();
        cudaEventRecord(ev[1], sa);
        TLW_ACUDA(h, cudaEventSynchronize(ev[1]));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        acc += ms;
        return rc;
    };
    bool used[2] = {false, false};
    auto recompute = [&](int sgi) -> int {
        if (resident && sgi == nseg - 1) return TLW_OK;
        const int b = sgi & 1, start = sgi * ck, len = std::min(ck, nsteps - start);
        return timed(rec_ms, [&]() -> int {
            if (overlap && used[b]) TLW_ACUDA(h, cudaStreamWaitEvent(sr, A.ev_free[b], 0));
            TLW_ACUDA(h, cudaMemcpyAsync(seg_state(h, b, 0), A.d_ckpt + (size_t)sgi * nstate(h),
                                         nstate(h) * sizeof(double), cudaMemcpyDeviceToDevice, sr));
            for (int j = 0; j < len; ++j) {
                if (j + 1 < len || is_mdrk(h)) {
                    // (MDRK: the last step too, for its u* and both stages' traces; its output goes to the spare slot)
                    enqueue_fixed_step(h, sr, seg_state(h, b, j), seg_state(h, b, j + 1), seg_trace(h, b, j),
                                       A.d_dts + start + j, seg_D(h, b, j), seg_ustar(h, b, j), seg_trace2(h, b, j));
                } else {
                    // the segment's output state is not needed, only the U traces and stage derivatives of its
                    // last step (volume kernel alone, its du into the free state slot)
                    VolArgs va = fwd_vol_args(h, seg_state(h, b, j), seg_state(h, b, len), seg_trace(h, b, j),
                                              A.d_dts + start + j);
                    va.dstore = seg_D(h, b, j);
                    adj_degree(h->N, [&](auto Nc) { AL<decltype(Nc)::value>::forward_volume(sr, MODE_RHS, va); });
                }
            }
            if (overlap) TLW_ACUDA(h, cudaEventRecord(A.ev_ready[b], sr));
            return TLW_OK;
        });
    };
    auto adjoint = [&](int sgi) -> int {
        const int b = sgi & 1, start = sgi * ck, len = std::min(ck, nsteps - start);
        return timed(adj_ms, [&]() -> int {
            if (overlap && !(resident && sgi == nseg - 1)) TLW_ACUDA(h, cudaStreamWaitEvent(sa, A.ev_ready[b], 0));
            for (int j = len - 1; j >= 0; --j) {
                enqueue_adjoint_step(h, seg_state(h, b, j), seg_trace(h, b, j), A.d_dts + start + j, A.d_lam[cur],
                                     A.d_lam[1 - cur], seg_D(h, b, j), sa, seg_ustar(h, b, j), seg_trace2(h, b, j));
                cur ^= 1;
            }
            if (overlap) TLW_ACUDA(h, cudaEventRecord(A.ev_free[b], sa));
            used[b] = true;
            return TLW_OK;
        });
    };
    int rc = TLW_OK;
    if (overlap) {
        TLW_ACUDA(h, cudaEventRecord(A.ev_fork, h->stream));
        TLW_ACUDA(h, cudaStreamWaitEvent(sr, A.ev_fork, 0));
        TLW_ACUDA(h, cudaStreamWaitEvent(sa, A.ev_fork, 0));
    }
    rc = recompute(nseg - 1);
    for (int k = nseg - 1; k >= 0 && !rc; --k) {
        if (k >= 1) rc = recompute(k - 1);
        if (!rc) rc = adjoint(k);
    }
    if (overlap) {
        // both streams rejoin the handle's stream
        TLW_ACUDA(h, cudaEventRecord(A.ev_join, sr));
        TLW_ACUDA(h, cudaEventRecord(A.ev_join2, sa));
        TLW_ACUDA(h, cudaStreamWaitEvent(h->stream, A.ev_join, 0));
        TLW_ACUDA(h, cudaStreamWaitEvent(h->stream, A.ev_join2, 0));
    }
    if (!overlap) {
        phase_ms[0] = rec_ms;
        phase_ms[1] = adj_ms;
        for (auto& x : ev) cudaEventDestroy(x);
    }
    return rc;
}

}  // namespace

int tlw_adjoint_sweep(tlw_handle* h, const double* lam_T, double* grad_out, int32_t where, double* phase_ms) {
    int rc = adj_ready(h);
    if (rc) return rc;
    if (!lam_T || !grad_out) return afail(h, TLW_E_ARG, "null array");
    if (h->adj.rec_steps < 1) return afail(h, TLW_E_STATE, "no recorded forward run: call tlw_forward_record first");
    const size_t ns = nstate(h);
    if ((rc = copy_in(h, h->adj.d_lam[0], lam_T, ns, where))) return rc;
    int cur = 0;
    if ((rc = reverse_sweep(h, cur, phase_ms))) return rc;
    if ((rc = copy_out(h, grad_out, h->adj.d_lam[cur], ns, where))) return rc;
    return adj_status(h);
}

int tlw_adjoint_solve(tlw_handle* h, const double* u0, int32_t nsteps, double cfl, int32_t checkpoint_every,
                      const double* rho_target, double* grad_out, double* J_out, double* uT_out, int32_t where,
                      double* phase_ms) {
    if (!h || !rho_target || !grad_out) return TLW_E_ARG;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (phase_ms) {
        TLW_ACUDA(h, cudaEventCreate(&e0));
        TLW_ACUDA(h, cudaEventCreate(&e1));
        TLW_ACUDA(h, cudaSetDevice(h->device));
        cudaEventRecord(e0, h->stream);
    }
    int rc = tlw_forward_record(h, u0, nsteps, cfl, checkpoint_every, uT_out, where);
    if (rc) return rc;
    AdjointBuffers& A = h->adj;
    const long long nodes = (long long)h->nn * h->E;
    const int blocks = (int)((nodes + OBJ_THREADS - 1) / OBJ_THREADS);
    double* d_target = A.d_bF;   // staged in the trace-adjoint buffer, which the sweep overwrites later
    if ((size_t)nodes > ntrace(h)) return afail(h, TLW_E_ARG, "internal: target staging");
    if ((rc = copy_in(h, d_target, rho_target, (size_t)nodes, where))) return rc;
    objective_kernel<<<blocks, OBJ_THREADS, 0, h->stream>>>(A.d_final, d_target, nodes, A.d_work, A.d_lam[0]);
    sum_kernel<<<1, OBJ_THREADS, 0, h->stream>>>(A.d_work, blocks, A.d_work + blocks);
    double J = 0.0;
    TLW_ACUDA(h, cudaMemcpyAsync(&J, A.d_work + blocks, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (phase_ms) cudaEventRecord(e1, h->stream);
    int cur = 0;
    if ((rc = reverse_sweep(h, cur, phase_ms ? phase_ms + 1 : nullptr))) return rc;
    if ((rc = copy_out(h, grad_out, A.d_lam[cur], nodes * NV, where))) return rc;
    rc = adj_status(h);
    if (J_out) *J_out = J;
    if (phase_ms) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        phase_ms[0] = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return rc;
}

int tlw_adjoint_dt_sequence(tlw_handle* h, double* dts, int32_t n) {
    if (!h || !dts || n < 0) return TLW_E_ARG;
    if (n > h->adj.capacity_steps || !h->adj.d_dts) return afail(h, TLW_E_STATE, "no recorded dt sequence of that length");
    TLW_ACUDA(h, cudaMemcpyAsync(dts, h->adj.d_dts, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TLW_ACUDA(h, cudaStreamSynchronize(h->stream));
    return TLW_OK;
}

}  // extern "C"
