// tlw_device.cuh -- device-side building blocks shared by the LW / MDRK kernels (FP64, sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tlw {

constexpr int NV = 4;   // compressible Euler 2D: rho, rho v1, rho v2, rho e

// status bits written by kernels (never a trap): the host maps them to TLW_E_* codes
constexpr unsigned STATUS_NONADMISSIBLE = 1u;   // sqrt of a negative number (reference: DomainError)

struct Basis {
    double D[16 * 16];      // derivative matrix, D[a*n + b] = l_b'(x_a)
    double Dhat[16 * 16];   // -M^{-1} D^T M
    double Vinv[16 * 16];   // inverse Legendre Vandermonde (nodal -> normalised modal), row-major
    double weights[16];
    double inv_w_first, inv_w_last;
};

// Derivative matrices per degree (index N), row-major n x n in 64 slots. Static: every translation unit
// that launches these kernels uploads its copy with upload_const_basis() on each device it uses.
static __constant__ double c_tlw_D[8][64];
static __constant__ double c_tlw_Dhat[8][64];
static __constant__ double c_tlw_Vinv[8][64];
static __constant__ double c_tlw_w[8][8];       // GLL weights
// D and Dhat in even-odd form (both are centro-antisymmetric on the symmetric GLL nodes: M[n-1-o][n-1-k] =
// -M[o][k]), for the line contractions of n >= 5 nodes; with h = n / 2, per matrix:
//   [0, h*h)        A[o][k] = (M[o][k] + M[o][n-1-k]) / 2      (o, k < h)
//   [h*h, 2h*h)     B[o][k] = (M[o][k] - M[o][n-1-k]) / 2
//   [2h*h, 2h*h+h)  M[o][h]                                    (odd n: the middle column)
//   [2h*h+h, ...)   M[h][k]                                    (odd n: the middle row)
// so that, with s_k = a_k + a_{n-1-k} and d_k = a_k - a_{n-1-k}, (M a)_o = A s + B d (+ M[o][h] a_h) and
// (M a)_{n-1-o} = B d - A s (- M[o][h] a_h): 2 h^2 + 2h multiply-adds per line instead of n^2 (Kopriva,
// Implementing Spectral Methods for PDEs, 2009, even-odd decomposition of the derivative matrix).
static __constant__ double c_tlw_D_eo[8][64];
static __constant__ double c_tlw_Dhat_eo[8][64];

static inline void even_odd_form(const double* M, int n, double* out) {
    const int h = n / 2;
    for (int o = 0; o < h; ++o)
        for (int k = 0; k < h; ++k) {
            out[o * h + k] = 0.5 * (M[o * n + k] + M[o * n + n - 1 - k]);
            out[h * h + o * h + k] = 0.5 * (M[o * n + k] - M[o * n + n - 1 - k]);
        }
    if (n % 2) {
        for (int o = 0; o < h; ++o) out[2 * h * h + o] = M[o * n + h];
        for (int k = 0; k < h; ++k) out[2 * h * h + h + k] = M[h * n + k];
    }
}

static inline cudaError_t upload_const_basis(const Basis* bases /* [8], index = N */) {
    static double d[8][64], dh[8][64], vi[8][64], w[8][8], deo[8][64], dheo[8][64];
    for (int N = 0; N < 8; ++N) {
        for (int k = 0; k < 64; ++k) {
            d[N][k] = bases[N].D[k];
            dh[N][k] = bases[N].Dhat[k];
            vi[N][k] = bases[N].Vinv[k];
        }
        for (int k = 0; k < 8; ++k) w[N][k] = bases[N].weights[k];
        const int n = N + 1;
        for (int k = 0; k < 64; ++k) deo[N][k] = dheo[N][k] = 0.0;
        if (n * n <= 64) {
            even_odd_form(d[N], n, deo[N]);
            even_odd_form(dh[N], n, dheo[N]);
        }
    }
    cudaError_t e = cudaMemcpyToSymbol(c_tlw_D, d, sizeof(d));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tlw_Dhat, dh, sizeof(dh));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tlw_Vinv, vi, sizeof(vi));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tlw_w, w, sizeof(w));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tlw_D_eo, deo, sizeof(deo));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tlw_Dhat_eo, dheo, sizeof(dheo));
    return e;
}

// Reciprocal by refinement of the hardware approximation (rcp.approx.ftz.f64, about 20 correct bits).
// With e = 1 - x y the exact reciprocal is y / (1 - e) = y (1 + e + e^2 + ...). TLW_RCP_CUBIC = 1 takes the
// series to e^2 in one step, y <- y + y (e + e^2), which cubes the relative error (third-order iteration; J.-M.
// Muller et al., Handbook of Floating-Point Arithmetic, 2010, ch. 5); 0 takes two Newton-Raphson steps
// y <- y + y e, which square it twice (P. Markstein, IBM J. Res. Dev. 34 (1990) 111-119). Either way the
// result is within one ulp of 1/x for normal x; no branch, 1 MUFU + 3 (or 4) DFMA instead of a correctly
// rounded divide.
#ifndef TLW_RCP_CUBIC
#define TLW_RCP_CUBIC 1
#endif
__device__ __forceinline__ double nr_reciprocal(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
#if TLW_RCP_CUBIC
    return fma(y, fma(e, e, e), y);
#else
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
#endif
}

// Euler flux pair (Trixi flux(u, 1|2, eq) for CompressibleEulerEquations2D) from 1/rho; ~17 flops.
__device__ __forceinline__ void euler_fluxes_ir(double gm1, double ir, double m1, double m2, double e, double* f,
                                                double* g) {
    const double v1 = m1 * ir, v2 = m2 * ir;
    const double p = gm1 * (e - 0.5 * (m1 * v1 + m2 * v2));
    const double ep = e + p;
    f[0] = m1;
    f[1] = m1 * v1 + p;
    f[2] = m1 * v2;
    f[3] = ep * v1;
    g[0] = m2;
    g[1] = f[2];
    g[2] = m2 * v2 + p;
    g[3] = ep * v2;
}
// the same from rho: 1 reciprocal
__device__ __forceinline__ void euler_fluxes(double gm1, double r, double m1, double m2, double e, double* f,
                                             double* g) {
    euler_fluxes_ir(gm1, nr_reciprocal(r), m1, m2, e, f, g);
}

__device__ __forceinline__ void euler_flux_dir(double gm1, const double* u, int orientation, double* fo) {
    double f[NV], g[NV];
    euler_fluxes(gm1, u[0], u[1], u[2], u[3], f, g);
#pragma unroll
    for (int v = 0; v < NV; ++v) fo[v] = orientation == 1 ? f[v] : g[v];
}

// sqrt that flags a negative argument instead of trapping
// Julia min: a NaN argument propagates (fmin would drop it)
__device__ __forceinline__ double julia_min(double a, double b) {
    return a != a ? a : (b != b ? b : fmin(a, b));
}

__device__ __forceinline__ double checked_sqrt(double x, unsigned* status) {
    if (!(x >= 0.0)) atomicOr(status, STATUS_NONADMISSIBLE);
    return sqrt(x);
}

// Trixi max_abs_speeds: |v1| + c and |v2| + c of a state, computed the same way by every CFL pass
__device__ __forceinline__ void node_speeds(double gamma, const double* x, unsigned* status, double& l1, double& l2) {
    const double ir = 1.0 / x[0];
    const double v1 = x[1] * ir, v2 = x[2] * ir;
    const double p = (gamma - 1.0) * (x[3] - 0.5 * (x[1] * v1 + x[2] * v2));
    const double c = checked_sqrt(gamma * p * ir, status);
    l1 = fabs(v1) + c;
    l2 = fabs(v2) + c;
}

// Per-element CFL slots written by the kernels that produce the final values of a step (plain LW on a
// periodic conforming TreeMesh): slot s of element e holds the bits of max(|v1| + c) and max(|v2| + c) over
// the nodes finalised there: 0 interior (volume kernel); 1 all face nodes (the element-centric surface pass),
// or with the interface sweeps 1 / 2 the -x / +x face without corners (x interfaces), 3 / 4 the -y / +y face
// with corners (y interfaces). The next step reduces them instead of reading the whole state again.
constexpr int CFL_SLOTS = 10;

// Trixi max_abs_speed_naive (kind 0) / max_abs_speed (kind 1) for CompressibleEulerEquations2D
__device__ __forceinline__ double max_abs_speed(double gamma, const double* ul, const double* ur, int orientation,
                                                int kind, unsigned* status) {
    const double gm1 = gamma - 1.0;
    const double irl = 1.0 / ul[0], irr = 1.0 / ur[0];
    const double v1l = ul[1] * irl, v2l = ul[2] * irl, v1r = ur[1] * irr, v2r = ur[2] * irr;
    const double pl = gm1 * (ul[3] - 0.5 * (ul[1] * v1l + ul[2] * v2l));
    const double pr = gm1 * (ur[3] - 0.5 * (ur[1] * v1r + ur[2] * v2r));
    const double vl = orientation == 1 ? v1l : v2l;
    const double vr = orientation == 1 ? v1r : v2r;
    const double cl = checked_sqrt(gamma * pl * irl, status);
    const double cr = checked_sqrt(gamma * pr * irr, status);
    if (kind == 0) return fmax(fabs(vl), fabs(vr)) + fmax(cl, cr);
    return fmax(fabs(vl) + cl, fabs(vr) + cr);
}

// Trixi min_max_speed_naive (FluxHLL default)
__device__ __forceinline__ void min_max_speed(double gamma, const double* ul, const double* ur, int orientation,
                                              double* lmin, double* lmax, unsigned* status) {
    const double gm1 = gamma - 1.0;
    const double irl = 1.0 / ul[0], irr = 1.0 / ur[0];
    const double v1l = ul[1] * irl, v2l = ul[2] * irl, v1r = ur[1] * irr, v2r = ur[2] * irr;
    const double pl = gm1 * (ul[3] - 0.5 * (ul[1] * v1l + ul[2] * v2l));
    const double pr = gm1 * (ur[3] - 0.5 * (ur[1] * v1r + ur[2] * v2r));
    const double vl = orientation == 1 ? v1l : v2l;
    const double vr = orientation == 1 ? v1r : v2r;
    *lmin = vl - checked_sqrt(gamma * pl * irl, status);
    *lmax = vr + checked_sqrt(gamma * pr * irr, status);
}

// The 8-argument LW surface flux as TreeMesh calls it: surface_flux(f_ll, f_rr, U_ll, U_rr, u_ll, u_rr).
// Rusanov (FluxPlusDissipation + DissipationLocalLaxFriedrichs): lambda from arguments 3/4, jump in 5/6.
// HLL (FluxHLL LW method): speeds from arguments 5/6, jump in 3/4.
__device__ __forceinline__ void lw_surface_flux(double gamma, int flux_kind, int speed_kind, const double* fl,
                                                const double* fr, const double* a3, const double* a4,
                                                const double* a5, const double* a6, int orientation, double* out,
                                                unsigned* status) {
    if (flux_kind == 0) {
        const double lambda = max_abs_speed(gamma, a3, a4, orientation, speed_kind, status);
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v] = 0.5 * (fl[v] + fr[v]) + (-0.5 * lambda * (a6[v] - a5[v]));
    } else {
        double lmin, lmax;
        min_max_speed(gamma, a5, a6, orientation, &lmin, &lmax, status);
        if (lmin >= 0 && lmax >= 0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) out[v] = fl[v];
        } else if (lmax <= 0 && lmin <= 0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) out[v] = fr[v];
        } else {
            const double inv = 1.0 / (lmax - lmin);
            const double cll = lmax * inv, crr = lmin * inv, cd = lmin * lmax * inv;
#pragma unroll
            for (int v = 0; v < NV; ++v) out[v] = cll * fl[v] - crr * fr[v] + cd * (a4[v] - a3[v]);
        }
    }
}

// Set-up copies ordered on a library stream and complete on return. A plain cudaMemcpy / cudaMemset runs on
// the legacy default stream, which the library's non-blocking streams do not wait for, and a pageable
// host-to-device cudaMemcpy may return before its DMA has landed.
inline cudaError_t upload_on(cudaStream_t s, void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}
inline cudaError_t download_on(cudaStream_t s, void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}
inline cudaError_t zero_on(cudaStream_t s, void* dst, size_t bytes) {
    cudaError_t e = cudaMemsetAsync(dst, 0, bytes, s);
    return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

__device__ __forceinline__ void load4(const double* __restrict__ p, double* x) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
}
__device__ __forceinline__ void load4_rw(const double* p, double* x) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *(reinterpret_cast<const double2*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
}
__device__ __forceinline__ void store4(double* p, const double* x) {
    reinterpret_cast<double2*>(p)[0] = make_double2(x[0], x[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(x[2], x[3]);
}
// One 256-bit access per 4-double node record (global memory only; the record 32-byte aligned): the surface
// pass, the interface sweeps, the curvilinear interfaces, the CFL / indicator passes and the adjoint kernels,
// whose arrays are the library's own or were checked (or copied) by the entry point.
__device__ __forceinline__ void load4w(const double* __restrict__ p, double* x) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(x[0]), "=d"(x[1]), "=d"(x[2]), "=d"(x[3]) : "l"(p));
}
__device__ __forceinline__ void load4w_rw(const double* p, double* x) {
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(x[0]), "=d"(x[1]), "=d"(x[2]), "=d"(x[3])
                 : "l"(p)
                 : "memory");
}
__device__ __forceinline__ void store4w(double* p, const double* x) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(x[0]), "d"(x[1]), "d"(x[2]), "d"(x[3])
                 : "memory");
}
// streaming store: the output is not re-read by this kernel
__device__ __forceinline__ void store4_cs(double* p, const double* x) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(x[0], x[1]));
    __stcs(reinterpret_cast<double2*>(p) + 1, make_double2(x[2], x[3]));
}

}  // namespace tlw
