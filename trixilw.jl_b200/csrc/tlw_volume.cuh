// tlw_volume.cuh -- fused per-element LW / MDRK volume kernels for TreeMesh{2} (FP64, sm_100a).
//
// One thread per GLL node; EB whole elements per CTA so that every CTA runs (nearly) full warps (N=3: 8 x 16,
// N=4: 5 x 25 (+3 idle lanes), N=5: 7 x 36 (+4 idle lanes) nodes). The 1-D derivative contractions read the stage fluxes
// of the element from shared memory (tiles of double2: (f0,f1) (f2,f3) (g0,g1) (g2,g3) per node, a
// layout with no bank conflicts for the row and column reads). All other LW stage state (perturbed
// states u+-ut, u+-2ut, the time averages U, F, G) lives in registers. HBM traffic per element: read u
// once, write du (or u^{n+1}) once, write the face traces of U and F.n for the surface kernels.
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

template <int N>
struct VolCfg {
    static constexpr int n = N + 1;
    static constexpr int nn = n * n;
    // whole elements per CTA, chosen so that the CTA is (nearly) full warps
    static constexpr int EB = N == 1 ? 32 : N == 2 ? 14 : N == 3 ? 8 : N == 4 ? 5 : N == 5 ? 7 : N == 6 ? 5 : 2;
    static constexpr int THREADS = ((EB * nn + 31) / 32) * 32;
    // resident CTAs per SM the register allocation must allow (<= 128 registers per thread)
    static constexpr int MIN_BLOCKS = THREADS <= 128 ? 4 : 2;
    // the MDRK stage kernels hold fewer values per thread: ask for more resident CTAs
    static constexpr int MDRK_MIN_BLOCKS = THREADS <= 128 ? 6 : 3;
    static constexpr int TILE = EB * nn;   // double2 entries per tile array
    // shared memory: 4 stage matrices + Dhat (5 nn doubles, padded to 16 B) + NT tiles of 4 double2 arrays
    static constexpr int MAT_D2 = (5 * nn + 1) / 2;
    static constexpr size_t smem_bytes(int ntiles) {
        return (size_t)MAT_D2 * sizeof(double2) + (size_t)ntiles * 4 * TILE * sizeof(double2);
    }
};

enum VolMode { MODE_RHS = 0, MODE_STEP = 1 };

struct VolArgs {
    const double* u;        // state the stage fluxes are evaluated at  [v,i,j,e]
    const double* u_base;   // MODE_STEP: out = u_base + dt * du        [v,i,j,e]
    double* out;            // du (MODE_RHS) or the updated state (MODE_STEP)
    double* tU;             // face traces of U   [v, l, face, e]
    double* tF;             // face traces of F.n [v, l, face, e]
    double* U2;             // MDRK: stage-1 U2 [v,i,j,e] (written by stage 1, read by stage 2)
    double* F2;             // MDRK: stage-1 F2 [v,d,i,j,e]
    const double* inv_jac;  // [e]
    const double* dt;       // device scalar
    const Basis* basis;
    int E;
    double gamma;
};

// writes the four double values (a,b,c,d) of node slot s into tile t
template <int TILE>
__device__ __forceinline__ void tile_put(double2* tiles, int t, int s, const double* f, const double* g) {
    double2* T = tiles + t * 4 * TILE;
    T[s] = make_double2(f[0], f[1]);
    T[TILE + s] = make_double2(f[2], f[3]);
    T[2 * TILE + s] = make_double2(g[0], g[1]);
    T[3 * TILE + s] = make_double2(g[2], g[3]);
}
template <int TILE>
__device__ __forceinline__ void tile_get(const double2* tiles, int t, int s, double* f, double* g) {
    const double2* T = tiles + t * 4 * TILE;
    const double2 a = T[s], b = T[TILE + s], c = T[2 * TILE + s], d = T[3 * TILE + s];
    f[0] = a.x; f[1] = a.y; f[2] = b.x; f[3] = b.y;
    g[0] = c.x; g[1] = c.y; g[2] = d.x; g[3] = d.y;
}

// acc = sum_k M[i,k] f(k,j) + sum_k M[j,k] g(i,k) over the element whose first slot is `base`
template <int n, int TILE>
__device__ __forceinline__ void contract(const double2* tiles, int t, const double* M, int base, int i, int j,
                                         double* acc) {
    const double2* T = tiles + t * 4 * TILE;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
    for (int k = 0; k < n; ++k) {
        const double mx = M[i * n + k];
        const int sx = base + k + n * j;
        const double2 p = T[sx], q = T[TILE + sx];
        a0 = fma(mx, p.x, a0); a1 = fma(mx, p.y, a1); a2 = fma(mx, q.x, a2); a3 = fma(mx, q.y, a3);
        const double my = M[j * n + k];
        const int sy = base + i + n * k;
        const double2 r = T[2 * TILE + sy], s = T[3 * TILE + sy];
        a0 = fma(my, r.x, a0); a1 = fma(my, r.y, a1); a2 = fma(my, s.x, a2); a3 = fma(my, s.y, a3);
    }
    acc[0] = a0; acc[1] = a1; acc[2] = a2; acc[3] = a3;
}

// out/traces epilogue shared by all volume kernels. acc = Dhat-contraction of (F, G).
template <int n, int MODE>
__device__ __forceinline__ void volume_epilogue(const VolArgs& a, int e, int i, int j, int node, double ij, double dt,
                                                const double* acc, const double* U, const double* F,
                                                const double* G) {
    const size_t off = ((size_t)e * n * n + node) * NV;
    double o[NV];
    if (MODE == MODE_RHS) {
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = -ij * acc[v];
    } else {
        double ub[NV];
        load4(a.u_base + off, ub);
        const double s = -dt * ij;
#pragma unroll
        for (int v = 0; v < NV; ++v) o[v] = fma(s, acc[v], ub[v]);
    }
    store4(a.out + off, o);
    // face traces [v, l, face, e]; face 0 = -x, 1 = +x, 2 = -y, 3 = +y
    const size_t tb = (size_t)e * 4 * n * NV;
    if (i == 0) { store4(a.tU + tb + (0 * n + j) * NV, U); store4(a.tF + tb + (0 * n + j) * NV, F); }
    if (i == n - 1) { store4(a.tU + tb + (1 * n + j) * NV, U); store4(a.tF + tb + (1 * n + j) * NV, F); }
    if (j == 0) { store4(a.tU + tb + (2 * n + i) * NV, U); store4(a.tF + tb + (2 * n + i) * NV, G); }
    if (j == n - 1) { store4(a.tU + tb + (3 * n + i) * NV, U); store4(a.tF + tb + (3 * n + i) * NV, G); }
}

// ------------------------------------------------------------------------------------------------
// Plain LW volume kernel (depth = min(N, 4)).
// The finite-difference stencils are accumulated unscaled ("raw") and their constant factors are folded
// into the matrices of the next contraction and into the F/G update coefficients:
//   depth 4: f_t = raw1/12, f_tt = raw2/12, f_ttt = raw3/2, f_tttt = raw4/2
//   depth 3: f_t = raw1/12, f_tt = raw2,    f_ttt = raw3/2
//   depth 2: f_t = raw1/2,  f_tt = raw2;    depth 1: f_t = raw1/2
// Shared memory holds M_k = -dt c_k D for the contraction of stage k's output (c_0 = 1) and Dhat.
// ------------------------------------------------------------------------------------------------
template <int N, int MODE>
__global__ void __launch_bounds__(VolCfg<N>::THREADS, VolCfg<N>::MIN_BLOCKS) lw_volume_kernel(VolArgs a) {
    using C = VolCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, TILE = C::TILE;
    constexpr int DEPTH = N >= 4 ? 4 : N;
    constexpr double C1 = DEPTH >= 3 ? 1.0 / 12.0 : 0.5;
    constexpr double C2 = DEPTH == 4 ? 1.0 / 12.0 : 1.0;
    constexpr double C3 = 0.5;
    constexpr double C4 = 0.5;
    extern __shared__ double2 smem[];
    double* sM = reinterpret_cast<double*>(smem);   // [4][nn]: -dt D, -dt C1 D, -dt C2 D, -dt C3 D
    double* sDh = sM + 4 * nn;                      // Dhat
    double2* tiles = smem + C::MAT_D2;

    const int tid = threadIdx.x;
    const double dt = *a.dt;
    const double gm1 = a.gamma - 1.0;
    for (int k = tid; k < nn; k += blockDim.x) {
        const double d = -dt * a.basis->D[k];
        sM[k] = d;
        sM[nn + k] = d * C1;
        sM[2 * nn + k] = d * C2;
        sM[3 * nn + k] = d * C3;
        sDh[k] = a.basis->Dhat[k];
    }
    const int el = tid / nn;
    const int node = tid - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    const int base = el * nn;
    const int slot = base + node;

    double U[NV], F[NV], G[NV], up[NV], um[NV], upp[NV], umm[NV];
    double ij = 0.0;
    // stage 0: f, g at u (dg_2d.jl:941-971)
    if (active) {
        double uu[NV], f[NV], g[NV];
        load4(a.u + ((size_t)e * nn + node) * NV, uu);
        ij = __ldg(a.inv_jac + e);
        euler_fluxes(gm1, uu[0], uu[1], uu[2], uu[3], f, g);
        tile_put<TILE>(tiles, 0, slot, f, g);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            F[v] = f[v]; G[v] = g[v]; U[v] = uu[v];
            up[v] = um[v] = upp[v] = umm[v] = uu[v];
        }
    }
    __syncthreads();

    // stage 1: ut; perturbed states; f_t (dg_2d.jl:972-1023 / :725-775 / :543-582 / :417-454)
    if (active) {
        double d[NV], r[NV], q[NV], f[NV], g[NV];
        contract<n, TILE>(tiles, 0, sM, base, i, j, d);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            d[v] *= ij;
            U[v] = fma(0.5, d[v], U[v]);
            up[v] += d[v];
            um[v] -= d[v];
            if (DEPTH >= 3) { upp[v] = fma(2.0, d[v], upp[v]); umm[v] = fma(-2.0, d[v], umm[v]); }
        }
        if (DEPTH >= 3) {
            // raw1 = -f(u+2ut) + 8 f(u+ut) - 8 f(u-ut) + f(u-2ut)
            euler_fluxes(gm1, upp[0], upp[1], upp[2], upp[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = -f[v]; q[v] = -g[v]; }
            euler_fluxes(gm1, up[0], up[1], up[2], up[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(8.0, f[v], r[v]); q[v] = fma(8.0, g[v], q[v]); }
            euler_fluxes(gm1, um[0], um[1], um[2], um[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-8.0, f[v], r[v]); q[v] = fma(-8.0, g[v], q[v]); }
            euler_fluxes(gm1, umm[0], umm[1], umm[2], umm[3], f, g);
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
        if (DEPTH >= 2) tile_put<TILE>(tiles, 1, slot, r, q);
    }
    if (DEPTH >= 2) {
        __syncthreads();
        // stage 2: utt; f_tt (dg_2d.jl:1025-1083 / :777-831 / :597-634)
        if (active) {
            double d[NV], f0[NV], g0[NV], r[NV], q[NV], f[NV], g[NV];
            contract<n, TILE>(tiles, 1, sM + nn, base, i, j, d);
            tile_get<TILE>(tiles, 0, slot, f0, g0);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                d[v] *= ij;
                U[v] = fma(1.0 / 6.0, d[v], U[v]);
                up[v] = fma(0.5, d[v], up[v]);
                um[v] = fma(0.5, d[v], um[v]);
                if (DEPTH >= 3) { upp[v] = fma(2.0, d[v], upp[v]); umm[v] = fma(2.0, d[v], umm[v]); }
            }
            if (DEPTH == 4) {
                // raw2 = -f(upp) + 16 f(up) - 30 f0 + 16 f(um) - f(umm)
                euler_fluxes(gm1, upp[0], upp[1], upp[2], upp[3], f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    r[v] = fma(-30.0, f0[v], -f[v]);
                    q[v] = fma(-30.0, g0[v], -g[v]);
                }
                euler_fluxes(gm1, up[0], up[1], up[2], up[3], f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] = fma(16.0, f[v], r[v]); q[v] = fma(16.0, g[v], q[v]); }
                euler_fluxes(gm1, um[0], um[1], um[2], um[3], f, g);
#pragma unroll
                for (int v = 0; v < NV; ++v) { r[v] = fma(16.0, f[v], r[v]); q[v] = fma(16.0, g[v], q[v]); }
                euler_fluxes(gm1, umm[0], umm[1], umm[2], umm[3], f, g);
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
            if (DEPTH >= 3) tile_put<TILE>(tiles, 2, slot, r, q);
        }
    }
    if (DEPTH >= 3) {
        __syncthreads();
        // stage 3: uttt; f_ttt (dg_2d.jl:1085-1138 / :833-875)
        if (active) {
            double d[NV], r[NV], q[NV], f[NV], g[NV];
            contract<n, TILE>(tiles, 2, sM + 2 * nn, base, i, j, d);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                d[v] *= ij;
                U[v] = fma(1.0 / 24.0, d[v], U[v]);
                um[v] = fma(-1.0 / 6.0, d[v], um[v]);
                up[v] = fma(1.0 / 6.0, d[v], up[v]);
                umm[v] = fma(-4.0 / 3.0, d[v], umm[v]);
                upp[v] = fma(4.0 / 3.0, d[v], upp[v]);
            }
            // raw3 = f(upp) - 2 f(up) + 2 f(um) - f(umm)
            euler_fluxes(gm1, upp[0], upp[1], upp[2], upp[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = f[v]; q[v] = g[v]; }
            euler_fluxes(gm1, up[0], up[1], up[2], up[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-2.0, f[v], r[v]); q[v] = fma(-2.0, g[v], q[v]); }
            euler_fluxes(gm1, um[0], um[1], um[2], um[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(2.0, f[v], r[v]); q[v] = fma(2.0, g[v], q[v]); }
            euler_fluxes(gm1, umm[0], umm[1], umm[2], umm[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                r[v] -= f[v];
                q[v] -= g[v];
                F[v] = fma(C3 / 24.0, r[v], F[v]);
                G[v] = fma(C3 / 24.0, q[v], G[v]);
            }
            if (DEPTH >= 4) tile_put<TILE>(tiles, 1, slot, r, q);
        }
    }
    if (DEPTH >= 4) {
        __syncthreads();
        // stage 4: utttt; f_tttt (dg_2d.jl:1140-1206)
        if (active) {
            double d[NV], f0[NV], g0[NV], r[NV], q[NV], f[NV], g[NV];
            contract<n, TILE>(tiles, 1, sM + 3 * nn, base, i, j, d);
            tile_get<TILE>(tiles, 0, slot, f0, g0);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                d[v] *= ij;
                U[v] = fma(1.0 / 120.0, d[v], U[v]);
                um[v] = fma(1.0 / 24.0, d[v], um[v]);
                up[v] = fma(1.0 / 24.0, d[v], up[v]);
                umm[v] = fma(2.0 / 3.0, d[v], umm[v]);
                upp[v] = fma(2.0 / 3.0, d[v], upp[v]);
            }
            // raw4 = f(upp) - 4 f(up) + 6 f0 - 4 f(um) + f(umm)
            euler_fluxes(gm1, upp[0], upp[1], upp[2], upp[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(6.0, f0[v], f[v]); q[v] = fma(6.0, g0[v], g[v]); }
            euler_fluxes(gm1, up[0], up[1], up[2], up[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-4.0, f[v], r[v]); q[v] = fma(-4.0, g[v], q[v]); }
            euler_fluxes(gm1, um[0], um[1], um[2], um[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) { r[v] = fma(-4.0, f[v], r[v]); q[v] = fma(-4.0, g[v], q[v]); }
            euler_fluxes(gm1, umm[0], umm[1], umm[2], umm[3], f, g);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                r[v] += f[v];
                q[v] += g[v];
                F[v] = fma(C4 / 120.0, r[v], F[v]);
                G[v] = fma(C4 / 120.0, q[v], G[v]);
            }
            // tile 2 was last read by the stage-3 contraction, before the barrier above
            tile_put<TILE>(tiles, 2, slot, F, G);
        }
    }
    // final: Dhat contraction of the time-averaged fluxes
    constexpr int TF = DEPTH == 4 ? 2 : DEPTH == 3 ? 1 : DEPTH == 2 ? 2 : 1;
    if (DEPTH < 4) {
        __syncthreads();
        if (active) tile_put<TILE>(tiles, TF, slot, F, G);
    }
    __syncthreads();
    if (active) {
        double acc[NV];
        contract<n, TILE>(tiles, TF, sDh, base, i, j, acc);
        volume_epilogue<n, MODE>(a, e, i, j, node, ij, dt, acc, U, F, G);
    }
}

// ------------------------------------------------------------------------------------------------
// MDRK stage 1 (mdrk_kernel_1!, multi_derivative_2d.jl:263-421): F = f/2 + f_t/8, U = u/2 + u_t/8,
// F2 = f + f_t/6, U2 = u + u_t/6 (stored whole for stage 2).
// ------------------------------------------------------------------------------------------------
template <int N, int MODE>
__global__ void __launch_bounds__(VolCfg<N>::THREADS, VolCfg<N>::MDRK_MIN_BLOCKS) mdrk1_volume_kernel(VolArgs a) {
    using C = VolCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, TILE = C::TILE;
    extern __shared__ double2 smem[];
    double* sDm = reinterpret_cast<double*>(smem);
    double* sDh = sDm + 4 * nn;
    double2* tiles = smem + C::MAT_D2;
    const int tid = threadIdx.x;
    const double dt = *a.dt;
    const double gm1 = a.gamma - 1.0;
    for (int k = tid; k < nn; k += blockDim.x) {
        sDm[k] = -dt * a.basis->D[k];
        sDh[k] = a.basis->Dhat[k];
    }
    const int el = tid / nn;
    const int node = tid - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    const int base = el * nn;
    const int slot = base + node;
    double uu[NV], f0[NV], g0[NV], ij = 0.0;
    if (active) {
        load4(a.u + ((size_t)e * nn + node) * NV, uu);
        ij = __ldg(a.inv_jac + e);
        euler_fluxes(gm1, uu[0], uu[1], uu[2], uu[3], f0, g0);
        tile_put<TILE>(tiles, 0, slot, f0, g0);
    }
    __syncthreads();
    double U[NV], F[NV], G[NV];
    if (active) {
        double d[NV], ft[NV], gt[NV], f[NV], g[NV], s[NV];
        contract<n, TILE>(tiles, 0, sDm, base, i, j, d);
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v] *= ij;
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
        store4(a.U2 + off * NV, U2v);
        store4(a.F2 + off * 2 * NV, F2v);
        store4(a.F2 + off * 2 * NV + NV, G2v);
    }
    __syncthreads();
    if (active) tile_put<TILE>(tiles, 1, slot, F, G);
    __syncthreads();
    if (active) {
        double acc[NV];
        contract<n, TILE>(tiles, 1, sDh, base, i, j, acc);
        volume_epilogue<n, MODE>(a, e, i, j, node, ij, dt, acc, U, F, G);
    }
}

// ------------------------------------------------------------------------------------------------
// MDRK stage 2 (mdrk_kernel_2!, multi_derivative_2d.jl:423-555): at u* = a.u,
// F = F2 + f_t(u*)/3, U = U2 + u*_t/3.
// ------------------------------------------------------------------------------------------------
template <int N, int MODE>
__global__ void __launch_bounds__(VolCfg<N>::THREADS, VolCfg<N>::MDRK_MIN_BLOCKS) mdrk2_volume_kernel(VolArgs a) {
    using C = VolCfg<N>;
    constexpr int n = C::n, nn = C::nn, EB = C::EB, TILE = C::TILE;
    extern __shared__ double2 smem[];
    double* sDm = reinterpret_cast<double*>(smem);
    double* sDh = sDm + 4 * nn;
    double2* tiles = smem + C::MAT_D2;
    const int tid = threadIdx.x;
    const double dt = *a.dt;
    const double gm1 = a.gamma - 1.0;
    for (int k = tid; k < nn; k += blockDim.x) {
        sDm[k] = -dt * a.basis->D[k];
        sDh[k] = a.basis->Dhat[k];
    }
    const int el = tid / nn;
    const int node = tid - el * nn;
    const int i = node % n, j = node / n;
    const int e = blockIdx.x * EB + el;
    const bool active = el < EB && e < a.E;
    const int base = el * nn;
    const int slot = base + node;
    double us[NV], ij = 0.0;
    if (active) {
        double f[NV], g[NV];
        load4(a.u + ((size_t)e * nn + node) * NV, us);
        ij = __ldg(a.inv_jac + e);
        euler_fluxes(gm1, us[0], us[1], us[2], us[3], f, g);
        tile_put<TILE>(tiles, 0, slot, f, g);
    }
    __syncthreads();
    double U[NV], F[NV], G[NV];
    if (active) {
        double d[NV], ft[NV], gt[NV], f[NV], g[NV], s[NV];
        contract<n, TILE>(tiles, 0, sDm, base, i, j, d);
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v] *= ij;
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
        load4(a.U2 + off * NV, U2v);
        load4(a.F2 + off * 2 * NV, F2v);
        load4(a.F2 + off * 2 * NV + NV, G2v);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            ft[v] = (ft[v] + f[v]) * (1.0 / 12.0);
            gt[v] = (gt[v] + g[v]) * (1.0 / 12.0);
            F[v] = fma(1.0 / 3.0, ft[v], F2v[v]);
            G[v] = fma(1.0 / 3.0, gt[v], G2v[v]);
            U[v] = fma(1.0 / 3.0, d[v], U2v[v]);
        }
    }
    __syncthreads();
    if (active) tile_put<TILE>(tiles, 1, slot, F, G);
    __syncthreads();
    if (active) {
        double acc[NV];
        contract<n, TILE>(tiles, 1, sDh, base, i, j, acc);
        volume_epilogue<n, MODE>(a, e, i, j, node, ij, dt, acc, U, F, G);
    }
}

}  // namespace tlw
