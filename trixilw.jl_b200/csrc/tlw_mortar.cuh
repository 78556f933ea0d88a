// tlw_mortar.cuh -- L2 mortars of a non-conforming TreeMesh{2} (one large face against two half-size faces,
// as an AMR step leaves them), with the LW face traces: prolong2mortars! / calc_mortar_flux!
// (src/solvers/dgsem_tree/dg_2d.jl:1456-1646) and Trixi's mortar_fluxes_to_elements!, fused with the surface
// lift and apply_jacobian like the interface kernels.
//
// One group of 2n threads per mortar: thread (half, l) takes the small element's face traces u, U, F.n at
// face index l, interpolates the large element's traces onto that node (forward operator of the half),
// evaluates the surface flux in the TreeMesh argument order (f, f, U, U, u, u) with the left side as _ll,
// lifts fstar into the small element's face node, and parks it in shared memory; then thread (0, m) lifts
// the L2 projection of both halves' fstar (reverse operators) into the large element's face node m.
// A launch takes the mortars of one orientation, after the interfaces of that orientation (corner nodes).
#pragma once
#include "tlw_basis.h"
#include "tlw_device.cuh"

namespace tlw {

// [N][0 forward_upper, 1 forward_lower, 2 reverse_upper, 3 reverse_lower][n x n]
static __constant__ double c_tlw_mortar[8][4][64];

static inline cudaError_t upload_const_mortar() {
    static double m[8][4][64];
    for (int N = 1; N <= 7; ++N) host_mortar_operators(N, m[N]);
    return cudaMemcpyToSymbol(c_tlw_mortar, m, sizeof(m));
}

struct MortarArgs {
    const double* u;          // state the jump is taken of [v, i, j, e]
    double* out;              // du (rhs) or the updated state (step)
    const double* tU;         // [v, l, face, e]
    const double* tF;         // normal flux traces [v, l, face, e]
    const int* lower;         // mortars of this orientation (0-based elements)
    const int* upper;
    const int* large;
    const int* large_side;    // 1: large element on the -side, 2: on the +side
    int count;
    int orientation;
    const double* inv_jac;    // [e]
    const double* dt;
    int step_mode;
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
};

template <int N>
struct MortarCfg {
    static constexpr int n = N + 1;
    static constexpr int GROUP = 2 * n;                 // threads per mortar
    static constexpr int PER_CTA = 128 / GROUP;         // mortars per CTA
    static constexpr int THREADS = PER_CTA * GROUP;
};

__device__ __forceinline__ int tree_face_node(int n, int f, int l) {
    return f == 0 ? n * l : f == 1 ? (n - 1) + n * l : f == 2 ? l : l + n * (n - 1);
}

template <int N>
static __global__ void __launch_bounds__(128) mortar_kernel(MortarArgs a) {
    using C = MortarCfg<N>;
    constexpr int n = C::n;
    constexpr int nn = n * n;
    __shared__ double fs[C::PER_CTA][2][n][NV];
    const int g = threadIdx.x / C::GROUP;
    const int r = threadIdx.x - g * C::GROUP;
    const int h = r / n;          // 0: lower half, 1: upper half
    const int l = r - h * n;
    const int k = blockIdx.x * C::PER_CTA + g;
    const bool active = g < C::PER_CTA && k < a.count;
    const int o = a.orientation;
    int lg = 0, small_face = 0, large_face = 0;
    bool left = true;
    double dts = 0.0;
    if (active) {
        const int se = h ? __ldg(a.upper + k) : __ldg(a.lower + k);
        lg = __ldg(a.large + k);
        left = __ldg(a.large_side + k) == 1;
        small_face = left ? (o == 1 ? 0 : 2) : (o == 1 ? 1 : 3);
        large_face = left ? (o == 1 ? 1 : 3) : (o == 1 ? 0 : 2);
        const int ns = tree_face_node(n, small_face, l);
        double us[NV], Us[NV], Fs[NV], ul[NV] = {0, 0, 0, 0}, Ul[NV] = {0, 0, 0, 0}, Fl[NV] = {0, 0, 0, 0};
        load4(a.u + ((size_t)se * nn + ns) * NV, us);
        const size_t ts = (((size_t)se * 4 + small_face) * n + l) * NV;
        load4(a.tU + ts, Us);
        load4(a.tF + ts, Fs);
        const double* fwd = c_tlw_mortar[N][h ? 0 : 1];
#pragma unroll
        for (int j = 0; j < n; ++j) {
            double x[NV], y[NV], z[NV];
            load4(a.u + ((size_t)lg * nn + tree_face_node(n, large_face, j)) * NV, x);
            const size_t tl = (((size_t)lg * 4 + large_face) * n + j) * NV;
            load4(a.tU + tl, y);
            load4(a.tF + tl, z);
            const double c = fwd[l * n + j];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                ul[v] = fma(c, x[v], ul[v]);
                Ul[v] = fma(c, y[v], Ul[v]);
                Fl[v] = fma(c, z[v], Fl[v]);
            }
        }
        double fstar[NV];
        if (left) lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, Fl, Fs, Ul, Us, ul, us, o, fstar, a.status);
        else lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, Fs, Fl, Us, Ul, us, ul, o, fstar, a.status);
        dts = a.step_mode ? *a.dt : 1.0;
        // small element: fstar is the flux along +x / +y through its face
        const double cs = left ? dts * __ldg(a.inv_jac + se) * a.inv_w_first : -dts * __ldg(a.inv_jac + se) * a.inv_w_last;
        double* os = a.out + ((size_t)se * nn + ns) * NV;
        double x[NV];
        load4_rw(os, x);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            x[v] = fma(cs, fstar[v], x[v]);
            fs[g][h][l][v] = fstar[v];
        }
        store4(os, x);
    }
    __syncthreads();
    if (active && h == 0) {
        const double* ru = c_tlw_mortar[N][2];
        const double* rl = c_tlw_mortar[N][3];
        double p[NV] = {0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < n; ++q)
#pragma unroll
            for (int v = 0; v < NV; ++v) p[v] = fma(ru[l * n + q], fs[g][1][q][v], fma(rl[l * n + q], fs[g][0][q][v], p[v]));
        const double cl = left ? -dts * __ldg(a.inv_jac + lg) * a.inv_w_last : dts * __ldg(a.inv_jac + lg) * a.inv_w_first;
        double* ol = a.out + ((size_t)lg * nn + tree_face_node(n, large_face, l)) * NV;
        double x[NV];
        load4_rw(ol, x);
#pragma unroll
        for (int v = 0; v < NV; ++v) x[v] = fma(cl, p[v], x[v]);
        store4(ol, x);
    }
}

}  // namespace tlw
