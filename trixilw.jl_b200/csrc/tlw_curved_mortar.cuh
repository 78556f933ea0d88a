// tlw_curved_mortar.cuh -- L2 mortars of a curvilinear mesh (one large face against two half-size faces, as a
// P4estMesh{2} is after an AMR step), with the LW face traces as the reference's P4estMesh path has them:
// prolong2mortars! / calc_mortar_flux! (src/solvers/dgsem_p4est/dg_2d.jl:395-603) and Trixi's
// mortar_fluxes_to_elements!, fused with the surface lift and apply_jacobian like the interface kernels.
//
// A mortar is (small element at position 1, small element at position 2, their face; large element, its face,
// whether its face index runs backwards along the mortar); the small faces run forward. One group of 2n threads
// per mortar: thread (position, l) takes the small element's u, U and outward normal flux at face index l
// (outward normal sigma Ja^d of that node), interpolates the large element's u and U onto the node (forward
// operator of its position) and with them the large element's instantaneous flux Trixi.flux(u, -n_large / 2)
// (the reference overwrites the time-averaged normal flux of the large side with it, :455-458), evaluates the
// surface flux in the curvilinear argument order with the small side as _ll along the small element's normal,
// lifts it into the small element's face node and parks it in shared memory; then thread (1, i) lifts -2 times
// the L2 projection of both positions' fluxes (reverse operators) into the large element's face node.
// Launches take the mortars colour by colour (no element has faces of both classes in one colour).
//
// With shock capturing each small node's flux goes through get_blended_flux (dg_2d.jl:227-250, called at
// :589-593) with the small element as the primary: the first-order flux fn along the small element's normal at
// (u_small, interpolated u_large), fn_inner_ll the small element's fn_low slot of its face at the node,
// fn_inner_rr the large element's fn_low slot of its face read in mortar order (index i, not reversed) and
// interpolated like u (prolong2mortars!, :429-500), J^{-1} = lw_mortars.inverse_jacobian of the node.
#pragma once
#include "tlw_curved.cuh"
#include "tlw_mortar.cuh"
#include "tlw_volume.cuh"

namespace tlw {

struct CurvedMortarArgs {
    const double* u;          // [v, i, j, e]
    double* out;              // du (rhs) or the updated state (step)
    const double* tU;         // [v, l, face, e]
    const double* tF;         // contravariant flux traces [v, l, face, e]
    const double* metrics;    // [4, i, j, e]
    const double* inv_jac;    // [i, j, e]
    const int* small1;        // mortars of this colour (0-based elements)
    const int* small2;
    const int* large;
    const int* code;          // small face | large face << 2 | large reversed << 4
    int count;
    const double* dt;
    int step_mode;
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
    // shock capturing (null alpha: the plain LW flux)
    const double* alpha;      // [e]
    const double* tFn;        // fn_low slots [v, l, face, e]
    const double* mortar_ij;  // lw_mortars.inverse_jacobian of this colour's mortars [k][l]
    double w_first, w_last;
};

template <int N>
static __global__ void __launch_bounds__(128) curved_mortar_kernel(CurvedMortarArgs a) {
    using C = MortarCfg<N>;
    constexpr int n = C::n;
    constexpr int nn = n * n;
    __shared__ double fs[C::PER_CTA][2][n][NV];
    const int g = threadIdx.x / C::GROUP;
    const int r = threadIdx.x - g * C::GROUP;
    const int h = r / n;          // position - 1
    const int l = r - h * n;
    const int k = blockIdx.x * C::PER_CTA + g;
    const bool active = g < C::PER_CTA && k < a.count;
    const double gm1 = a.gamma - 1.0;
    int lg = 0, lf = 0;
    bool rev = false;
    double dts = 0.0;
    if (active) {
        const int code = __ldg(a.code + k);
        const int sf = code & 3;
        lf = (code >> 2) & 3;
        rev = (code >> 4) & 1;
        const int se = h ? __ldg(a.small2 + k) : __ldg(a.small1 + k);
        lg = __ldg(a.large + k);
        const int ns = face_node_index(n, sf, l);
        const double sgS = (sf & 1) ? 1.0 : -1.0, sgL = (lf & 1) ? 1.0 : -1.0;
        double us[NV], Us[NV], Fs[NV], ul[NV] = {0, 0, 0, 0}, Ul[NV] = {0, 0, 0, 0}, Fl[NV] = {0, 0, 0, 0}, J[4];
        load4(a.u + ((size_t)se * nn + ns) * NV, us);
        const size_t ts = (((size_t)se * 4 + sf) * n + l) * NV;
        load4(a.tU + ts, Us);
        load4(a.tF + ts, Fs);
#pragma unroll
        for (int v = 0; v < NV; ++v) Fs[v] *= sgS;   // F_S . n_S
        load4(a.metrics + ((size_t)se * nn + ns) * 4, J);
        const double nrm[2] = {sgS * (sf < 2 ? J[0] : J[2]), sgS * (sf < 2 ? J[1] : J[3])};
        const double* fwd = c_tlw_mortar[N][h ? 0 : 1];
        double fir[NV] = {0, 0, 0, 0};
#pragma unroll
        for (int i = 0; i < n; ++i) {
            const int li = rev ? n - 1 - i : i;
            const int nl = face_node_index(n, lf, li);
            double x[NV], y[NV], z[NV], JL[4];
            load4(a.u + ((size_t)lg * nn + nl) * NV, x);
            load4(a.tU + (((size_t)lg * 4 + lf) * n + li) * NV, y);
            load4(a.metrics + ((size_t)lg * nn + nl) * 4, JL);
            const double nL[2] = {-0.5 * (sgL * (lf < 2 ? JL[0] : JL[2])), -0.5 * (sgL * (lf < 2 ? JL[1] : JL[3]))};
            euler_flux_normal(gm1, x, nL, z);
            const double c = fwd[l * n + i];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                ul[v] = fma(c, x[v], ul[v]);
                Ul[v] = fma(c, y[v], Ul[v]);
                Fl[v] = fma(c, z[v], Fl[v]);
            }
            if (a.alpha) {
                load4(a.tFn + (((size_t)lg * 4 + lf) * n + i) * NV, x);
#pragma unroll
                for (int v = 0; v < NV; ++v) fir[v] = fma(c, x[v], fir[v]);
            }
        }
        double fstar[NV];
        lw_surface_flux_normal(a.gamma, a.flux_kind, a.speed_kind, Fs, Fl, us, ul, Us, Ul, nrm, fstar, a.status);
        if (a.alpha) {   // get_blended_flux, small element as the primary
            double fS[NV], gS[NV], fL[NV], gL[NV], fn[NV], fil[NV], test[NV], low[NV];
            euler_fluxes(gm1, us[0], us[1], us[2], us[3], fS, gS);
            euler_fluxes(gm1, ul[0], ul[1], ul[2], ul[3], fL, gL);
            const double lam = max_abs_speed_normal(a.gamma, us, ul, nrm, a.speed_kind, a.status);
#pragma unroll
            for (int v = 0; v < NV; ++v)
                fn[v] = 0.5 * ((fS[v] * nrm[0] + gS[v] * nrm[1]) + (fL[v] * nrm[0] + gL[v] * nrm[1])) +
                        (-0.5 * lam * (ul[v] - us[v]));
            load4(a.tFn + ts, fil);
            const double alp = 0.5 * (__ldg(a.alpha + se) + __ldg(a.alpha + lg));
#pragma unroll
            for (int v = 0; v < NV; ++v) fstar[v] = (1.0 - alp) * fstar[v] + alp * fn[v];
            const double dt = *a.dt;
            const double J = __ldg(a.mortar_ij + (size_t)k * n + l);
            const double cl = dt * J / (a.w_last * 0.5);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                test[v] = us[v] - cl * (fstar[v] - fil[v]);
                low[v] = us[v] - cl * (fn[v] - fil[v]);
            }
            if (!admissible(gm1, test)) zhang_shu_flux_fix(gm1, us, low, fstar, fil, fn, cl);
            const double cr = -dt * J / (a.w_first * 0.5);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                test[v] = ul[v] - cr * (fstar[v] - fir[v]);
                low[v] = ul[v] - cr * (fn[v] - fir[v]);
            }
            if (!admissible(gm1, test)) zhang_shu_flux_fix(gm1, ul, low, fstar, fir, fn, cr);
        }
        dts = a.step_mode ? *a.dt : 1.0;
        const double cs = -dts * __ldg(a.inv_jac + (size_t)se * nn + ns) * ((sf & 1) ? a.inv_w_last : a.inv_w_first);
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
    if (active && h == 1) {
        const double* ru = c_tlw_mortar[N][2];
        const double* rl = c_tlw_mortar[N][3];
        double p[NV] = {0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < n; ++q)
#pragma unroll
            for (int v = 0; v < NV; ++v) p[v] = fma(ru[l * n + q], fs[g][1][q][v], fma(rl[l * n + q], fs[g][0][q][v], p[v]));
        const int li = rev ? n - 1 - l : l;
        const int nl = face_node_index(n, lf, li);
        const double cl = -dts * __ldg(a.inv_jac + (size_t)lg * nn + nl) * ((lf & 1) ? a.inv_w_last : a.inv_w_first);
        double* ol = a.out + ((size_t)lg * nn + nl) * NV;
        double x[NV];
        load4_rw(ol, x);
#pragma unroll
        for (int v = 0; v < NV; ++v) x[v] = fma(cl, -2.0 * p[v], x[v]);
        store4(ol, x);
    }
}

}  // namespace tlw
