// tlw_launch.cu -- the kernel launches of one polynomial degree (tlw::Launch<N>, declared in tlw_launch.cuh).
// Compiled once per degree with -DTLW_LAUNCH_N=<N> (or once for all degrees without it), so that the
// degree instantiations of the volume, surface, mortar, parabolic and limiter kernels build in parallel.
// Every degree's unit holds its own copy of the constant-memory matrices: Launch<N>::upload_constants sets it.
#include "tlw_launch.cuh"

namespace tlw {
namespace {

static NSParams ns_params(const tlw_handle* h) {
    NSParams p{};
    p.gamma = h->opts.gamma;
    p.mu = h->ns_mu;
    p.Pr = h->ns_Pr;
    p.kappa = h->opts.gamma / ((h->opts.gamma - 1.0) * h->ns_Pr);
    return p;
}

// ---- kernel launch helpers (template dispatch over N) -------------------------------------------
template <int N>
struct LaunchImpl {
    using C = VolCfg<N>;
    template <bool SC>
    static void set_attr_sc() {
        const int lw = (int)C::smem_bytes(SC ? 8 : 4), md = (int)C::smem_bytes(SC ? 8 : 2);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_RHS, SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_STEP, SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_RHS, SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, SC>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
    }
    static void set_attributes() {
        set_attr_sc<false>();
        set_attr_sc<true>();
        const int lw = (int)C::smem_bytes(4);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        te_volume(nullptr, VolArgs{}, 0, false, true);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        curved_sc_attributes<0>();
        curved_sc_attributes<1>();
        curved_sc_attributes<2>();
        const int md = (int)C::smem_bytes(2);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_RHS, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_STEP, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_RHS, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, false, false, 0, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_bytes(5));
        // source terms (FR)
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, false, 0, false, false, false, 0, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false, 0, false, false, false, 0, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, false, 0, true, false, false, 0, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false, 0, true, false, false, 0, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, lw);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_RHS, false, true, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_STEP, false, true, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_RHS, false, true, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, false, true, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_RHS, false, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_STEP, false, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_RHS, false, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, false, false, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, md);
    }
    // source terms (FR volume integral, TreeMesh or curvilinear): LW or an MDRK stage
    template <bool CURVED>
    static void volume_src_on(cudaStream_t s, int stage, int mode, const VolArgs& a, int grid) {
        const size_t lw = C::smem_bytes(4), md = C::smem_bytes(2);
        if (stage == TLW_STAGE_LW) {
            if (mode == MODE_RHS) lw_volume_kernel<N, MODE_RHS, false, 0, CURVED, false, false, 0, true><<<grid, C::THREADS, lw, s>>>(a);
            else lw_volume_kernel<N, MODE_STEP, false, 0, CURVED, false, false, 0, true><<<grid, C::THREADS, lw, s>>>(a);
        } else if (stage == TLW_STAGE_MDRK1) {
            if (mode == MODE_RHS) mdrk1_volume_kernel<N, MODE_RHS, false, CURVED, 0, true><<<grid, C::THREADS, md, s>>>(a);
            else mdrk1_volume_kernel<N, MODE_STEP, false, CURVED, 0, true><<<grid, C::THREADS, md, s>>>(a);
        } else {
            if (mode == MODE_RHS) mdrk2_volume_kernel<N, MODE_RHS, false, CURVED, 0, true><<<grid, C::THREADS, md, s>>>(a);
            else mdrk2_volume_kernel<N, MODE_STEP, false, CURVED, 0, true><<<grid, C::THREADS, md, s>>>(a);
        }
    }
    static void volume_src(cudaStream_t s, int stage, int mode, const VolArgs& a, int grid) {
        if (a.metrics) volume_src_on<true>(s, stage, mode, a, grid);
        else volume_src_on<false>(s, stage, mode, a, grid);
    }
    template <bool SC>
    static void volume_sc(cudaStream_t s, int stage, int mode, const VolArgs& a, int grid) {
        const size_t lw = C::smem_bytes(SC ? 8 : 4), md = C::smem_bytes(SC ? 8 : 2);
        if (stage == TLW_STAGE_LW) {
            if (mode == MODE_RHS) lw_volume_kernel<N, MODE_RHS, SC><<<grid, C::THREADS, lw, s>>>(a);
            else lw_volume_kernel<N, MODE_STEP, SC><<<grid, C::THREADS, lw, s>>>(a);
        } else if (stage == TLW_STAGE_MDRK1) {
            if (mode == MODE_RHS) mdrk1_volume_kernel<N, MODE_RHS, SC><<<grid, C::THREADS, md, s>>>(a);
            else if (!SC && a.compact) mdrk1_volume_kernel<N, MODE_STEP, false, false, 0, false, true><<<grid, C::THREADS, md, s>>>(a);
            else mdrk1_volume_kernel<N, MODE_STEP, SC><<<grid, C::THREADS, md, s>>>(a);
        } else {
            if (mode == MODE_RHS) mdrk2_volume_kernel<N, MODE_RHS, SC><<<grid, C::THREADS, md, s>>>(a);
            else if (!SC && a.compact)
                mdrk2_volume_kernel<N, MODE_STEP, false, false, 0, false, true><<<grid, C::THREADS, C::smem_bytes(5), s>>>(a);
            else mdrk2_volume_kernel<N, MODE_STEP, SC><<<grid, C::THREADS, md, s>>>(a);
        }
    }
    // curvilinear shock capturing: LW or an MDRK stage with first-order (REC 0), MUSCL (REC 1) or MUSCL-Hancock
    // (REC 2) subcells
    template <int REC>
    static void curved_sc(cudaStream_t s, int stage, int mode, const VolArgs& a, int grid) {
        const size_t sm = C::smem_bytes(REC ? 12 : 8);
        if (stage == TLW_STAGE_MDRK1) {
            if (mode == MODE_RHS) mdrk1_volume_kernel<N, MODE_RHS, true, true, REC><<<grid, C::THREADS, sm, s>>>(a);
            else mdrk1_volume_kernel<N, MODE_STEP, true, true, REC><<<grid, C::THREADS, sm, s>>>(a);
        } else if (stage == TLW_STAGE_MDRK2) {
            if (mode == MODE_RHS) mdrk2_volume_kernel<N, MODE_RHS, true, true, REC><<<grid, C::THREADS, sm, s>>>(a);
            else mdrk2_volume_kernel<N, MODE_STEP, true, true, REC><<<grid, C::THREADS, sm, s>>>(a);
        } else {
            if (mode == MODE_RHS) lw_volume_kernel<N, MODE_RHS, true, 0, true, false, false, REC><<<grid, C::THREADS, sm, s>>>(a);
            else lw_volume_kernel<N, MODE_STEP, true, 0, true, false, false, REC><<<grid, C::THREADS, sm, s>>>(a);
        }
    }
    template <int REC>
    static void curved_sc_attributes() {
        const int sm = (int)C::smem_bytes(REC ? 12 : 8);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, true, 0, true, false, false, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, true, 0, true, false, false, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_RHS, true, true, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(mdrk1_volume_kernel<N, MODE_STEP, true, true, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_RHS, true, true, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(mdrk2_volume_kernel<N, MODE_STEP, true, true, REC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    // Adaptive trial step: the LW kernel with the temporal error estimate (a step into a.out), on a TreeMesh
    // (N >= 4) or a curvilinear mesh (N >= 3), with or without shock capturing; attr_only sets the shared
    // memory attributes of every variant instead
    template <bool SC, bool CURVED, int REC>
    static void te_launch(cudaStream_t s, const VolArgs& a, int grid, bool attr_only) {
        const int sm = (int)C::smem_bytes(!SC ? 4 : REC ? 12 : 8);
        if (attr_only)
            cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, SC, 0, CURVED, true, false, REC>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        else
            lw_volume_kernel<N, MODE_STEP, SC, 0, CURVED, true, false, REC><<<grid, C::THREADS, sm, s>>>(a);
    }
    static void te_volume(cudaStream_t s, const VolArgs& a, int grid, bool sc, bool attr_only) {
        if constexpr (N >= 3) {
            const bool curved = attr_only || a.metrics;
            const int rec = a.reconstruction;
            if (curved && (attr_only || !sc)) te_launch<false, true, 0>(s, a, grid, attr_only);
            if (curved && (attr_only || (sc && rec == TLW_RECONSTRUCTION_FIRST_ORDER))) te_launch<true, true, 0>(s, a, grid, attr_only);
            if (curved && (attr_only || (sc && rec == TLW_RECONSTRUCTION_MUSCL))) te_launch<true, true, 1>(s, a, grid, attr_only);
            if (curved && (attr_only || (sc && rec == TLW_RECONSTRUCTION_MUSCL_HANCOCK))) te_launch<true, true, 2>(s, a, grid, attr_only);
            if constexpr (N >= 4) {
                const bool tree = attr_only || !a.metrics;
                if (tree && (attr_only || !sc)) te_launch<false, false, 0>(s, a, grid, attr_only);
                if (tree && (attr_only || sc)) te_launch<true, false, 0>(s, a, grid, attr_only);
            }
        }
    }
    static void volume(cudaStream_t s, int stage, int mode, bool sc, const VolArgs& a) {
        const int grid = (int)((a.E + C::EB - 1) / C::EB);
        if (grid == 0) return;
        if (a.temporal_errors) {
            te_volume(s, a, grid, sc, false);
            return;
        }
        if (a.source && !sc) {
            volume_src(s, stage, mode, a, grid);
            return;
        }
        if (a.metrics && sc) {   // curvilinear mesh with shock capturing (MUSCL when the geometry is given)
            if (a.reconstruction == TLW_RECONSTRUCTION_MUSCL_HANCOCK) curved_sc<2>(s, stage, mode, a, grid);
            else if (a.reconstruction == TLW_RECONSTRUCTION_MUSCL) curved_sc<1>(s, stage, mode, a, grid);
            else curved_sc<0>(s, stage, mode, a, grid);
            return;
        }
        if (a.metrics) {   // curvilinear mesh (LW or MDRK, FR volume integral)
            const size_t md = C::smem_bytes(2);
            if (stage == TLW_STAGE_MDRK1) {
                if (mode == MODE_RHS) mdrk1_volume_kernel<N, MODE_RHS, false, true><<<grid, C::THREADS, md, s>>>(a);
                else mdrk1_volume_kernel<N, MODE_STEP, false, true><<<grid, C::THREADS, md, s>>>(a);
            } else if (stage == TLW_STAGE_MDRK2) {
                if (mode == MODE_RHS) mdrk2_volume_kernel<N, MODE_RHS, false, true><<<grid, C::THREADS, md, s>>>(a);
                else mdrk2_volume_kernel<N, MODE_STEP, false, true><<<grid, C::THREADS, md, s>>>(a);
            } else if (mode == MODE_RHS) {
                lw_volume_kernel<N, MODE_RHS, false, 0, true><<<grid, C::THREADS, C::smem_bytes(4), s>>>(a);
            } else {
                lw_volume_kernel<N, MODE_STEP, false, 0, true><<<grid, C::THREADS, C::smem_bytes(4), s>>>(a);
            }
            return;
        }
        if (sc) volume_sc<true>(s, stage, mode, a, grid);
        else volume_sc<false>(s, stage, mode, a, grid);
    }
    static void interfaces(cudaStream_t s, const SurfArgs& a) {
        const long long threads = (long long)a.count * (N + 1);
        if (threads == 0) return;
        interface_kernel<N><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
    }
    static void surfaces(cudaStream_t s, const SurfArgs& a, const BndArgs& b) {
        if (a.E <= 0) return;
        using C = SurfCfg<N>;
        const unsigned grid = (unsigned)((a.E + C::EB - 1) / C::EB);
        if (a.shock_capturing) {
            if (b.element) surface_kernel<N, true, true><<<grid, C::THREADS, 0, s>>>(a, b);
            else surface_kernel<N, false, true><<<grid, C::THREADS, 0, s>>>(a, b);
        } else {
            if (b.element) surface_kernel<N, true, false><<<grid, C::THREADS, 0, s>>>(a, b);
            else surface_kernel<N, false, false><<<grid, C::THREADS, 0, s>>>(a, b);
        }
    }
    static void parabolic(cudaStream_t s, const tlw_handle* h, int mode, const double* u, double* out,
                          const double* dtp) {
        if constexpr (N >= 3) {
            const int E = (int)h->E;
            using P = ParCfg<N>;
            const int grid = (E + P::EB - 1) / P::EB;
            const double iwf = h->h_basis.inv_w_first, iwl = h->h_basis.inv_w_last;
            if (h->curved) {
                grad_volume_kernel<N, true><<<grid, P::THREADS, 0, s>>>(u, h->d_ijn, E, h->d_gx, h->d_gy, h->d_Ja);
                for (size_t c = 0; c + 1 < h->color_off.size(); ++c) {
                    const int b = h->color_off[c], cnt = h->color_off[c + 1] - b;
                    const long long th = (long long)cnt * (N + 1);
                    if (th)
                        curved_grad_interface_kernel<N><<<(unsigned)((th + 127) / 128), 128, 0, s>>>(
                            u, h->d_cp + b, h->d_cs + b, h->d_cf + b, cnt, h->d_Ja, h->d_ijn, iwf, iwl, h->d_gx,
                            h->d_gy);
                }
                // xi-face boundaries, then eta-face ones (they share corner nodes)
                const int first[2] = {0, h->ncbx}, count[2] = {h->ncbx, h->ncb - h->ncbx};
                for (int cls = 0; cls < 2; ++cls) {
                    const long long tb = (long long)count[cls] * (N + 1);
                    if (tb)
                        curved_grad_boundary_kernel<N><<<(unsigned)((tb + 127) / 128), 128, 0, s>>>(
                            u, h->d_cbe + first[cls], h->d_cbf + first[cls], h->d_cbi + first[cls], count[cls],
                            h->d_wkind, h->d_wall, h->d_Ja, h->d_ijn, h->opts.gamma, iwf, iwl, h->d_gx, h->d_gy);
                }
            } else {
                grad_volume_kernel<N><<<grid, P::THREADS, 0, s>>>(u, h->d_inv_jac, E, h->d_gx, h->d_gy);
                const long long th = (long long)(h->nx + h->ny) * (N + 1);
                if (th)
                    grad_interface_kernel<N><<<(unsigned)((th + 127) / 128), 128, 0, s>>>(
                        u, h->d_xl, h->d_xr, h->nx, h->d_yl, h->d_yr, h->ny, h->d_inv_jac, iwf, iwl, h->d_gx,
                        h->d_gy);
                const long long tb = (long long)h->nb * (N + 1);
                if (tb)
                    grad_boundary_kernel<N><<<(unsigned)((tb + 127) / 128), 128, 0, s>>>(
                        u, h->d_b_elem, h->d_b_dir, h->d_wkind, h->d_wall, (int)h->nb, h->d_inv_jac, h->opts.gamma,
                        iwf, iwl, h->d_gx, h->d_gy);
            }
            ParArgs pa{};
            pa.u = u;
            pa.gx = h->d_gx;
            pa.gy = h->d_gy;
            pa.out = out;
            pa.tU = h->d_tU;
            pa.tF = h->d_tF;
            pa.tFv = h->d_tFv;
            pa.inv_jac = h->d_inv_jac;
            pa.dt = dtp;
            pa.E = E;
            pa.ns = ns_params(h);
            if (h->curved) {
                pa.inv_jac = h->d_ijn;
                pa.metrics = h->d_Ja;
                if (mode == MODE_RHS) par_volume_kernel<N, MODE_RHS, true><<<grid, P::THREADS, P::smem_bytes(), s>>>(pa);
                else par_volume_kernel<N, MODE_STEP, true><<<grid, P::THREADS, P::smem_bytes(), s>>>(pa);
            } else {
                if (mode == MODE_RHS) par_volume_kernel<N, MODE_RHS><<<grid, P::THREADS, P::smem_bytes(), s>>>(pa);
                else par_volume_kernel<N, MODE_STEP><<<grid, P::THREADS, P::smem_bytes(), s>>>(pa);
            }
        }
    }
    static void par_speed(cudaStream_t s, const tlw_handle* h, const double* u) {
        if constexpr (N >= 3) {
            const int E = (int)h->E;
            const int grid = (E + MsCfg<N>::ELEMS - 1) / MsCfg<N>::ELEMS;
            if (h->curved) {
                // the CFL maximum of the curvilinear max_dt and the parabolic max_dt's own maxima, one pass
                curved_par_speed_kernel<N><<<grid, MS_THREADS, 0, s>>>(u, h->d_Ja, h->d_ijn, E, ns_params(h),
                                                                        h->d_step, h->d_visc, h->d_visc + 1);
            } else {
                par_speed_kernel<N><<<grid, MS_THREADS, 0, s>>>(u, h->d_inv_jac, E, ns_params(h), h->d_step,
                                                                 h->d_visc, &h->d_step->max_bits);
            }
        }
    }
    static void par_attributes() {
        if constexpr (N >= 3) {
            cudaFuncSetAttribute(par_volume_kernel<N, MODE_RHS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ParCfg<N>::smem_bytes());
            cudaFuncSetAttribute(par_volume_kernel<N, MODE_STEP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ParCfg<N>::smem_bytes());
            cudaFuncSetAttribute(par_volume_kernel<N, MODE_RHS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ParCfg<N>::smem_bytes());
            cudaFuncSetAttribute(par_volume_kernel<N, MODE_STEP, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ParCfg<N>::smem_bytes());
        }
    }
    static void mortars(cudaStream_t s, const MortarArgs& a) {
        if (a.count == 0) return;
        using M = MortarCfg<N>;
        mortar_kernel<N><<<(a.count + M::PER_CTA - 1) / M::PER_CTA, M::THREADS, 0, s>>>(a);
    }
    static void curved_interfaces(cudaStream_t s, const CurvedSurfArgs& a) {
        const long long threads = (long long)a.count * (N + 1);
        if (threads == 0) return;
        curved_interface_kernel<N><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
    }
    static void curved_speed(cudaStream_t s, const double* u, const double* Ja, const double* ij, int E, double g,
                             StepState* st) {
        if (E == 0) return;
        curved_max_speed_kernel<N><<<(E + MsCfg<N>::ELEMS - 1) / MsCfg<N>::ELEMS, MS_THREADS, 0, s>>>(u, Ja, ij, E, g, st);
    }
    static void boundaries(cudaStream_t s, const BndArgs& a) {
        const long long threads = (long long)a.count * (N + 1);
        if (threads == 0) return;
        boundary_kernel<N><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
    }
    // speed: CFL reduction; ind: Hennemann-Gassner indicator (both read u once)
    static void max_speed(cudaStream_t s, const double* u, const double* ij, int E, double gamma, StepState* st,
                          bool speed, bool ind, const IndicatorArgs& ia, BatchSpeedArgs bs = BatchSpeedArgs{}) {
        if (E == 0) return;
        const int grid = (E + MsCfg<N>::ELEMS - 1) / MsCfg<N>::ELEMS;
        if (speed && ind && ia.metrics) max_speed_kernel<N, true, true, true><<<grid, MS_THREADS, 0, s>>>(u, ij, E, gamma, st, ia, bs);
        else if (speed && ind) max_speed_kernel<N, true, true><<<grid, MS_THREADS, 0, s>>>(u, ij, E, gamma, st, ia, bs);
        else if (speed) max_speed_kernel<N, true, false><<<grid, MS_THREADS, 0, s>>>(u, ij, E, gamma, st, ia, bs);
        else if (ind) max_speed_kernel<N, false, true><<<grid, MS_THREADS, 0, s>>>(u, ij, E, gamma, st, ia, bs);
    }
};

template <int N> struct LimImpl {
    static void run(cudaStream_t s, const LimiterArgs& a) {
        if (a.E == 0) return;
        positivity_limiter_kernel<N><<<(a.E + LIMITER_WARPS - 1) / LIMITER_WARPS, 32 * LIMITER_WARPS, 0, s>>>(a);
    }
};

}  // namespace

template <int N> cudaError_t Launch<N>::upload_constants(const Basis* all) {
    cudaError_t e = upload_const_basis(all);
    return e == cudaSuccess ? upload_const_mortar() : e;
}
template <int N> void Launch<N>::set_attributes() { LaunchImpl<N>::set_attributes(); }
template <int N> void Launch<N>::par_attributes() { LaunchImpl<N>::par_attributes(); }
template <int N> void Launch<N>::volume(cudaStream_t s, int stage, int mode, bool sc, const VolArgs& a) {
    LaunchImpl<N>::volume(s, stage, mode, sc, a);
}
template <int N> void Launch<N>::interfaces(cudaStream_t s, const SurfArgs& a) { LaunchImpl<N>::interfaces(s, a); }
template <int N> void Launch<N>::surfaces(cudaStream_t s, const SurfArgs& a, const BndArgs& b) {
    LaunchImpl<N>::surfaces(s, a, b);
}
template <int N> void Launch<N>::boundaries(cudaStream_t s, const BndArgs& a) { LaunchImpl<N>::boundaries(s, a); }
template <int N>
void Launch<N>::parabolic(cudaStream_t s, const tlw_handle* h, int mode, const double* u, double* out,
                          const double* dtp) {
    LaunchImpl<N>::parabolic(s, h, mode, u, out, dtp);
}
template <int N> void Launch<N>::par_speed(cudaStream_t s, const tlw_handle* h, const double* u) {
    LaunchImpl<N>::par_speed(s, h, u);
}
template <int N> void Launch<N>::mortars(cudaStream_t s, const MortarArgs& a) { LaunchImpl<N>::mortars(s, a); }
template <int N> void Launch<N>::curved_mortars(cudaStream_t s, const CurvedMortarArgs& a) {
    if (a.count == 0) return;
    using M = MortarCfg<N>;
    curved_mortar_kernel<N><<<(a.count + M::PER_CTA - 1) / M::PER_CTA, M::THREADS, 0, s>>>(a);
}
template <int N> void Launch<N>::curved_interfaces(cudaStream_t s, const CurvedSurfArgs& a) {
    LaunchImpl<N>::curved_interfaces(s, a);
}
template <int N> void Launch<N>::curved_boundaries(cudaStream_t s, const CurvedBndArgs& a) {
    const long long threads = (long long)a.count * (N + 1);
    if (threads == 0) return;
    curved_boundary_kernel<N><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
}
template <int N>
void Launch<N>::curved_speed(cudaStream_t s, const double* u, const double* Ja, const double* ij, int E, double g,
                             StepState* st) {
    LaunchImpl<N>::curved_speed(s, u, Ja, ij, E, g, st);
}
template <int N> void Launch<N>::halo(cudaStream_t s, const HaloArgs& a, bool pack) {
    const long long threads = (long long)a.count * (N + 1);
    if (threads == 0) return;
    if (pack) halo_pack_kernel<N><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
    else halo_face_kernel<N><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a);
}
template <int N> void Launch<N>::limiter(cudaStream_t s, const LimiterArgs& a) { LimImpl<N>::run(s, a); }
template <int N>
void Launch<N>::max_speed(cudaStream_t s, const double* u, const double* ij, int E, double gamma, StepState* st,
                          bool speed, bool ind, const IndicatorArgs& ia) {
    LaunchImpl<N>::max_speed(s, u, ij, E, gamma, st, speed, ind, ia);
}

#ifdef TLW_LAUNCH_N
template struct Launch<TLW_LAUNCH_N>;
#else
template struct Launch<1>;
template struct Launch<2>;
template struct Launch<3>;
template struct Launch<4>;
template struct Launch<5>;
template struct Launch<6>;
template struct Launch<7>;
#endif

}  // namespace tlw
