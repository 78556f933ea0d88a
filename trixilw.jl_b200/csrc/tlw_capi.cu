// tlw_capi.cu -- host side of libtlw: handle, device memory, kernel launches, the device-resident CFL
// step loop (captured as CUDA graphs) and the extern "C" entry points declared in include/tlw.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "../../include/tlw.h"
#include "tlw_basis.h"
#include "tlw_curved.cuh"
#include "tlw_curved_mortar.cuh"
#include "tlw_handle.h"
#include "tlw_mortar.cuh"
#include "tlw_limiter.cuh"
#include "tlw_halo.cuh"
#include "tlw_parabolic.cuh"
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"
#include "tlw_launch.cuh"

using namespace tlw;

namespace {

int fail(tlw_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

#define TLW_CUDA(h, call)                                                                        \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(h, TLW_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

size_t state_doubles(const tlw_handle* h) { return (size_t)NV * h->nn * h->E; }
size_t trace_doubles(const tlw_handle* h) { return (size_t)NV * h->n * 4 * h->E; }

void drop_graphs(tlw_handle* h) {
    for (int k = 0; k < 2; ++k) {
        if (h->g_one[k]) cudaGraphExecDestroy(h->g_one[k]);
        if (h->g_two[k]) cudaGraphExecDestroy(h->g_two[k]);
        h->g_one[k] = h->g_two[k] = nullptr;
    }
}

void free_mesh(tlw_handle* h) {
    drop_graphs(h);
    dfree(h->d_inv_jac);
    dfree(h->d_xl); dfree(h->d_xr); dfree(h->d_yl); dfree(h->d_yr); dfree(h->d_nbr);
    dfree(h->d_xnode); dfree(h->d_S2);
    h->source = 0;
    dfree(h->d_b_elem); dfree(h->d_b_dir); dfree(h->d_bx); dfree(h->d_by);
    dfree(h->d_levels); dfree(h->d_now);
    if (h->d_bkind) { cudaFree(h->d_bkind); h->d_bkind = nullptr; }
    if (h->d_wkind) { cudaFree(h->d_wkind); h->d_wkind = nullptr; }
    dfree(h->d_wall);
    h->bnd_dirichlet = true;
    if (h->s_up) cudaStreamSynchronize(h->s_up);
    if (h->s_down) cudaStreamSynchronize(h->s_down);
    h->async_pending = false;
    if (h->host_pool[0]) {   // the state buffers are members of the host-stepping pool
        for (double*& p : h->host_pool) dfree(p);
        h->d_state[0] = h->d_state[1] = nullptr;
    } else {
        dfree(h->d_state[0]); dfree(h->d_state[1]);
    }
    dfree(h->d_us); dfree(h->d_in); dfree(h->d_in2); dfree(h->d_out);
    dfree(h->d_tU); dfree(h->d_tF); dfree(h->d_U2); dfree(h->d_F2);
    dfree(h->d_alpha); dfree(h->d_alpha_raw); dfree(h->d_tFn); dfree(h->d_il); dfree(h->d_ir);
    dfree(h->d_subn); dfree(h->d_subq); dfree(h->d_mgeom);
    if (h->d_atb) { cudaFree(h->d_atb); h->d_atb = nullptr; }
    free_adjoint(h->adj);
    dfree(h->d_Ja); dfree(h->d_ijn); dfree(h->d_cp); dfree(h->d_cs); dfree(h->d_cf);
    dfree(h->d_ml); dfree(h->d_mu); dfree(h->d_mg); dfree(h->d_ms);
    h->nmx = h->nmy = 0;
    if (h->d_mface) { cudaFree(h->d_mface); h->d_mface = nullptr; }
    dfree(h->d_gx); dfree(h->d_gy); dfree(h->d_tFv); dfree(h->d_visc);
    h->parabolic = false;
    dfree(h->d_slots);
    h->slots_valid = false;
    dfree(h->d_te); dfree(h->d_check);
    if (h->d_bad) { cudaFree(h->d_bad); h->d_bad = nullptr; }
    if (h->d_adapt) { cudaFree(h->d_adapt); h->d_adapt = nullptr; }
    h->color_off.clear();
    h->face_used.clear();
    for (int** d : {&h->d_he, &h->d_hf, &h->d_hs})
        if (*d) { cudaFree(*d); *d = nullptr; }
    dfree(h->d_send); dfree(h->d_recv); dfree(h->d_asend); dfree(h->d_arecv);
    h->nh = h->nhx = 0;
    if (h->d_cbe) { cudaFree(h->d_cbe); h->d_cbe = nullptr; }
    if (h->d_cbf) { cudaFree(h->d_cbf); h->d_cbf = nullptr; }
    if (h->d_cbk) { cudaFree(h->d_cbk); h->d_cbk = nullptr; }
    if (h->d_cbi) { cudaFree(h->d_cbi); h->d_cbi = nullptr; }
    h->ncb = h->ncbx = 0;
    for (int** d : {&h->d_cms1, &h->d_cms2, &h->d_cml, &h->d_cmc, &h->d_cmsl, &h->d_cmsr})
        if (*d) { cudaFree(*d); *d = nullptr; }
    if (h->d_cmj) { cudaFree(h->d_cmj); h->d_cmj = nullptr; }
    h->ncm = 0;
    h->mortar_off.clear();
    dfree(h->d_unorm); dfree(h->d_tG);
    h->unstructured = false;
    h->curved = false;
    h->have_mesh = false;
    h->have_bdata = false;
}


template <template <int> class F, class... A>
void dispatch(int N, A&&... args) {
    switch (N) {
        case 1: F<1>::run(args...); break;
        case 2: F<2>::run(args...); break;
        case 3: F<3>::run(args...); break;
        case 4: F<4>::run(args...); break;
        case 5: F<5>::run(args...); break;
        case 6: F<6>::run(args...); break;
        case 7: F<7>::run(args...); break;
        default: break;
    }
}
template <int N> struct SetAttr { static void run() { Launch<N>::set_attributes(); } };
template <int N> struct Vol {
    static void run(cudaStream_t s, int st, int m, bool sc, const VolArgs& a) { Launch<N>::volume(s, st, m, sc, a); }
};
template <int N> struct Ifc { static void run(cudaStream_t s, const SurfArgs& a) { Launch<N>::interfaces(s, a); } };
template <int N> struct Srf {
    static void run(cudaStream_t s, const SurfArgs& a, const BndArgs& b) { Launch<N>::surfaces(s, a, b); }
};
template <int N> struct Bnd { static void run(cudaStream_t s, const BndArgs& a) { Launch<N>::boundaries(s, a); } };
template <int N> struct Par {
    static void run(cudaStream_t s, const tlw_handle* h, int mode, const double* u, double* out, const double* dtp) {
        Launch<N>::parabolic(s, h, mode, u, out, dtp);
    }
};
template <int N> struct ParSpd { static void run(cudaStream_t s, const tlw_handle* h, const double* u) { Launch<N>::par_speed(s, h, u); } };
template <int N> struct ParAttr { static void run() { Launch<N>::par_attributes(); } };
template <int N> struct Mrt { static void run(cudaStream_t s, const MortarArgs& a) { Launch<N>::mortars(s, a); } };
template <int N> struct CMrt { static void run(cudaStream_t s, const CurvedMortarArgs& a) { Launch<N>::curved_mortars(s, a); } };
template <int N> struct CIfc { static void run(cudaStream_t s, const CurvedSurfArgs& a) { Launch<N>::curved_interfaces(s, a); } };
template <int N> struct Halo { static void run(cudaStream_t s, const HaloArgs& a, bool pack) { Launch<N>::halo(s, a, pack); } };
template <int N> struct CBnd { static void run(cudaStream_t s, const CurvedBndArgs& a) { Launch<N>::curved_boundaries(s, a); } };
template <int N> struct Lim { static void run(cudaStream_t s, const LimiterArgs& a) { Launch<N>::limiter(s, a); } };
template <int N> struct Const { static void run(const Basis* all, cudaError_t* e) { if (*e == cudaSuccess) *e = Launch<N>::upload_constants(all); } };
template <int N> struct CSpd {
    static void run(cudaStream_t s, const double* u, const double* Ja, const double* ij, int E, double g, StepState* st) {
        Launch<N>::curved_speed(s, u, Ja, ij, E, g, st);
    }
};
template <int N> struct Spd {
    static void run(cudaStream_t s, const double* u, const double* ij, int E, double g, StepState* st, bool speed,
                    bool ind, const IndicatorArgs& ia) {
        Launch<N>::max_speed(s, u, ij, E, g, st, speed, ind, ia);
    }
};

// Events recorded between the phases of a step (tlw_step_timed); null when not timing.
struct PhaseEvents {
    cudaEvent_t after_volume, after_x, after_y;
};

// One rhs (volume + surfaces) launched on h->stream.
//   u_flux: state the volume fluxes use (u, or u* for MDRK stage 2); u_jump: u^n for the interfaces
//   out: du (mode RHS) or the stage/updated state (mode STEP, base = u_base)
IndicatorArgs indicator_args(tlw_handle* h) {
    IndicatorArgs ia{};
    ia.alpha_raw = h->d_alpha_raw;
    ia.alpha = h->d_alpha;
    ia.alpha_max = h->opts.alpha_max;
    ia.alpha_min = h->opts.alpha_min;
    // Trixi IndicatorHennemannGassner: threshold = 0.5 * 10^(-1.8 * nnodes^0.25), s = log((1 - 1e-4) / 1e-4)
    ia.threshold = 0.5 * std::pow(10.0, -1.8 * std::pow((double)h->n, 0.25));
    ia.parameter_s = std::log((1.0 - 0.0001) / 0.0001);
    return ia;
}

// alpha of u (indicator + smoothing); with `speed` the same pass also feeds the CFL reduction
void enqueue_indicator(tlw_handle* h, const double* u, bool speed) {
    IndicatorArgs ia = indicator_args(h);
    if (speed && h->curved) {   // the curvilinear CFL speeds in the same pass
        ia.metrics = h->d_Ja;
        ia.inv_jac_node = h->d_ijn;
    }
    dispatch<Spd>(h->N, h->stream, u, (const double*)h->d_inv_jac, (int)h->E, h->opts.gamma, h->d_step, speed, true,
                  ia);
    // interfaces for the smoothing: the TreeMesh list, or the curvilinear mesh's (primary, secondary) pairs
    const int ni = h->curved ? (h->color_off.empty() ? 0 : h->color_off.back()) : h->ni;
    if (h->opts.alpha_smooth && ni > 0)
        alpha_smooth_kernel<<<(ni + 255) / 256, 256, 0, h->stream>>>(h->curved ? h->d_cp : h->d_il,
                                                                    h->curved ? h->d_cs : h->d_ir, ni,
                                                                    h->d_alpha_raw, h->d_alpha);
    // and over the curvilinear mesh's mortars (each small element with the large one)
    if (h->opts.alpha_smooth && h->curved && h->ncms > 0)
        alpha_smooth_kernel<<<(h->ncms + 255) / 256, 256, 0, h->stream>>>(h->d_cmsl, h->d_cmsr, h->ncms,
                                                                         h->d_alpha_raw, h->d_alpha);
}

// the step's final values all come from the volume and interface kernels: the plain LW step on a periodic
// conforming TreeMesh (no boundaries, mortars, shock capturing, curvilinear or parabolic terms)
bool use_slots(const tlw_handle* h) {
    return h->d_slots && !h->sc && !h->curved && !h->parabolic && h->nb == 0 && h->nmx + h->nmy == 0 && h->nh == 0;
}

// one element-centric pass for all faces instead of the x and y interface sweeps
#ifndef TLW_SURFACE_PASS
#define TLW_SURFACE_PASS 1
#endif
#ifndef TLW_MDRK_COMPACT
#define TLW_MDRK_COMPACT 1
#endif
// (not with shock capturing: on the 512^2 Riemann problem the blended variant's steps took 1.099 ms at 142
// registers (one CTA per SM's worth) and 1.029 ms capped at 96 registers, against 0.993 ms with the sweeps)
#ifndef TLW_SURFACE_PASS_SC
#define TLW_SURFACE_PASS_SC 0
#endif
bool use_surface_pass(const tlw_handle* h) {
    return TLW_SURFACE_PASS && h->d_nbr && !h->curved && (!h->sc || TLW_SURFACE_PASS_SC) && h->nmx + h->nmy == 0 &&
           h->nh == 0;
}

// the halo faces of one class (cls 0: x, 1: y) as kernel arguments
HaloArgs halo_args(tlw_handle* h, int cls, int mode, const double* u_jump, double* out, const double* dt_ptr) {
    HaloArgs a{};
    const int first = cls == 0 ? 0 : h->nhx;
    a.u = u_jump;
    a.out = out;
    a.tU = h->d_tU;
    a.tF = h->d_tF;
    a.send = h->d_send;
    a.recv = h->d_recv;
    a.elem = h->d_he + first;
    a.face = h->d_hf + first;
    a.slot = h->d_hs + first;
    a.count = cls == 0 ? h->nhx : h->nh - h->nhx;
    a.orientation = cls + 1;
    a.inv_jac = h->d_inv_jac;
    a.dt = dt_ptr;
    a.step_mode = mode == MODE_STEP;
    a.gamma = h->opts.gamma;
    a.flux_kind = h->opts.surface_flux;
    a.speed_kind = h->opts.max_speed;
    a.inv_w_first = h->h_basis.inv_w_first;
    a.inv_w_last = h->h_basis.inv_w_last;
    a.status = &h->d_step->status;
    a.values = h->halo_values;
    if (h->sc) {
        a.alpha = h->d_alpha;
        a.tFn = h->d_tFn;
        a.jac_first = h->jac_first;
        a.w_first = h->h_basis.weights[0];
        a.w_last = h->h_basis.weights[h->n - 1];
    }
    return a;
}

// `reps` applications of the positivity limiter to u (in place); slots: the CFL slots of u to keep current
void enqueue_limiter(tlw_handle* h, double* u, int reps, unsigned long long* slots) {
    if (h->lim_count == 0) return;
    LimiterArgs a{};
    a.u = u;
    a.E = (int)h->E;
    a.gamma = h->opts.gamma;
    a.npairs = h->lim_count;
    a.reps = reps;
    for (int p = 0; p < h->lim_count; ++p) { a.threshold[p] = h->lim_thr[p]; a.variable[p] = h->lim_var[p]; }
    a.mortar_faces = h->d_mface;
    a.p4est = h->curved && h->ncm > 0 ? 1 : 0;
    a.cfl_slots = slots;
    a.status = &h->d_step->status;
    dispatch<Lim>(h->N, h->stream, a);
}

// the surfaces of a curvilinear mesh: interfaces colour by colour (no two threads of a launch share a node),
// then the xi-face and the eta-face boundaries; with the viscous traces for Navier-Stokes
void enqueue_curved_surfaces(tlw_handle* h, int mode, const double* u_jump, double* out, const double* dt_ptr,
                             const PhaseEvents* ev, double scaling_factor = 1.0) {
    CurvedSurfArgs ca{};
    ca.u = u_jump;
    ca.out = out;
    ca.tU = h->d_tU;
    ca.tF = h->d_tF;
    ca.tFv = h->parabolic ? h->d_tFv : nullptr;
    ca.metrics = h->d_Ja;
    ca.inv_jac = h->d_ijn;
    ca.dt = dt_ptr;
    ca.step_mode = mode == MODE_STEP;
    ca.gamma = h->opts.gamma;
    ca.flux_kind = h->opts.surface_flux;
    ca.speed_kind = h->opts.max_speed;
    ca.inv_w_first = h->h_basis.inv_w_first;
    ca.inv_w_last = h->h_basis.inv_w_last;
    ca.status = &h->d_step->status;
    if (h->sc) {
        ca.alpha = h->d_alpha;
        ca.tFn = h->d_tFn;
        ca.w_first = h->h_basis.weights[0];
        ca.w_last = h->h_basis.weights[h->n - 1];
    }
    if (h->unstructured) {
        ca.tG = h->d_tG;
        ca.unorm = h->d_unorm;
    }
    for (size_t c = 0; c + 1 < h->color_off.size(); ++c) {
        const int b = h->color_off[c];
        ca.p_elem = h->d_cp + b;
        ca.s_elem = h->d_cs + b;
        ca.faces = h->d_cf + b;
        ca.count = h->color_off[c + 1] - b;
        dispatch<CIfc>(h->N, h->stream, ca);
        if (ev && c == 0) cudaEventRecord(ev->after_x, h->stream);
    }
    if (ev && h->color_off.size() <= 2) cudaEventRecord(ev->after_x, h->stream);
    if (h->ncm > 0) {
        CurvedMortarArgs ma{};
        ma.u = u_jump;
        ma.out = out;
        ma.tU = h->d_tU;
        ma.tF = h->d_tF;
        ma.metrics = h->d_Ja;
        ma.inv_jac = h->d_ijn;
        ma.dt = dt_ptr;
        ma.step_mode = mode == MODE_STEP;
        ma.gamma = h->opts.gamma;
        ma.flux_kind = h->opts.surface_flux;
        ma.speed_kind = h->opts.max_speed;
        ma.inv_w_first = h->h_basis.inv_w_first;
        ma.inv_w_last = h->h_basis.inv_w_last;
        ma.status = &h->d_step->status;
        if (h->sc) {
            ma.alpha = h->d_alpha;
            ma.tFn = h->d_tFn;
            ma.w_first = h->h_basis.weights[0];
            ma.w_last = h->h_basis.weights[h->n - 1];
        }
        for (size_t c = 0; c + 1 < h->mortar_off.size(); ++c) {
            const int b = h->mortar_off[c];
            if (h->sc) ma.mortar_ij = h->d_cmj + (size_t)b * h->n;
            ma.small1 = h->d_cms1 + b;
            ma.small2 = h->d_cms2 + b;
            ma.large = h->d_cml + b;
            ma.code = h->d_cmc + b;
            ma.count = h->mortar_off[c + 1] - b;
            dispatch<CMrt>(h->N, h->stream, ma);
        }
    }
    if (h->ncb > 0) {
        CurvedBndArgs cb{};
        cb.u = u_jump;
        cb.out = out;
        cb.tU = h->d_tU;
        cb.tF = h->d_tF;
        cb.tFv = h->parabolic ? h->d_tFv : nullptr;
        cb.metrics = h->d_Ja;
        cb.inv_jac = h->d_ijn;
        cb.wall_kind = h->d_wkind;
        cb.wall = h->d_wall;
        cb.dt = dt_ptr;
        cb.step_mode = mode == MODE_STEP;
        cb.gamma = h->opts.gamma;
        cb.flux_kind = h->opts.surface_flux;
        cb.speed_kind = h->opts.max_speed;
        cb.inv_w_first = h->h_basis.inv_w_first;
        cb.inv_w_last = h->h_basis.inv_w_last;
        cb.status = &h->d_step->status;
        cb.levels = h->d_levels;
        cb.weights = h->d_basis->weights;
        cb.scaling_factor = scaling_factor;
        const int first[2] = {0, h->ncbx}, count[2] = {h->ncbx, h->ncb - h->ncbx};
        for (int cls = 0; cls < 2; ++cls) {
            cb.elem = h->d_cbe + first[cls];
            cb.face = h->d_cbf + first[cls];
            cb.kind = h->d_cbk + first[cls];
            cb.index = h->d_cbi + first[cls];
            cb.count = count[cls];
            dispatch<CBnd>(h->N, h->stream, cb);
        }
    }
    if (ev) cudaEventRecord(ev->after_y, h->stream);
}

BndArgs boundary_args(tlw_handle* h, int stage, int mode, const double* u_jump, double* out, const double* dt_ptr) {
    BndArgs ba{};
    ba.u = u_jump;
    ba.out = out;
    ba.tU = h->d_tU;
    ba.tF = h->d_tF;
    ba.element = h->d_b_elem;
    ba.direction = h->d_b_dir;
    ba.levels = h->d_levels;
    ba.now = h->d_now;
    ba.inv_jac = h->d_inv_jac;
    ba.dt = dt_ptr;
    ba.step_mode = mode == MODE_STEP;
    ba.scaling_factor = stage == TLW_STAGE_MDRK1 ? 0.5 : 1.0;
    ba.gamma = h->opts.gamma;
    ba.flux_kind = h->opts.surface_flux;
    ba.speed_kind = h->opts.max_speed;
    ba.inv_w_first = h->h_basis.inv_w_first;
    ba.inv_w_last = h->h_basis.inv_w_last;
    ba.weights = h->d_basis->weights;
    ba.status = &h->d_step->status;
    ba.kind = h->d_bkind;
    if (h->parabolic && h->nb > 0) {
        ba.tFv = h->d_tFv;
        ba.wall_kind = h->d_wkind;
        ba.wall = h->d_wall;
    }
    return ba;
}

// phases: 1 the volume kernel (and the halo packing); 2 the surfaces up to the x faces inside the part (x
// interfaces, boundaries, mortars; everything on meshes without cut faces); 4 the x cut faces and the y faces.
// 7: all of it. The split step runs 1 | 2 before the exchange and 4 after it.
void enqueue_rhs(tlw_handle* h, int stage, int mode, const double* u_flux, const double* u_jump, const double* u_base,
                 double* out, const double* dt_ptr, const PhaseEvents* ev = nullptr, bool alpha_ready = false,
                 int phases = 7) {
    if (h->sc && !alpha_ready) enqueue_indicator(h, u_jump, false);   // indicator of the instantaneous u
    if (h->parabolic) {
        // BR1 gradients, parabolic LW volume kernel, then the interfaces with the viscous traces
        dispatch<Par>(h->N, h->stream, (const tlw_handle*)h, mode, u_flux, out, dt_ptr);
        if (ev) cudaEventRecord(ev->after_volume, h->stream);
        if (h->curved) {
            enqueue_curved_surfaces(h, mode, u_jump, out, dt_ptr, ev);
            return;
        }
        SurfArgs sp{};
        sp.u = u_jump;
        sp.out = out;
        sp.tU = h->d_tU;
        sp.tF = h->d_tF;
        sp.tFv = h->d_tFv;
        sp.inv_jac = h->d_inv_jac;
        sp.dt = dt_ptr;
        sp.step_mode = mode == MODE_STEP;
        sp.gamma = h->opts.gamma;
        sp.flux_kind = h->opts.surface_flux;
        sp.speed_kind = h->opts.max_speed;
        sp.inv_w_first = h->h_basis.inv_w_first;
        sp.inv_w_last = h->h_basis.inv_w_last;
        sp.status = &h->d_step->status;
        BndArgs bp = boundary_args(h, stage, mode, u_jump, out, dt_ptr);
        if (use_surface_pass(h)) {
            sp.nbr = h->d_nbr;
            sp.E = (int)h->E;
            dispatch<Srf>(h->N, h->stream, sp, bp);
            if (ev) {
                cudaEventRecord(ev->after_x, h->stream);
                cudaEventRecord(ev->after_y, h->stream);
            }
            return;
        }
        sp.left = h->d_xl; sp.right = h->d_xr; sp.count = h->nx; sp.orientation = 1;
        dispatch<Ifc>(h->N, h->stream, sp);
        bp.bidx = h->d_bx; bp.count = h->nbx; bp.orientation = 1;
        dispatch<Bnd>(h->N, h->stream, bp);
        if (ev) cudaEventRecord(ev->after_x, h->stream);
        sp.left = h->d_yl; sp.right = h->d_yr; sp.count = h->ny; sp.orientation = 2;
        dispatch<Ifc>(h->N, h->stream, sp);
        bp.bidx = h->d_by; bp.count = h->nby; bp.orientation = 2;
        dispatch<Bnd>(h->N, h->stream, bp);
        if (ev) cudaEventRecord(ev->after_y, h->stream);
        return;
    }
    VolArgs va{};
    va.u = u_flux;
    va.u_base = u_base;
    va.out = out;
    va.tU = h->d_tU;
    va.tF = h->d_tF;
    va.U2 = h->d_U2;
    va.F2 = h->d_F2;
    va.inv_jac = h->d_inv_jac;
    va.dt = dt_ptr;
    va.basis = h->d_basis;
    va.E = (int)h->E;
    va.gamma = h->opts.gamma;
    va.alpha = h->d_alpha;
    va.tFn = h->d_tFn;
    va.status = &h->d_step->status;
    va.speed_kind = h->opts.max_speed;
    // the stage that produces the step's final values (LW, or MDRK stage 2) fills the next step's CFL slots
    if (mode == MODE_STEP && stage != TLW_STAGE_MDRK1 && use_slots(h) && !h->te_request) va.cfl_slots = h->d_slots;
    // an MDRK step on a plain TreeMesh passes only u_t between its stages (stage 2 rebuilds U2 and F2)
    va.compact = TLW_MDRK_COMPACT && mode == MODE_STEP && stage != TLW_STAGE_LW && !h->sc && !h->curved &&
                 !h->source && !h->parabolic;
    if (h->source) {
        va.source = h->source;
        va.xnode = h->d_xnode;
        va.tnow = dt_ptr == &h->d_step->dt_call ? &h->d_step->t_call : &h->d_step->t_step;
        va.S2 = h->d_S2;
    }
    if (h->te_request) {
        va.temporal_errors = h->d_te;
        va.abstol = h->te_abstol;
        va.reltol = h->te_reltol;
    }
    if (h->curved) {
        va.metrics = h->d_Ja;
        va.inv_jac_node = h->d_ijn;
        if (h->unstructured) va.tG = h->d_tG;
        if (h->sc) {
            va.subn = h->d_subn;
            va.subq = h->d_subq;
            va.atb = h->d_atb;
            va.muscl_geom = h->d_mgeom;
            va.reconstruction = h->reconstruction;
        }
    }
    if (phases & 1) {
        dispatch<Vol>(h->N, h->stream, stage, mode, h->sc, va);
        if (ev) cudaEventRecord(ev->after_volume, h->stream);
        for (int cls = 0; cls < 2 && h->nh > 0; ++cls)
            dispatch<Halo>(h->N, h->stream, halo_args(h, cls, mode, u_jump, out, dt_ptr), true);
    }
    if (!(phases & 6)) return;
    if (h->curved) {
        if (!(phases & 2)) return;
        // MDRK stage 1 scales the Dirichlet time averages by 1/2, as the P4estMesh path does
        // (src/solvers/dgsem_tree/multi_derivative_2d.jl:34)
        enqueue_curved_surfaces(h, mode, u_jump, out, dt_ptr, ev, stage == TLW_STAGE_MDRK1 ? 0.5 : 1.0);
        return;
    }

    SurfArgs sa{};
    sa.u = u_jump;
    sa.out = out;
    sa.tU = h->d_tU;
    sa.tF = h->d_tF;
    sa.inv_jac = h->d_inv_jac;
    sa.dt = dt_ptr;
    sa.step_mode = mode == MODE_STEP;
    sa.gamma = h->opts.gamma;
    sa.flux_kind = h->opts.surface_flux;
    sa.speed_kind = h->opts.max_speed;
    sa.inv_w_first = h->h_basis.inv_w_first;
    sa.inv_w_last = h->h_basis.inv_w_last;
    sa.status = &h->d_step->status;
    sa.shock_capturing = h->sc ? 1 : 0;
    sa.alpha = h->d_alpha;
    sa.tFn = h->d_tFn;
    sa.jac_first = h->jac_first;
    sa.w_first = h->h_basis.weights[0];
    sa.w_last = h->h_basis.weights[h->n - 1];
    sa.cfl_slots = va.cfl_slots;

    BndArgs ba = boundary_args(h, stage, mode, u_jump, out, dt_ptr);

    // x interfaces, x boundaries, y interfaces, y boundaries: corner nodes are shared only between
    // launches of different orientation, which the stream orders.
    MortarArgs ma{};
    ma.u = u_jump;
    ma.out = out;
    ma.tU = h->d_tU;
    ma.tF = h->d_tF;
    ma.inv_jac = h->d_inv_jac;
    ma.dt = dt_ptr;
    ma.step_mode = mode == MODE_STEP;
    ma.gamma = h->opts.gamma;
    ma.flux_kind = h->opts.surface_flux;
    ma.speed_kind = h->opts.max_speed;
    ma.inv_w_first = h->h_basis.inv_w_first;
    ma.inv_w_last = h->h_basis.inv_w_last;
    ma.status = &h->d_step->status;
    if (use_surface_pass(h)) {
        if (!(phases & 2)) return;
        sa.nbr = h->d_nbr;
        sa.E = (int)h->E;
        dispatch<Srf>(h->N, h->stream, sa, ba);
        if (ev) {
            cudaEventRecord(ev->after_x, h->stream);
            cudaEventRecord(ev->after_y, h->stream);
        }
        return;
    }
    if (phases & 2) {
        sa.left = h->d_xl; sa.right = h->d_xr; sa.count = h->nx; sa.orientation = 1;
        dispatch<Ifc>(h->N, h->stream, sa);
        ba.bidx = h->d_bx; ba.count = h->nbx; ba.orientation = 1;
        dispatch<Bnd>(h->N, h->stream, ba);
        if (h->nmx) {
            ma.lower = h->d_ml; ma.upper = h->d_mu; ma.large = h->d_mg; ma.large_side = h->d_ms;
            ma.count = h->nmx; ma.orientation = 1;
            dispatch<Mrt>(h->N, h->stream, ma);
        }
    }
    if (!(phases & 4)) return;
    if (h->nh > 0) dispatch<Halo>(h->N, h->stream, halo_args(h, 0, mode, u_jump, out, dt_ptr), false);
    if (ev) cudaEventRecord(ev->after_x, h->stream);
    sa.left = h->d_yl; sa.right = h->d_yr; sa.count = h->ny; sa.orientation = 2;
    dispatch<Ifc>(h->N, h->stream, sa);
    ba.bidx = h->d_by; ba.count = h->nby; ba.orientation = 2;
    dispatch<Bnd>(h->N, h->stream, ba);
    if (h->nmy) {
        ma.lower = h->d_ml + h->nmx; ma.upper = h->d_mu + h->nmx; ma.large = h->d_mg + h->nmx;
        ma.large_side = h->d_ms + h->nmx;
        ma.count = h->nmy; ma.orientation = 2;
        dispatch<Mrt>(h->N, h->stream, ma);
    }
    if (h->nh > 0) dispatch<Halo>(h->N, h->stream, halo_args(h, 1, mode, u_jump, out, dt_ptr), false);
    if (ev) cudaEventRecord(ev->after_y, h->stream);
}

// one CFL step from state[from] into state[1 - from]; ev (optional): [after dt, stage 1 phases, stage 2 phases]
void enqueue_step(tlw_handle* h, int from, cudaEvent_t after_dt = nullptr, const PhaseEvents* ev = nullptr) {
    const double* u = h->d_state[from];
    double* unew = h->d_state[1 - from];
    if (use_slots(h) && h->slots_valid) {
        // the previous step left the per-element maxima of this state
        const int grid = std::min<int>((int)((h->E + 255) / 256), 4 * 148);
        cfl_slots_reduce_kernel<<<grid, 256, 0, h->stream>>>(h->d_slots, h->d_inv_jac, (int)h->E, h->d_step);
    } else if (h->sc) enqueue_indicator(h, u, true);   // CFL reduction and indicator in one pass over u
    else if (h->parabolic) dispatch<ParSpd>(h->N, h->stream, (const tlw_handle*)h, u);   // (curvilinear too)
    else if (h->curved) dispatch<CSpd>(h->N, h->stream, u, (const double*)h->d_Ja, (const double*)h->d_ijn, (int)h->E,
                                       h->opts.gamma, h->d_step);
    else dispatch<Spd>(h->N, h->stream, u, (const double*)h->d_inv_jac, (int)h->E, h->opts.gamma, h->d_step, true,
                       false, indicator_args(h));
    if (h->parabolic) par_finalize_dt_kernel<<<1, 1, 0, h->stream>>>(h->d_step, h->d_visc, h->N, h->curved ? 1 : 0);
    else finalize_dt_kernel<<<1, 1, 0, h->stream>>>(h->d_step, h->n);
    if (after_dt) cudaEventRecord(after_dt, h->stream);
    const double* dtp = &h->d_step->dt;
    if (h->opts.time_discretization == TLW_LW) {
        enqueue_rhs(h, TLW_STAGE_LW, MODE_STEP, u, u, u, unew, dtp, ev, true);
        // solve_lwfr limits twice per LW step: in perform_step! (src/solvers/lwfr.jl:226) and in its loop (:257)
        enqueue_limiter(h, unew, 2, use_slots(h) ? h->d_slots : nullptr);
    } else {
        enqueue_rhs(h, TLW_STAGE_MDRK1, MODE_STEP, u, u, u, h->d_us, dtp, ev, true);
        enqueue_rhs(h, TLW_STAGE_MDRK2, MODE_STEP, h->d_us, u, u, unew, dtp, ev ? ev + 1 : nullptr, true);
        // once per MDRK step (the loop); perform_step!'s mid-step call (src/solvers/mdrk.jl:19) acts on u^n,
        // which the previous step's application has limited already
        enqueue_limiter(h, unew, 1, use_slots(h) ? h->d_slots : nullptr);
    }
}

__global__ void fp64_probe_kernel(double* out, int iters, double a, double b) {
    double x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = 1e-3 * (threadIdx.x + k);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 16; ++k) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += x[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void reciprocal_probe_kernel(const double* __restrict__ x, double* __restrict__ y, long long n) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = nr_reciprocal(x[k]);
}

int check_ready(tlw_handle* h, bool join_downloads = true) {
    if (!h) return TLW_E_ARG;
    if (join_downloads && h->async_pending) {
        // the entry point's work on the compute stream waits for tlw_step_host's last download
        TLW_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_dl[(h->host_calls - 1) % tlw_handle::HOST_CALLS], 0));
        h->async_pending = false;
    }
    if (!h->have_mesh) return fail(h, TLW_E_STATE, "no mesh: call tlw_set_tree_mesh first");
    if ((h->nb > 0 || h->ncb > 0) && h->bnd_dirichlet && !h->have_bdata)
        return fail(h, TLW_E_STATE, "mesh has Dirichlet boundaries: call tlw_set_boundary_data first");
    if (h->parabolic && (h->nb > 0 || h->ncb > 0) && !h->d_wkind)
        return fail(h, TLW_E_STATE, "Navier-Stokes with boundaries: call tlw_set_parabolic_walls first");
    return TLW_OK;
}

int read_status(tlw_handle* h) {
    unsigned st = 0;
    TLW_CUDA(h, cudaMemcpyAsync(&st, &h->d_step->status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (st) {
        const unsigned zero = 0;
        TLW_CUDA(h, upload_on(h->stream, &h->d_step->status, &zero, sizeof(zero)));
        return fail(h, TLW_E_NONADMISSIBLE, "non-admissible state: square root of a negative number (DomainError)");
    }
    return TLW_OK;
}

int ensure(tlw_handle* h, double*& p, size_t doubles) {
    if (!p) TLW_CUDA(h, cudaMalloc(&p, doubles * sizeof(double)));
    return TLW_OK;
}

}  // namespace

extern "C" {

int32_t tlw_abi_version(void) { return TLW_ABI_VERSION; }

int tlw_create(const tlw_opts* opts, tlw_handle** out) {
    if (!opts || !out) return TLW_E_ARG;
    *out = nullptr;
    if (opts->polydeg < 1 || opts->polydeg > 7) return TLW_E_ARG;
    if (opts->time_discretization != TLW_LW && opts->time_discretization != TLW_MDRK) return TLW_E_ARG;
    if (opts->surface_flux != TLW_FLUX_RUSANOV && opts->surface_flux != TLW_FLUX_HLL) return TLW_E_ARG;
    if (opts->max_speed != TLW_SPEED_NAIVE && opts->max_speed != TLW_SPEED_DAVIS) return TLW_E_ARG;
    if (!(opts->gamma > 1.0)) return TLW_E_ARG;
    if (opts->volume_integral != TLW_VOLUME_FR && opts->volume_integral != TLW_VOLUME_FR_SHOCK_CAPTURING) return TLW_E_ARG;
    if (opts->volume_integral == TLW_VOLUME_FR_SHOCK_CAPTURING &&
        !(opts->alpha_max >= 0.0 && opts->alpha_max <= 1.0 && opts->alpha_min >= 0.0 && opts->alpha_min < 0.5))
        return TLW_E_ARG;
    tlw_handle* h = new (std::nothrow) tlw_handle();
    if (!h) return TLW_E_ARG;
    h->opts = *opts;
    h->N = opts->polydeg;
    h->n = h->N + 1;
    h->nn = h->n * h->n;
    h->device = opts->device;
    h->sc = opts->volume_integral == TLW_VOLUME_FR_SHOCK_CAPTURING;
    host_build_basis(h->N, h->h_basis, &h->nodes);
    int rc = TLW_OK;
    do {
        if (cudaSetDevice(h->device) != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "cudaSetDevice failed"); break; }
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "stream"); break; }
        if (cudaMalloc(&h->d_basis, sizeof(tlw::Basis)) != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "alloc basis"); break; }
        if (upload_on(h->stream, h->d_basis, &h->h_basis, sizeof(tlw::Basis)) != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "copy basis"); break; }
        if (cudaMalloc(&h->d_step, sizeof(StepState)) != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "alloc step"); break; }
        StepState st{};
        st.cfl = 1.0;
        st.t_end = INFINITY;
        if (upload_on(h->stream, h->d_step, &st, sizeof(st)) != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "init step"); break; }
        tlw::Basis all[8];
        std::memset(&all[0], 0, sizeof(all[0]));
        for (int N = 1; N <= 7; ++N) host_build_basis(N, all[N]);
        cudaError_t ce = cudaSuccess;
        for (int k = 1; k <= 7; ++k) dispatch<Const>(k, (const Basis*)all, &ce);   // each degree's launch unit
        if (ce != cudaSuccess || upload_const_basis(all) != cudaSuccess || upload_const_mortar() != cudaSuccess) {
            rc = fail(h, TLW_E_CUDA, "constant basis");
            break;
        }
        dispatch<SetAttr>(h->N);
        if (cudaGetLastError() != cudaSuccess) { rc = fail(h, TLW_E_CUDA, "kernel attributes"); break; }
    } while (0);
    if (rc != TLW_OK) {
        tlw_destroy(h);
        return rc;
    }
    *out = h;
    return TLW_OK;
}

int tlw_destroy(tlw_handle* h) {
    if (!h) return TLW_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_mesh(h);
    dfree(h->d_basis);
    dfree(h->d_step);
    if (h->s_comm) cudaStreamSynchronize(h->s_comm);
    for (cudaEvent_t ev : {h->ev_up, h->ev_computed, h->ev_prior, h->ev_lib, h->ev_comm})
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : h->ev_free)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : h->ev_dl)
        if (ev) cudaEventDestroy(ev);
    if (h->s_comm) cudaStreamDestroy(h->s_comm);
    if (h->s_up) cudaStreamDestroy(h->s_up);
    if (h->s_down) cudaStreamDestroy(h->s_down);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return TLW_OK;
}

int tlw_set_tree_mesh(tlw_handle* h, int64_t n_elements, const double* inverse_jacobian, int64_t n_interfaces,
                      const int64_t* interface_neighbor_ids, const int64_t* interface_orientations,
                      int64_t n_boundaries, const int64_t* boundary_neighbor_ids,
                      const int64_t* boundary_orientations, const int64_t* boundary_neighbor_sides,
                      const int64_t* n_boundaries_per_direction) {
    if (!h) return TLW_E_ARG;
    if (n_elements <= 0 || n_elements > (int64_t)0x7fffffff / 64 || !inverse_jacobian) return fail(h, TLW_E_ARG, "n_elements");
    if (n_interfaces < 0 || (n_interfaces > 0 && (!interface_neighbor_ids || !interface_orientations)))
        return fail(h, TLW_E_ARG, "interfaces");
    if (n_boundaries < 0 || (n_boundaries > 0 && (!boundary_neighbor_ids || !boundary_orientations ||
                                                  !boundary_neighbor_sides || !n_boundaries_per_direction)))
        return fail(h, TLW_E_ARG, "boundaries");
    std::vector<int> xl, xr, yl, yr, al, ar;
    for (int64_t k = 0; k < n_interfaces; ++k) {
        const int64_t l = interface_neighbor_ids[2 * k] - 1, r = interface_neighbor_ids[2 * k + 1] - 1;
        const int64_t o = interface_orientations[k];
        if (l < 0 || l >= n_elements || r < 0 || r >= n_elements || (o != 1 && o != 2))
            return fail(h, TLW_E_ARG, "interface " + std::to_string(k + 1) + " out of range");
        (o == 1 ? xl : yl).push_back((int)l);
        (o == 1 ? xr : yr).push_back((int)r);
        al.push_back((int)l);
        ar.push_back((int)r);
    }
    std::vector<int> belem, bdir, bx, by;
    if (n_boundaries > 0) {
        int64_t sum = 0;
        for (int d = 0; d < 4; ++d) sum += n_boundaries_per_direction[d];
        if (sum != n_boundaries) return fail(h, TLW_E_ARG, "n_boundaries_per_direction does not sum to n_boundaries");
        int64_t k = 0;
        for (int d = 1; d <= 4; ++d)
            for (int64_t c = 0; c < n_boundaries_per_direction[d - 1]; ++c, ++k) {
                const int64_t e = boundary_neighbor_ids[k] - 1;
                const int64_t o = boundary_orientations[k];
                const int64_t side = boundary_neighbor_sides[k];
                if (e < 0 || e >= n_elements) return fail(h, TLW_E_ARG, "boundary element out of range");
                // direction d: 1/2 are x faces (orientation 1), 3/4 y faces; odd d -> element on the + side
                if (o != (d <= 2 ? 1 : 2) || side != (d % 2 == 1 ? 2 : 1))
                    return fail(h, TLW_E_ARG, "boundary " + std::to_string(k + 1) + " inconsistent with its direction");
                belem.push_back((int)e);
                bdir.push_back(d);
                (o == 1 ? bx : by).push_back((int)k);
            }
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    free_mesh(h);
    h->E = n_elements;
    auto up_i = [&](int*& d, const std::vector<int>& v) -> int {
        if (v.empty()) return TLW_OK;
        TLW_CUDA(h, cudaMalloc(&d, v.size() * sizeof(int)));
        TLW_CUDA(h, upload_on(h->stream, d, v.data(), v.size() * sizeof(int)));
        return TLW_OK;
    };
    int rc;
    TLW_CUDA(h, cudaMalloc(&h->d_inv_jac, n_elements * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_inv_jac, inverse_jacobian, n_elements * sizeof(double)));
    if ((rc = up_i(h->d_xl, xl)) || (rc = up_i(h->d_xr, xr)) || (rc = up_i(h->d_yl, yl)) || (rc = up_i(h->d_yr, yr)) ||
        (rc = up_i(h->d_b_elem, belem)) || (rc = up_i(h->d_b_dir, bdir)) || (rc = up_i(h->d_bx, bx)) ||
        (rc = up_i(h->d_by, by)))
        return rc;
    h->nx = (int)xl.size(); h->ny = (int)yl.size();
    if (2 * (int64_t)(xl.size() + yl.size()) + n_boundaries == 4 * n_elements) {
        // every face a conforming interface or a boundary: the element-centric surface pass takes the element
        // across each face, or -(k + 1) for boundary k
        constexpr int unset = std::numeric_limits<int>::min();
        std::vector<int> nbr((size_t)4 * n_elements, unset);
        bool ok = true;
        auto put = [&](int e, int f, int other) {
            int& slot = nbr[(size_t)4 * e + f];
            if (slot != unset) ok = false;
            slot = other;
        };
        for (size_t k = 0; k < xl.size(); ++k) { put(xl[k], 1, xr[k]); put(xr[k], 0, xl[k]); }
        for (size_t k = 0; k < yl.size(); ++k) { put(yl[k], 3, yr[k]); put(yr[k], 2, yl[k]); }
        for (size_t k = 0; k < belem.size(); ++k) put(belem[k], bdir[k] - 1, -(int)k - 1);
        if (ok && (rc = up_i(h->d_nbr, nbr))) return rc;
    }
    h->jac_first = inverse_jacobian[0];
    if (h->sc) {
        if ((rc = up_i(h->d_il, al)) || (rc = up_i(h->d_ir, ar))) return rc;
        h->ni = h->ni_if = (int)al.size();
    }
    h->nb = n_boundaries; h->nbx = (int)bx.size(); h->nby = (int)by.size();
    TLW_CUDA(h, cudaMalloc(&h->d_slots, (size_t)n_elements * CFL_SLOTS * sizeof(unsigned long long)));
    h->slots_valid = false;
    const size_t sd = state_doubles(h), td = trace_doubles(h);
    if ((rc = ensure(h, h->d_state[0], sd)) || (rc = ensure(h, h->d_state[1], sd)) || (rc = ensure(h, h->d_tU, td)) ||
        (rc = ensure(h, h->d_tF, td)))
        return rc;
    if (h->opts.time_discretization == TLW_MDRK) {
        if ((rc = ensure(h, h->d_U2, sd)) || (rc = ensure(h, h->d_F2, 2 * sd)) || (rc = ensure(h, h->d_us, sd))) return rc;
    }
    if (h->sc) {
        if ((rc = ensure(h, h->d_alpha, (size_t)h->E)) || (rc = ensure(h, h->d_alpha_raw, (size_t)h->E)) ||
            (rc = ensure(h, h->d_tFn, td)))
            return rc;
    }
    h->cur = 0;
    h->have_mesh = true;
    return TLW_OK;
}

}  // extern "C"

namespace {

// Shock capturing on a curvilinear mesh: the subcell-face normals of every element (Trixi calcflux_fv! for
// curved meshes: along xi, face f between nodes f-1 and f of row j has Ja^1(0, j) + sum_{k < f} w_k
// sum_m D[k][m] Ja^1(m, j); along eta likewise), the normal the reference's calc_fn_low! takes for face n-1
// (src/solvers/dgsem_structured/dg_2d.jl:111-174: the increments of faces 1 and n-1 only), the MUSCL geometry
// (compute_subcells, src/solvers/dgsem_tree/dg_2d.jl:1806-1824) and the buffers of the blending.
int upload_curved_subcells(tlw_handle* h, const double* Ja) {
    const int n = h->n, nn = h->nn;
    const int64_t E = h->E;
    const tlw::Basis& b = h->h_basis;
    std::vector<double> subn((size_t)E * 2 * n * (n - 1) * 2), subq((size_t)E * 2 * n * 2);
    for (int64_t e = 0; e < E; ++e)
        for (int d = 0; d < 2; ++d)
            for (int line = 0; line < n; ++line) {
                auto J = [&](int m, int c) {
                    const int node = d == 0 ? m + n * line : line + n * m;
                    return Ja[4 * ((size_t)e * nn + node) + 2 * d + c];
                };
                auto inc = [&](int k, double* o) {
                    o[0] = o[1] = 0.0;
                    for (int m = 0; m < n; ++m) {
                        const double c = b.weights[k] * b.D[k * n + m];
                        o[0] += c * J(m, 0);
                        o[1] += c * J(m, 1);
                    }
                };
                const size_t row = ((size_t)e * 2 + d) * n + line;
                double nrm[2] = {J(0, 0), J(0, 1)}, q[2] = {J(0, 0), J(0, 1)}, o[2];
                for (int f = 1; f < n; ++f) {
                    inc(f - 1, o);
                    nrm[0] += o[0];
                    nrm[1] += o[1];
                    subn[(row * (n - 1) + (f - 1)) * 2] = nrm[0];
                    subn[(row * (n - 1) + (f - 1)) * 2 + 1] = nrm[1];
                    if (f == 1 || f == n - 1) { q[0] += o[0]; q[1] += o[1]; }
                }
                subq[row * 2] = q[0];
                subq[row * 2 + 1] = q[1];
            }
    std::vector<double> geom(2 * n + 3, -1.0);
    double acc = 0.0;
    for (int i = 1; i <= n; ++i) {
        acc += b.weights[i - 1];
        geom[i] = -1.0 + acc;
    }
    for (int i = 0; i < n; ++i) geom[n + 2 + i] = h->nodes[i];
    geom[2 * n + 2] = 1.0;
    int rc;
    if ((rc = ensure(h, h->d_subn, subn.size())) || (rc = ensure(h, h->d_subq, subq.size())) ||
        (rc = ensure(h, h->d_mgeom, geom.size())) || (rc = ensure(h, h->d_alpha, (size_t)E)) ||
        (rc = ensure(h, h->d_alpha_raw, (size_t)E)) || (rc = ensure(h, h->d_tFn, trace_doubles(h))))
        return rc;
    TLW_CUDA(h, upload_on(h->stream, h->d_subn, subn.data(), subn.size() * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_subq, subq.data(), subq.size() * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_mgeom, geom.data(), geom.size() * sizeof(double)));
    TLW_CUDA(h, cudaMalloc(&h->d_atb, (size_t)E));
    TLW_CUDA(h, zero_on(h->stream, h->d_atb, (size_t)E));
    return TLW_OK;
}

}  // namespace

extern "C" {

int tlw_set_reconstruction(tlw_handle* h, int32_t reconstruction) {
    if (!h) return TLW_E_ARG;
    if (reconstruction != TLW_RECONSTRUCTION_FIRST_ORDER && reconstruction != TLW_RECONSTRUCTION_MUSCL &&
        reconstruction != TLW_RECONSTRUCTION_MUSCL_HANCOCK)
        return fail(h, TLW_E_ARG, "reconstruction");
    if (reconstruction != TLW_RECONSTRUCTION_FIRST_ORDER && (!h->sc || (h->have_mesh && !h->curved)))
        return fail(h, TLW_E_UNSUPPORTED, "MUSCL / MUSCL-Hancock subcells: shock capturing on a curvilinear mesh");
    drop_graphs(h);
    h->reconstruction = reconstruction;
    return TLW_OK;
}

int tlw_set_curved_mesh(tlw_handle* h, int64_t n_elements, const double* contravariant_vectors,
                        const double* inverse_jacobian, int64_t n_interfaces, const int64_t* primary_elements,
                        const int32_t* primary_faces, const int64_t* secondary_elements,
                        const int32_t* secondary_faces, const int32_t* secondary_reversed) {
    if (!h) return TLW_E_ARG;
    if (h->N < 3) return fail(h, TLW_E_UNSUPPORTED, "curvilinear meshes: N >= 3");
    if (h->sc && h->opts.surface_flux != TLW_FLUX_RUSANOV)
        return fail(h, TLW_E_UNSUPPORTED, "curvilinear shock capturing: the Rusanov surface flux");
    if (n_elements <= 0 || n_elements > (int64_t)0x7fffffff / 64 || !contravariant_vectors || !inverse_jacobian)
        return fail(h, TLW_E_ARG, "n_elements / metrics");
    if (n_interfaces < 0 || (n_interfaces > 0 && (!primary_elements || !primary_faces || !secondary_elements ||
                                                  !secondary_faces || !secondary_reversed)))
        return fail(h, TLW_E_ARG, "interfaces");
    // greedy colouring: within a colour, every element has interfaces on faces of one class only (xi or
    // eta), so no two threads of a launch update the same corner node
    struct Ifc { int p, s, code, cp, cs; };
    std::vector<Ifc> all((size_t)n_interfaces);
    std::vector<int64_t> seen((size_t)n_elements * 4, -1);
    for (int64_t k = 0; k < n_interfaces; ++k) {
        const int64_t p = primary_elements[k] - 1, q = secondary_elements[k] - 1;
        const int pf = primary_faces[k], sf = secondary_faces[k], rv = secondary_reversed[k];
        if (p < 0 || p >= n_elements || q < 0 || q >= n_elements || pf < 0 || pf > 3 || sf < 0 || sf > 3 ||
            (rv != 0 && rv != 1))
            return fail(h, TLW_E_ARG, "interface " + std::to_string(k + 1) + " out of range");
        if (seen[(size_t)p * 4 + pf] >= 0 || seen[(size_t)q * 4 + sf] >= 0 || (p == q && pf == sf))
            return fail(h, TLW_E_ARG, "interface " + std::to_string(k + 1) + ": element face used twice");
        seen[(size_t)p * 4 + pf] = k;
        seen[(size_t)q * 4 + sf] = k;
        if (p == q && (pf >> 1) != (sf >> 1))
            return fail(h, TLW_E_ARG, "interface " + std::to_string(k + 1) + " joins two face classes of one element");
        all[(size_t)k] = Ifc{(int)p, (int)q, pf | (sf << 2) | (rv << 4), pf >> 1, sf >> 1};
    }
    std::stable_sort(all.begin(), all.end(), [](const Ifc& a, const Ifc& b) {
        return (a.cp != a.cs) < (b.cp != b.cs) || ((a.cp != a.cs) == (b.cp != b.cs) && a.cp < b.cp);
    });
    std::vector<std::vector<signed char>> cls;   // [colour][element] face class used, -1 none
    std::vector<std::vector<int>> bucket;
    for (const Ifc& f : all) {
        size_t c = 0;
        for (; c < cls.size(); ++c) {
            const signed char a = cls[c][f.p], b = cls[c][f.s];
            if ((a < 0 || a == f.cp) && (b < 0 || b == f.cs)) break;
        }
        if (c == cls.size()) {
            cls.emplace_back((size_t)n_elements, (signed char)-1);
            bucket.emplace_back();
        }
        cls[c][f.p] = (signed char)f.cp;
        cls[c][f.s] = (signed char)f.cs;
        bucket[c].push_back((int)(&f - all.data()));
    }
    std::vector<int> cp, cs, cf, off{0};
    for (const auto& bk : bucket) {
        for (int k : bk) {
            cp.push_back(all[k].p);
            cs.push_back(all[k].s);
            cf.push_back(all[k].code);
        }
        off.push_back((int)cp.size());
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    free_mesh(h);
    h->E = n_elements;
    const size_t nodes = (size_t)h->nn * n_elements;
    auto up_i = [&](int*& d, const std::vector<int>& v) -> int {
        if (v.empty()) return TLW_OK;
        TLW_CUDA(h, cudaMalloc(&d, v.size() * sizeof(int)));
        TLW_CUDA(h, upload_on(h->stream, d, v.data(), v.size() * sizeof(int)));
        return TLW_OK;
    };
    int rc;
    TLW_CUDA(h, cudaMalloc(&h->d_Ja, nodes * 4 * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_Ja, contravariant_vectors, nodes * 4 * sizeof(double)));
    TLW_CUDA(h, cudaMalloc(&h->d_ijn, nodes * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_ijn, inverse_jacobian, nodes * sizeof(double)));
    if ((rc = up_i(h->d_cp, cp)) || (rc = up_i(h->d_cs, cs)) || (rc = up_i(h->d_cf, cf))) return rc;
    h->color_off = off;
    h->face_used.assign((size_t)n_elements * 4, 0);
    for (const Ifc& f : all) {
        h->face_used[(size_t)f.p * 4 + (f.code & 3)] = 1;
        h->face_used[(size_t)f.s * 4 + ((f.code >> 2) & 3)] = 1;
    }
    h->nx = h->ny = 0;
    h->nb = 0; h->nbx = h->nby = 0;
    const size_t sd = state_doubles(h), td = trace_doubles(h);
    if ((rc = ensure(h, h->d_state[0], sd)) || (rc = ensure(h, h->d_state[1], sd)) || (rc = ensure(h, h->d_tU, td)) ||
        (rc = ensure(h, h->d_tF, td)))
        return rc;
    if (h->opts.time_discretization == TLW_MDRK) {
        if ((rc = ensure(h, h->d_U2, sd)) || (rc = ensure(h, h->d_F2, 2 * sd)) || (rc = ensure(h, h->d_us, sd))) return rc;
    }
    if (h->sc && (rc = upload_curved_subcells(h, contravariant_vectors))) return rc;
    h->curved = true;
    h->cur = 0;
    h->have_mesh = true;
    return TLW_OK;
}

int tlw_set_unstructured_mesh(tlw_handle* h, int64_t n_elements, const double* contravariant_vectors,
                              const double* inverse_jacobian, const double* normal_directions, int64_t n_interfaces,
                              const int64_t* element_ids, const int64_t* element_side_ids, const int64_t* start_index,
                              const int64_t* index_increment) {
    if (!h) return TLW_E_ARG;
    if (h->opts.time_discretization != TLW_LW)
        return fail(h, TLW_E_UNSUPPORTED, "UnstructuredMesh2D: LW (the reference has no MDRK rhs for it)");
    if (!normal_directions || n_elements <= 0 || n_elements > (int64_t)0x7fffffff / 64) return fail(h, TLW_E_ARG, "normals");
    if (n_interfaces < 0 || (n_interfaces > 0 && (!element_ids || !element_side_ids || !start_index || !index_increment)))
        return fail(h, TLW_E_ARG, "interfaces");
    // Trixi sides 1: bottom (j = 1), 2: right (i = n), 3: top (j = n), 4: left (i = 1) as faces 0: -xi, 1: +xi,
    // 2: -eta, 3: +eta; the secondary index runs forward (start 1, increment 1) or backward (start n, increment -1)
    static const int face_of_side[5] = {-1, 2, 1, 3, 0};
    std::vector<int64_t> pe((size_t)n_interfaces), se((size_t)n_interfaces);
    std::vector<int32_t> pf((size_t)n_interfaces), sf((size_t)n_interfaces), rv((size_t)n_interfaces);
    for (int64_t k = 0; k < n_interfaces; ++k) {
        const int64_t s1 = element_side_ids[2 * k], s2 = element_side_ids[2 * k + 1];
        const int64_t st = start_index[k], inc = index_increment[k];
        if (s1 < 1 || s1 > 4 || s2 < 1 || s2 > 4 || !((st == 1 && inc == 1) || (st == h->n && inc == -1)))
            return fail(h, TLW_E_ARG, "interface " + std::to_string(k + 1) + ": side or secondary index out of range");
        pe[(size_t)k] = element_ids[2 * k];
        se[(size_t)k] = element_ids[2 * k + 1];
        pf[(size_t)k] = face_of_side[s1];
        sf[(size_t)k] = face_of_side[s2];
        rv[(size_t)k] = inc == -1 ? 1 : 0;
    }
    int rc = tlw_set_curved_mesh(h, n_elements, contravariant_vectors, inverse_jacobian, n_interfaces, pe.data(),
                                 pf.data(), se.data(), sf.data(), rv.data());
    if (rc) return rc;
    // normal_directions [2, node, side, element] -> [2, l, face, e]
    const int n = h->n;
    std::vector<double> nd((size_t)2 * n * 4 * n_elements);
    for (int64_t e = 0; e < n_elements; ++e)
        for (int side = 1; side <= 4; ++side)
            for (int l = 0; l < n; ++l)
                for (int d = 0; d < 2; ++d)
                    nd[(((size_t)e * 4 + face_of_side[side]) * n + l) * 2 + d] =
                        normal_directions[d + 2 * (l + (size_t)n * ((side - 1) + 4 * (size_t)e))];
    TLW_CUDA(h, cudaMalloc(&h->d_unorm, nd.size() * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_unorm, nd.data(), nd.size() * sizeof(double)));
    if ((rc = ensure(h, h->d_tG, trace_doubles(h)))) return rc;
    h->unstructured = true;
    return TLW_OK;
}

int tlw_set_tree_mortars(tlw_handle* h, int64_t n_mortars, const int64_t* mortar_neighbor_ids,
                         const int64_t* mortar_large_sides, const int64_t* mortar_orientations) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || h->curved) return fail(h, TLW_E_STATE, "mortars follow tlw_set_tree_mesh");
    if (n_mortars < 0 || (n_mortars > 0 && (!mortar_neighbor_ids || !mortar_large_sides || !mortar_orientations)))
        return fail(h, TLW_E_ARG, "mortars");
    std::vector<int> ml[2], mu[2], mg[2], ms[2];
    std::vector<int> mface(n_mortars > 0 ? (size_t)h->E : 0, 0);
    for (int64_t k = 0; k < n_mortars; ++k) {
        const int64_t lo = mortar_neighbor_ids[3 * k] - 1, up = mortar_neighbor_ids[3 * k + 1] - 1;
        const int64_t lg = mortar_neighbor_ids[3 * k + 2] - 1;
        const int64_t side = mortar_large_sides[k], o = mortar_orientations[k];
        if (lo < 0 || lo >= h->E || up < 0 || up >= h->E || lg < 0 || lg >= h->E || (side != 1 && side != 2) ||
            (o != 1 && o != 2) || lo == up || lo == lg || up == lg)
            return fail(h, TLW_E_ARG, "mortar " + std::to_string(k + 1) + " out of range");
        const int d = (int)o - 1;
        int& desc = mface[(size_t)lg];
        if ((desc & 7) >= 4) return fail(h, TLW_E_ARG, "element " + std::to_string(lg + 1) + " is the large side of more than 4 mortars");
        const int face = side == 1 ? (o == 1 ? 1 : 3) : (o == 1 ? 0 : 2);
        desc = ((desc & ~7) | ((desc & 7) + 1)) | (face << (3 + 2 * (desc & 7)));
        ml[d].push_back((int)lo); mu[d].push_back((int)up); mg[d].push_back((int)lg); ms[d].push_back((int)side);
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    dfree(h->d_ml); dfree(h->d_mu); dfree(h->d_mg); dfree(h->d_ms);
    if (h->d_mface) { cudaFree(h->d_mface); h->d_mface = nullptr; }
    h->nmx = (int)ml[0].size();
    h->nmy = (int)ml[1].size();
    if (n_mortars > 0) {
        auto up_cat = [&](int*& d, const std::vector<int>& a, const std::vector<int>& b) -> int {
            std::vector<int> v(a);
            v.insert(v.end(), b.begin(), b.end());
            TLW_CUDA(h, cudaMalloc(&d, v.size() * sizeof(int)));
            TLW_CUDA(h, upload_on(h->stream, d, v.data(), v.size() * sizeof(int)));
            return TLW_OK;
        };
        int rc;
        if ((rc = up_cat(h->d_ml, ml[0], ml[1])) || (rc = up_cat(h->d_mu, mu[0], mu[1])) ||
            (rc = up_cat(h->d_mg, mg[0], mg[1])) || (rc = up_cat(h->d_ms, ms[0], ms[1])) ||
            (rc = up_cat(h->d_mface, mface, std::vector<int>())))
            return rc;
    }
    if (h->sc) {
        // the blending factors are smoothed over the mortars too (each small element with the large one): the
        // interface pairs, then (lower, large) and (upper, large) of every mortar
        std::vector<int> l(h->ni_if), r(h->ni_if);
        if (h->ni_if > 0) {
            TLW_CUDA(h, download_on(h->stream, l.data(), h->d_il, h->ni_if * sizeof(int)));
            TLW_CUDA(h, download_on(h->stream, r.data(), h->d_ir, h->ni_if * sizeof(int)));
        }
        for (int d = 0; d < 2; ++d)
            for (size_t k = 0; k < ml[d].size(); ++k) {
                l.push_back(ml[d][k]); r.push_back(mg[d][k]);
                l.push_back(mu[d][k]); r.push_back(mg[d][k]);
            }
        dfree(h->d_il); dfree(h->d_ir);
        if (!l.empty()) {
            TLW_CUDA(h, cudaMalloc(&h->d_il, l.size() * sizeof(int)));
            TLW_CUDA(h, cudaMalloc(&h->d_ir, r.size() * sizeof(int)));
            TLW_CUDA(h, upload_on(h->stream, h->d_il, l.data(), l.size() * sizeof(int)));
            TLW_CUDA(h, upload_on(h->stream, h->d_ir, r.data(), r.size() * sizeof(int)));
        }
        h->ni = (int)l.size();
    }
    return TLW_OK;
}

int tlw_set_source_terms(tlw_handle* h, int32_t kind, const double* node_coordinates) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh) return fail(h, TLW_E_STATE, "source terms follow the mesh upload");
    if (kind < 0 || kind > 1) return fail(h, TLW_E_ARG, "source kind: 0 none, 1 source_terms_convergence_test");
    if (kind && (h->parabolic || h->sc))
        return fail(h, TLW_E_UNSUPPORTED, "source terms: FR volume integral, Euler");
    if (kind && !node_coordinates) return fail(h, TLW_E_ARG, "node coordinates");
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    dfree(h->d_xnode); dfree(h->d_S2);
    h->source = 0;
    if (!kind) return TLW_OK;
    const size_t nx = (size_t)2 * h->n * h->n * h->E;
    TLW_CUDA(h, cudaMalloc(&h->d_xnode, nx * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_xnode, node_coordinates, nx * sizeof(double)));
    if (h->opts.time_discretization == TLW_MDRK) {
        int rc = ensure(h, h->d_S2, state_doubles(h));
        if (rc) return rc;
    }
    h->source = kind;
    return TLW_OK;
}

int tlw_set_halo(tlw_handle* h, int64_t n_halo, const int64_t* elements, const int32_t* faces) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || h->curved) return fail(h, TLW_E_STATE, "halo faces follow tlw_set_tree_mesh");
    if (n_halo > 0 && (h->parabolic || h->nmx + h->nmy > 0))
        return fail(h, TLW_E_UNSUPPORTED, "domain decomposition: LW or MDRK, conforming TreeMesh, Euler");
    if (n_halo < 0 || (n_halo > 0 && (!elements || !faces))) return fail(h, TLW_E_ARG, "halo faces");
    std::vector<int> he[2], hf[2], hs[2];
    std::vector<signed char> seen((size_t)h->E * 4, 0);
    for (int64_t k = 0; k < n_halo; ++k) {
        const int64_t e = elements[k] - 1;
        const int f = faces[k];
        if (e < 0 || e >= h->E || f < 0 || f > 3 || seen[(size_t)e * 4 + f])
            return fail(h, TLW_E_ARG, "halo face " + std::to_string(k + 1) + " out of range or repeated");
        seen[(size_t)e * 4 + f] = 1;
        const int c = f >> 1;
        he[c].push_back((int)e); hf[c].push_back(f); hs[c].push_back((int)k);
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    for (int** d : {&h->d_he, &h->d_hf, &h->d_hs})
        if (*d) { cudaFree(*d); *d = nullptr; }
    dfree(h->d_send); dfree(h->d_recv); dfree(h->d_asend); dfree(h->d_arecv);
    h->nh = (int)n_halo;
    h->nhx = (int)he[0].size();
    h->halo_values = h->sc ? HALO_VALUES_SC : HALO_VALUES;
    if (!h->s_comm) {
        TLW_CUDA(h, cudaStreamCreateWithFlags(&h->s_comm, cudaStreamNonBlocking));
        TLW_CUDA(h, cudaEventCreateWithFlags(&h->ev_lib, cudaEventDisableTiming));
        TLW_CUDA(h, cudaEventCreateWithFlags(&h->ev_comm, cudaEventDisableTiming));
    }
    h->slots_valid = false;
    if (n_halo > 0) {
        auto up = [&](int*& d, const std::vector<int>& a, const std::vector<int>& b) -> int {
            std::vector<int> v(a);
            v.insert(v.end(), b.begin(), b.end());
            TLW_CUDA(h, cudaMalloc(&d, v.size() * sizeof(int)));
            TLW_CUDA(h, upload_on(h->stream, d, v.data(), v.size() * sizeof(int)));
            return TLW_OK;
        };
        int rc;
        if ((rc = up(h->d_he, he[0], he[1])) || (rc = up(h->d_hf, hf[0], hf[1])) || (rc = up(h->d_hs, hs[0], hs[1])))
            return rc;
        const size_t nd = (size_t)n_halo * h->n * h->halo_values;
        TLW_CUDA(h, cudaMalloc(&h->d_send, nd * sizeof(double)));
        TLW_CUDA(h, cudaMalloc(&h->d_recv, nd * sizeof(double)));
        TLW_CUDA(h, zero_on(h->stream, h->d_send, nd * sizeof(double)));
        TLW_CUDA(h, zero_on(h->stream, h->d_recv, nd * sizeof(double)));
        if (h->sc) {
            TLW_CUDA(h, cudaMalloc(&h->d_asend, (size_t)n_halo * sizeof(double)));
            TLW_CUDA(h, cudaMalloc(&h->d_arecv, (size_t)n_halo * sizeof(double)));
            TLW_CUDA(h, zero_on(h->stream, h->d_asend, (size_t)n_halo * sizeof(double)));
            TLW_CUDA(h, zero_on(h->stream, h->d_arecv, (size_t)n_halo * sizeof(double)));
        }
    }
    return TLW_OK;
}

int32_t tlw_dd_halo_values(tlw_handle* h) { return h ? h->halo_values : 0; }

int tlw_dd_alpha_buffers(tlw_handle* h, double** send, double** recv) {
    if (!h) return TLW_E_ARG;
    if (send) *send = h->d_asend;
    if (recv) *recv = h->d_arecv;
    return TLW_OK;
}

int tlw_dd_buffers(tlw_handle* h, double** send, double** recv, unsigned long long** max_bits) {
    if (!h) return TLW_E_ARG;
    if (send) *send = h->d_send;
    if (recv) *recv = h->d_recv;
    if (max_bits) *max_bits = h->d_step ? &h->d_step->max_bits : nullptr;
    return TLW_OK;
}

// the comm stream continues after the work enqueued so far (the caller's collectives read what it wrote)
int dd_to_comm(tlw_handle* h) {
    if (!h->s_comm) return TLW_OK;
    TLW_CUDA(h, cudaEventRecord(h->ev_lib, h->stream));
    TLW_CUDA(h, cudaStreamWaitEvent(h->s_comm, h->ev_lib, 0));
    return TLW_OK;
}
// the stream continues after the caller's collectives enqueued on the comm stream so far
int dd_from_comm(tlw_handle* h) {
    if (!h->s_comm) return TLW_OK;
    TLW_CUDA(h, cudaEventRecord(h->ev_comm, h->s_comm));
    TLW_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_comm, 0));
    return TLW_OK;
}

int tlw_dd_comm_stream(tlw_handle* h, void** stream) {
    if (!h || !stream) return TLW_E_ARG;
    if (!h->s_comm) return fail(h, TLW_E_STATE, "the comm stream follows tlw_set_halo");
    *stream = (void*)h->s_comm;
    return TLW_OK;
}

int tlw_dd_begin(tlw_handle* h, double cfl, double fixed_dt, double t_end) {
    int rc = check_ready(h);
    if (rc) return rc;
    TLW_CUDA(h, cudaSetDevice(h->device));
    if ((rc = dd_from_comm(h))) return rc;
    double params[3] = {t_end, cfl, fixed_dt};
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->t_end, params, sizeof(params), cudaMemcpyHostToDevice, h->stream));
    h->dd_stage = 0;   // a step starts with its first stage
    // this part's maximum; the caller reduces it over the ranks (MAX) before tlw_dd_volume
    const double* u = h->d_state[h->cur];
    // with shock capturing the same pass gives the raw blending factors; the cut faces' go to the alpha buffer
    dispatch<Spd>(h->N, h->stream, u, (const double*)h->d_inv_jac, (int)h->E, h->opts.gamma, h->d_step, true, h->sc,
                  indicator_args(h));
    if (h->sc && h->nh > 0)
        halo_alpha_pack_kernel<<<(h->nh + 127) / 128, 128, 0, h->stream>>>(h->d_he, h->d_hs, h->nh, h->d_alpha_raw,
                                                                          h->d_asend);
    TLW_CUDA(h, cudaGetLastError());
    return dd_to_comm(h);
}

int32_t tlw_dd_stages(tlw_handle* h) {
    return (h && h->opts.time_discretization == TLW_MDRK) ? 2 : 1;
}

int tlw_dd_volume(tlw_handle* h) {
    int rc = check_ready(h);
    if (rc) return rc;
    TLW_CUDA(h, cudaSetDevice(h->device));
    if ((rc = dd_from_comm(h))) return rc;   // the all-reduce (and the alpha exchange) first
    const double* u = h->d_state[h->cur];
    double* unew = h->d_state[1 - h->cur];
    if (h->dd_stage == 0) {
        if (h->sc && h->opts.alpha_smooth) {
            // the smoothing inside the part and, with the neighbours' raw alpha, across the cut faces
            if (h->ni > 0)
                alpha_smooth_kernel<<<(h->ni + 255) / 256, 256, 0, h->stream>>>(h->d_il, h->d_ir, h->ni,
                                                                                h->d_alpha_raw, h->d_alpha);
            if (h->nh > 0)
                halo_alpha_smooth_kernel<<<(h->nh + 127) / 128, 128, 0, h->stream>>>(h->d_he, h->d_hs, h->nh,
                                                                                    h->d_arecv, h->d_alpha);
        }
        finalize_dt_kernel<<<1, 1, 0, h->stream>>>(h->d_step, h->n);
    }
    // the volume kernel and the packing, the hand-over to the comm stream (the exchange can start), then the x
    // faces inside the part while the traces travel
    for (int phases : {1, 2}) {
        if (h->opts.time_discretization == TLW_LW)
            enqueue_rhs(h, TLW_STAGE_LW, MODE_STEP, u, u, u, unew, &h->d_step->dt, nullptr, true, phases);
        else if (h->dd_stage == 0)   // MDRK stage 1 into u*, stage 2 from u* (the jumps are in u^n in both)
            enqueue_rhs(h, TLW_STAGE_MDRK1, MODE_STEP, u, u, u, h->d_us, &h->d_step->dt, nullptr, true, phases);
        else
            enqueue_rhs(h, TLW_STAGE_MDRK2, MODE_STEP, h->d_us, u, u, unew, &h->d_step->dt, nullptr, true, phases);
        if (phases == 1 && (rc = dd_to_comm(h))) return rc;
    }
    TLW_CUDA(h, cudaGetLastError());
    return TLW_OK;
}

int tlw_dd_finish(tlw_handle* h) {
    int rc = check_ready(h);
    if (rc) return rc;
    TLW_CUDA(h, cudaSetDevice(h->device));
    if ((rc = dd_from_comm(h))) return rc;   // the received traces
    const double* u = h->d_state[h->cur];
    double* unew = h->d_state[1 - h->cur];
    if (h->opts.time_discretization == TLW_LW) {
        enqueue_rhs(h, TLW_STAGE_LW, MODE_STEP, u, u, u, unew, &h->d_step->dt, nullptr, true, 4);
        enqueue_limiter(h, unew, 2, nullptr);
    } else if (h->dd_stage == 0) {
        enqueue_rhs(h, TLW_STAGE_MDRK1, MODE_STEP, u, u, u, h->d_us, &h->d_step->dt, nullptr, true, 4);
        h->dd_stage = 1;
        TLW_CUDA(h, cudaGetLastError());
        return TLW_OK;
    } else {
        enqueue_rhs(h, TLW_STAGE_MDRK2, MODE_STEP, h->d_us, u, u, unew, &h->d_step->dt, nullptr, true, 4);
        enqueue_limiter(h, unew, 1, nullptr);
        h->dd_stage = 0;
    }
    TLW_CUDA(h, cudaGetLastError());
    h->cur ^= 1;
    return TLW_OK;
}

int tlw_set_curved_mortars(tlw_handle* h, int64_t n_mortars, const int64_t* small1, const int64_t* small2,
                           const int32_t* small_faces, const int64_t* large, const int32_t* large_faces,
                           const int32_t* large_reversed) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || !h->curved) return fail(h, TLW_E_STATE, "curved mortars follow tlw_set_curved_mesh");
    if (h->unstructured && n_mortars > 0) return fail(h, TLW_E_UNSUPPORTED, "UnstructuredMesh2D is conforming");
    if (h->parabolic || h->ncb > 0)
        return fail(h, TLW_E_UNSUPPORTED, "curvilinear mortars: before the boundaries, without Navier-Stokes");
    if (n_mortars < 0 || (n_mortars > 0 && (!small1 || !small2 || !small_faces || !large || !large_faces || !large_reversed)))
        return fail(h, TLW_E_ARG, "mortars");
    struct Mtr { int s1, s2, l, code, cs, cl; };
    std::vector<Mtr> all;
    std::vector<signed char> used = h->face_used;
    for (int64_t k = 0; k < n_mortars; ++k) {
        const int64_t a = small1[k] - 1, b = small2[k] - 1, g = large[k] - 1;
        const int sf = small_faces[k], lf = large_faces[k], rv = large_reversed[k];
        if (a < 0 || a >= h->E || b < 0 || b >= h->E || g < 0 || g >= h->E || sf < 0 || sf > 3 || lf < 0 || lf > 3 ||
            (rv != 0 && rv != 1) || a == b || a == g || b == g)
            return fail(h, TLW_E_ARG, "mortar " + std::to_string(k + 1) + " out of range");
        for (size_t f : {(size_t)a * 4 + sf, (size_t)b * 4 + sf, (size_t)g * 4 + lf}) {
            if (used[f]) return fail(h, TLW_E_ARG, "mortar " + std::to_string(k + 1) + ": element face used twice");
            used[f] = 1;
        }
        all.push_back(Mtr{(int)a, (int)b, (int)g, sf | (lf << 2) | (rv << 4), sf >> 1, lf >> 1});
    }
    // colours as for the interfaces: within a colour no element has faces of both classes
    std::vector<std::vector<signed char>> cls;
    std::vector<std::vector<int>> bucket;
    for (size_t k = 0; k < all.size(); ++k) {
        const Mtr& m = all[k];
        size_t c = 0;
        for (; c < cls.size(); ++c) {
            const signed char x = cls[c][m.s1], y = cls[c][m.s2], z = cls[c][m.l];
            if ((x < 0 || x == m.cs) && (y < 0 || y == m.cs) && (z < 0 || z == m.cl)) break;
        }
        if (c == cls.size()) {
            cls.emplace_back((size_t)h->E, (signed char)-1);
            bucket.emplace_back();
        }
        cls[c][m.s1] = cls[c][m.s2] = (signed char)m.cs;
        cls[c][m.l] = (signed char)m.cl;
        bucket[c].push_back((int)k);
    }
    std::vector<int> v1, v2, vl, vc, off{0}, order;
    for (const auto& bk : bucket) {
        for (int k : bk) {
            v1.push_back(all[k].s1); v2.push_back(all[k].s2); vl.push_back(all[k].l); vc.push_back(all[k].code);
            order.push_back(k);
        }
        off.push_back((int)v1.size());
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    for (int** d : {&h->d_cms1, &h->d_cms2, &h->d_cml, &h->d_cmc, &h->d_cmsl, &h->d_cmsr})
        if (*d) { cudaFree(*d); *d = nullptr; }
    if (h->d_cmj) { cudaFree(h->d_cmj); h->d_cmj = nullptr; }
    auto up = [&](int*& d, const std::vector<int>& v) -> int {
        if (v.empty()) return TLW_OK;
        TLW_CUDA(h, cudaMalloc(&d, v.size() * sizeof(int)));
        TLW_CUDA(h, upload_on(h->stream, d, v.data(), v.size() * sizeof(int)));
        return TLW_OK;
    };
    int rc;
    if ((rc = up(h->d_cms1, v1)) || (rc = up(h->d_cms2, v2)) || (rc = up(h->d_cml, vl)) || (rc = up(h->d_cmc, vc)))
        return rc;
    // the positivity limiter's mortar pass: per large element its mortars in the caller's order (count in bits
    // 0-2, then the large face and whether its index runs backwards, 3 bits each)
    std::vector<int> desc((size_t)h->E, 0);
    for (int64_t k = 0; k < n_mortars; ++k) {
        const int g = (int)(large[k] - 1), c = desc[g] & 7;
        if (c >= 4) return fail(h, TLW_E_ARG, "mortar " + std::to_string(k + 1) + ": a fifth mortar of one element");
        desc[g] = (desc[g] & ~7) | (c + 1) | (((large_faces[k] & 3) | (large_reversed[k] << 2)) << (3 + 3 * c));
    }
    if (h->d_mface) { cudaFree(h->d_mface); h->d_mface = nullptr; }
    if (n_mortars > 0 && (rc = up(h->d_mface, desc))) return rc;
    // shock capturing: the blending factors are smoothed over the mortars too, (small 1, large) and
    // (small 2, large); lw_mortars.inverse_jacobian starts as zeros (tlw_set_curved_mortar_jacobian)
    std::vector<int> sl, sr;
    for (const Mtr& m : all) {
        sl.push_back(m.s1); sr.push_back(m.l);
        sl.push_back(m.s2); sr.push_back(m.l);
    }
    if ((rc = up(h->d_cmsl, sl)) || (rc = up(h->d_cmsr, sr))) return rc;
    h->ncms = (int)sl.size();
    if (n_mortars > 0) {
        TLW_CUDA(h, cudaMalloc(&h->d_cmj, (size_t)n_mortars * h->n * sizeof(double)));
        TLW_CUDA(h, zero_on(h->stream, h->d_cmj, (size_t)n_mortars * h->n * sizeof(double)));
    }
    h->mortar_order = order;
    h->ncm = (int)n_mortars;
    h->mortar_off = off;
    h->face_used = used;
    return TLW_OK;
}

int tlw_set_curved_mortar_jacobian(tlw_handle* h, const double* inverse_jacobian) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || !h->curved) return fail(h, TLW_E_STATE, "curved mortars follow tlw_set_curved_mesh");
    if (h->ncm == 0) return TLW_OK;
    std::vector<double> v((size_t)h->ncm * h->n, 0.0);
    if (inverse_jacobian)
        for (size_t c = 0; c < h->mortar_order.size(); ++c)
            for (int l = 0; l < h->n; ++l) v[c * h->n + l] = inverse_jacobian[(size_t)h->mortar_order[c] * h->n + l];
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    TLW_CUDA(h, upload_on(h->stream, h->d_cmj, v.data(), v.size() * sizeof(double)));
    return TLW_OK;
}

int tlw_set_curved_boundaries(tlw_handle* h, int64_t n_boundaries, const int64_t* elements, const int32_t* faces,
                              const int32_t* kinds) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || !h->curved) return fail(h, TLW_E_STATE, "curved boundaries follow tlw_set_curved_mesh");
    if (h->unstructured && n_boundaries > 0)
        return fail(h, TLW_E_UNSUPPORTED, "UnstructuredMesh2D: meshes without boundaries (the reference's boundary "
                                          "call matches no boundary-condition method)");
    if (n_boundaries < 0 || (n_boundaries > 0 && (!elements || !faces || !kinds))) return fail(h, TLW_E_ARG, "boundaries");
    std::vector<int> be[2], bf[2], bk[2], bi[2];
    std::vector<signed char> used = h->face_used;
    bool dirichlet = false;
    for (int64_t k = 0; k < n_boundaries; ++k) {
        const int64_t e = elements[k] - 1;
        const int f = faces[k];
        if (e < 0 || e >= h->E || f < 0 || f > 3)
            return fail(h, TLW_E_ARG, "boundary " + std::to_string(k + 1) + " out of range");
        if (kinds[k] != TLW_BC_DIRICHLET && kinds[k] != TLW_BC_SLIP_WALL_VERTICAL && kinds[k] != TLW_BC_SLIP_WALL_HORIZONTAL)
            return fail(h, TLW_E_ARG, "boundary " + std::to_string(k + 1) + ": unknown kind");
        if (kinds[k] == TLW_BC_DIRICHLET && h->parabolic)
            return fail(h, TLW_E_UNSUPPORTED, "curvilinear Navier-Stokes: slip walls are built");
        dirichlet = dirichlet || kinds[k] == TLW_BC_DIRICHLET;
        if (used[(size_t)e * 4 + f])
            return fail(h, TLW_E_ARG, "boundary " + std::to_string(k + 1) + ": the face already has a neighbour");
        used[(size_t)e * 4 + f] = 1;
        const int c = f >> 1;
        be[c].push_back((int)e); bf[c].push_back(f); bk[c].push_back(kinds[k]); bi[c].push_back((int)k);
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    for (int** d : {&h->d_cbe, &h->d_cbf, &h->d_cbk, &h->d_cbi})
        if (*d) { cudaFree(*d); *d = nullptr; }
    if (h->d_wkind) { cudaFree(h->d_wkind); h->d_wkind = nullptr; }
    dfree(h->d_wall);
    h->ncb = (int)n_boundaries;
    h->ncbx = (int)be[0].size();
    h->bnd_dirichlet = dirichlet;
    h->have_bdata = false;
    dfree(h->d_levels); dfree(h->d_now);
    if (n_boundaries > 0) {
        auto up = [&](int*& d, const std::vector<int>& a, const std::vector<int>& b) -> int {
            std::vector<int> v(a);
            v.insert(v.end(), b.begin(), b.end());
            TLW_CUDA(h, cudaMalloc(&d, v.size() * sizeof(int)));
            TLW_CUDA(h, upload_on(h->stream, d, v.data(), v.size() * sizeof(int)));
            return TLW_OK;
        };
        int rc;
        if ((rc = up(h->d_cbe, be[0], be[1])) || (rc = up(h->d_cbf, bf[0], bf[1])) || (rc = up(h->d_cbk, bk[0], bk[1])) ||
            (rc = up(h->d_cbi, bi[0], bi[1])))
            return rc;
    }
    if (h->d_atb) {
        // shock capturing: calcflux_muscl! falls back to first-order subcells on elements with a boundary face
        std::vector<unsigned char> atb((size_t)h->E, 0);
        for (int64_t k = 0; k < n_boundaries; ++k) atb[(size_t)(elements[k] - 1)] = 1;
        TLW_CUDA(h, upload_on(h->stream, h->d_atb, atb.data(), atb.size()));
    }
    return TLW_OK;
}

int tlw_set_boundary_kinds(tlw_handle* h, const int32_t* kinds) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || h->curved) return fail(h, TLW_E_STATE, "boundary kinds follow tlw_set_tree_mesh");
    if (h->nb == 0) return TLW_OK;
    if (!kinds) return fail(h, TLW_E_ARG, "kinds");
    bool dirichlet = false;
    for (int64_t k = 0; k < h->nb; ++k) {
        if (kinds[k] < TLW_BC_DIRICHLET || kinds[k] > TLW_BC_SLIP_WALL_HORIZONTAL)
            return fail(h, TLW_E_ARG, "boundary " + std::to_string(k + 1) + ": unknown kind");
        dirichlet = dirichlet || kinds[k] == TLW_BC_DIRICHLET;
    }
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    if (!h->d_bkind) TLW_CUDA(h, cudaMalloc(&h->d_bkind, (size_t)h->nb * sizeof(int)));
    TLW_CUDA(h, upload_on(h->stream, h->d_bkind, kinds, (size_t)h->nb * sizeof(int)));
    h->bnd_dirichlet = dirichlet;
    return TLW_OK;
}

int tlw_set_parabolic_walls(tlw_handle* h, const int32_t* kinds, const double* wall_data) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh || !h->parabolic) return fail(h, TLW_E_STATE, "walls follow tlw_set_parabolic");
    const int64_t nbnd = h->curved ? h->ncb : h->nb;
    if (nbnd == 0) return TLW_OK;
    if (!kinds || !wall_data) return fail(h, TLW_E_ARG, "kinds / wall data");
    for (int64_t k = 0; k < nbnd; ++k)
        if (kinds[k] != TLW_WALL_NOSLIP_ADIABATIC && kinds[k] != TLW_WALL_NOSLIP_ISOTHERMAL)
            return fail(h, TLW_E_ARG, "boundary " + std::to_string(k + 1) + ": unknown wall kind");
    const size_t nd = (size_t)3 * h->n * nbnd;
    for (size_t k = 0; k < nd; ++k)
        if (!std::isfinite(wall_data[k])) return fail(h, TLW_E_ARG, "wall data must be finite");
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    if (!h->d_wkind) TLW_CUDA(h, cudaMalloc(&h->d_wkind, (size_t)nbnd * sizeof(int)));
    if (!h->d_wall) TLW_CUDA(h, cudaMalloc(&h->d_wall, nd * sizeof(double)));
    TLW_CUDA(h, upload_on(h->stream, h->d_wkind, kinds, (size_t)nbnd * sizeof(int)));
    TLW_CUDA(h, upload_on(h->stream, h->d_wall, wall_data, nd * sizeof(double)));
    return TLW_OK;
}

int tlw_set_positivity_limiter(tlw_handle* h, int32_t count, const double* thresholds, const int32_t* variables) {
    if (!h) return TLW_E_ARG;
    if (count < 0 || count > TLW_LIMITER_MAX_PAIRS || (count > 0 && (!thresholds || !variables)))
        return fail(h, TLW_E_ARG, "limiter: 0..4 (threshold, variable) pairs");
    for (int p = 0; p < count; ++p)
        if (variables[p] < TLW_LIMIT_DENSITY || variables[p] > TLW_LIMIT_DENSITY_PRESSURE || !std::isfinite(thresholds[p]))
            return fail(h, TLW_E_ARG, "limiter: variable " + std::to_string(p + 1));
    if (h->stream) {
        TLW_CUDA(h, cudaSetDevice(h->device));
        TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    drop_graphs(h);
    h->lim_count = count;
    for (int p = 0; p < count; ++p) { h->lim_thr[p] = thresholds[p]; h->lim_var[p] = variables[p]; }
    return TLW_OK;
}

int tlw_apply_positivity_limiter(tlw_handle* h) {
    int rc = check_ready(h);
    if (rc) return rc;
    TLW_CUDA(h, cudaSetDevice(h->device));
    enqueue_limiter(h, h->d_state[h->cur], 1, (use_slots(h) && h->slots_valid) ? h->d_slots : nullptr);
    TLW_CUDA(h, cudaGetLastError());
    return TLW_OK;
}

int tlw_set_parabolic(tlw_handle* h, double mu, double prandtl) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh) return fail(h, TLW_E_STATE, "the parabolic terms follow tlw_set_tree_mesh / tlw_set_curved_mesh");
    if (h->unstructured) return fail(h, TLW_E_UNSUPPORTED, "Navier-Stokes: TreeMesh or P4estMesh-style curvilinear meshes");
    if (h->opts.time_discretization != TLW_LW || h->sc || h->N < 3 || h->nmx + h->nmy > 0 || h->ncm > 0)
        return fail(h, TLW_E_UNSUPPORTED, "Navier-Stokes: LW, FR volume integral, N >= 3, conforming mesh");
    if (!(mu >= 0.0) || !(prandtl > 0.0)) return fail(h, TLW_E_ARG, "mu / Prandtl");
    if (h->curved && h->ncb > 0 && h->bnd_dirichlet)
        return fail(h, TLW_E_UNSUPPORTED, "curvilinear Navier-Stokes: slip walls are built");
    TLW_CUDA(h, cudaSetDevice(h->device));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    int rc;
    if ((rc = ensure(h, h->d_gx, state_doubles(h))) || (rc = ensure(h, h->d_gy, state_doubles(h))) ||
        (rc = ensure(h, h->d_tFv, trace_doubles(h))))
        return rc;
    if (!h->d_visc) {
        TLW_CUDA(h, cudaMalloc(&h->d_visc, 2 * sizeof(unsigned long long)));
        TLW_CUDA(h, zero_on(h->stream, h->d_visc, 2 * sizeof(unsigned long long)));
    }
    if (h->source) return fail(h, TLW_E_UNSUPPORTED, "Navier-Stokes: without source terms");
    dispatch<ParAttr>(h->N);
    TLW_CUDA(h, cudaGetLastError());
    h->ns_mu = mu;
    h->ns_Pr = prandtl;
    h->parabolic = true;
    return TLW_OK;
}

static bool adaptive_finished_host(double t, double te) {
    return t == te || std::fabs(t - te) <= 1.4901161193847656e-08 * std::max(std::fabs(t), std::fabs(te));
}

// the trial of one Adaptive iteration into the other state buffer, dt from d_step->dt_call: the LW step with
// the temporal error estimate, the positivity limiter (perform_step!, adaptive.jl:131-132), the admissibility
// check and the sum of the per-element errors (d_check[4 * 148])
static int enqueue_adaptive_trial(tlw_handle* h, double abstol, double reltol) {
    const int blocks = (int)std::min<int64_t>(((int64_t)h->nn * h->E + 255) / 256, 4 * 148);
    const double* u = h->d_state[h->cur];
    double* trial = h->d_state[1 - h->cur];
    h->te_request = true;
    h->te_abstol = abstol;
    h->te_reltol = reltol;
    enqueue_rhs(h, TLW_STAGE_LW, MODE_STEP, u, u, u, trial, &h->d_step->dt_call);
    h->te_request = false;
    enqueue_limiter(h, trial, 1, nullptr);
    adaptive_check_kernel<<<blocks, 256, 0, h->stream>>>(h->d_te, (int)h->E, trial, (long long)h->nn * h->E,
                                                          h->opts.gamma, h->d_check, h->d_bad);
    adaptive_sum_kernel<<<1, 32, 0, h->stream>>>(h->d_check, blocks, h->d_check + 4 * 148);
    TLW_CUDA(h, cudaGetLastError());
    return TLW_OK;
}

static int adaptive_supported(tlw_handle* h) {
    // the reference's estimate comes from the LW volume kernels of depth 4 (TreeMesh) or 3 and 4 (curvilinear);
    // its MDRK kernels and the TreeMesh kernel of depth 3 leave temporal_errors unset
    if (h->opts.time_discretization != TLW_LW || h->parabolic || h->N < (h->curved ? 3 : 4))
        return fail(h, TLW_E_UNSUPPORTED, "Adaptive: LW, hyperbolic, N >= 4 on a TreeMesh or N >= 3 on a curvilinear mesh");
    if (h->source) return fail(h, TLW_E_UNSUPPORTED, "Adaptive: without source terms");
    TLW_CUDA(h, cudaSetDevice(h->device));
    if (!h->d_te) {
        TLW_CUDA(h, cudaMalloc(&h->d_te, (size_t)h->E * sizeof(double)));
        TLW_CUDA(h, cudaMalloc(&h->d_check, (size_t)(4 * 148 + 1) * sizeof(double)));
        TLW_CUDA(h, cudaMalloc(&h->d_bad, sizeof(unsigned)));
        TLW_CUDA(h, zero_on(h->stream, h->d_bad, sizeof(unsigned)));
    }
    return TLW_OK;
}

int tlw_adaptive_begin(tlw_handle* h, double t_end, double dt_initial, const double* controller) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!(dt_initial > 0.0) || !std::isfinite(t_end)) return fail(h, TLW_E_ARG, "t_end / dt_initial");
    if ((rc = adaptive_supported(h))) return rc;
    if (!h->d_adapt) TLW_CUDA(h, cudaMalloc(&h->d_adapt, sizeof(AdaptiveState)));
    StepState st{};
    TLW_CUDA(h, cudaMemcpyAsync(&st, h->d_step, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    AdaptiveState a{};
    a.eps[0] = a.eps[1] = a.eps[2] = 1.0;
    a.beta[0] = controller ? controller[0] : 0.6;
    a.beta[1] = controller ? controller[1] : -0.2;
    a.beta[2] = controller ? controller[2] : 0.0;
    a.t_end = t_end;
    a.dt = st.t + dt_initial > t_end ? t_end - st.t : dt_initial;   // set_dt!
    a.k = (double)h->n;
    a.ndofs = (double)h->nn * (double)h->E;
    TLW_CUDA(h, upload_on(h->stream, h->d_adapt, &a, sizeof(a)));
    TLW_CUDA(h, zero_on(h->stream, h->d_bad, sizeof(unsigned)));
    TLW_CUDA(h, zero_on(h->stream, &h->d_step->status, sizeof(unsigned)));   // no stale flag rejects trial 1
    return TLW_OK;
}

int tlw_adaptive_run(tlw_handle* h, int32_t n_trials, double abstol, double reltol, int64_t* steps,
                     int64_t* rejected, int32_t* finished) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!h->d_adapt) return fail(h, TLW_E_STATE, "tlw_adaptive_run follows tlw_adaptive_begin");
    if (n_trials < 0 || !steps || !rejected || !finished) return fail(h, TLW_E_ARG, "arguments");
    if ((rc = adaptive_supported(h))) return rc;
    const long long count = (long long)h->nn * h->E * NV;
    const int cblocks = (int)std::min<long long>((count + 255) / 256, 8 * 148);
    for (int q = 0; q < n_trials; ++q) {
        adaptive_prepare_kernel<<<1, 1, 0, h->stream>>>(h->d_step, h->d_adapt);
        if ((rc = enqueue_adaptive_trial(h, abstol, reltol))) return rc;
        adaptive_judge_kernel<<<1, 1, 0, h->stream>>>(h->d_step, h->d_adapt, h->d_check + 4 * 148, h->d_bad);
        // the accepted state is limited once more (solve_lwfr's loop, lwfr.jl:257); a rejected trial is
        // overwritten by the next one
        enqueue_limiter(h, h->d_state[1 - h->cur], 1, nullptr);
        adaptive_commit_kernel<<<cblocks, 256, 0, h->stream>>>(h->d_adapt, h->d_state[1 - h->cur],
                                                               h->d_state[h->cur], count);
        TLW_CUDA(h, cudaGetLastError());
    }
    AdaptiveState a{};
    StepState st{};
    TLW_CUDA(h, cudaMemcpyAsync(&a, h->d_adapt, sizeof(a), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&st, h->d_step, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    h->slots_valid = false;
    *steps = st.steps;
    *rejected = a.nreject;
    *finished = adaptive_finished_host(st.t, a.t_end) ? 1 : 0;
    if (a.stalled && !*finished)
        return fail(h, TLW_E_NONADMISSIBLE, "Adaptive: dt fell below 1e-14 |t| after repeated rejections "
                                            "(persistently non-admissible state)");
    return TLW_OK;
}

int tlw_adaptive_trial(tlw_handle* h, double dt, double abstol, double reltol, double* total_temporal_error,
                       int32_t* admissible) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!total_temporal_error || !admissible || !(dt > 0.0)) return fail(h, TLW_E_ARG, "arguments");
    if ((rc = adaptive_supported(h))) return rc;
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->dt_call, &dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    TLW_CUDA(h, cudaMemsetAsync(h->d_bad, 0, sizeof(unsigned), h->stream));
    if ((rc = enqueue_adaptive_trial(h, abstol, reltol))) return rc;
    double sum = 0.0;
    unsigned bad = 0, st = 0;
    TLW_CUDA(h, cudaMemcpyAsync(&sum, h->d_check + 4 * 148, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&bad, h->d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&st, &h->d_step->status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    if (st) {   // a square root of a negative number: the reference's test_rhs! catches the DomainError
        const unsigned zero = 0;
        TLW_CUDA(h, upload_on(h->stream, &h->d_step->status, &zero, sizeof(zero)));
    }
    *admissible = (bad == 0 && st == 0) ? 1 : 0;
    *total_temporal_error = std::sqrt(sum / ((double)h->nn * (double)h->E));
    return TLW_OK;
}

int tlw_adaptive_accept(tlw_handle* h, double dt) {
    int rc = check_ready(h);
    if (rc) return rc;
    TLW_CUDA(h, cudaSetDevice(h->device));
    adaptive_accept_kernel<<<1, 1, 0, h->stream>>>(h->d_step, dt);
    enqueue_limiter(h, h->d_state[1 - h->cur], 1, nullptr);   // solve_lwfr's loop (lwfr.jl:257)
    TLW_CUDA(h, cudaGetLastError());
    h->cur ^= 1;
    h->slots_valid = false;
    return TLW_OK;
}

int32_t tlw_curved_colors(tlw_handle* h) {
    return (h && h->curved) ? (int32_t)h->color_off.size() - 1 : 0;
}

int tlw_set_boundary_data(tlw_handle* h, const double* levels, const double* now, int32_t where) {
    if (!h) return TLW_E_ARG;
    if (!h->have_mesh) return fail(h, TLW_E_STATE, "no mesh");
    const int64_t nbnd = h->curved ? h->ncb : h->nb;
    if (nbnd == 0) return TLW_OK;
    if (!levels || !now) return fail(h, TLW_E_ARG, "boundary data pointers");
    const size_t nl = (size_t)NV * h->n * h->n * nbnd, nw = (size_t)NV * h->n * nbnd;
    int rc;
    if ((rc = ensure(h, h->d_levels, nl)) || (rc = ensure(h, h->d_now, nw))) return rc;
    const cudaMemcpyKind k = where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    TLW_CUDA(h, cudaMemcpyAsync(h->d_levels, levels, nl * sizeof(double), k, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(h->d_now, now, nw * sizeof(double), k, h->stream));
    if (where != TLW_WHERE_DEVICE) TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    h->have_bdata = true;
    return TLW_OK;
}

int tlw_rhs(tlw_handle* h, int32_t stage, double* du, const double* u, const double* us, double t, double dt,
            int32_t where) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (h->nh > 0) return fail(h, TLW_E_STATE, "a partitioned mesh steps with tlw_dd_begin / _volume / _finish");
    if (!du || !u || (stage == TLW_STAGE_MDRK2 && !us)) return fail(h, TLW_E_ARG, "null pointer");
    if (stage < TLW_STAGE_LW || stage > TLW_STAGE_MDRK2) return fail(h, TLW_E_ARG, "stage");
    if (stage != TLW_STAGE_LW && h->opts.time_discretization != TLW_MDRK)
        return fail(h, TLW_E_STATE, "MDRK stages need a handle created with TLW_MDRK");
    TLW_CUDA(h, cudaSetDevice(h->device));
    const size_t bytes = state_doubles(h) * sizeof(double);
    const double tdt[2] = {dt, t};   // dt_call, then (after t_step) t_call: the source terms' time
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->dt_call, &tdt[0], sizeof(double), cudaMemcpyHostToDevice, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->t_call, &tdt[1], sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const double *du_in = u, *dus = us;
    double* dout = du;
    // host arrays, and device arrays whose node records are not 32-byte aligned (the surface pass reads and writes
    // a node's four doubles at once), go through the handle's own buffers
    const uintptr_t bits = (uintptr_t)u | (uintptr_t)du | (stage == TLW_STAGE_MDRK2 ? (uintptr_t)us : 0);
    const bool staged = where == TLW_WHERE_HOST || bits % 32 != 0;
    if (staged) {
        const cudaMemcpyKind in = where == TLW_WHERE_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        if ((rc = ensure(h, h->d_in, state_doubles(h))) || (rc = ensure(h, h->d_out, state_doubles(h)))) return rc;
        TLW_CUDA(h, cudaMemcpyAsync(h->d_in, u, bytes, in, h->stream));
        du_in = h->d_in;
        if (stage == TLW_STAGE_MDRK2) {
            if ((rc = ensure(h, h->d_in2, state_doubles(h)))) return rc;
            TLW_CUDA(h, cudaMemcpyAsync(h->d_in2, us, bytes, in, h->stream));
            dus = h->d_in2;
        }
        dout = h->d_out;
    }
    const double* u_flux = stage == TLW_STAGE_MDRK2 ? dus : du_in;
    enqueue_rhs(h, stage, MODE_RHS, u_flux, du_in, du_in, dout, &h->d_step->dt_call);
    TLW_CUDA(h, cudaGetLastError());
    if (staged) {
        const cudaMemcpyKind out = where == TLW_WHERE_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        TLW_CUDA(h, cudaMemcpyAsync(du, h->d_out, bytes, out, h->stream));
        if (where == TLW_WHERE_HOST) return read_status(h);
    }
    return TLW_OK;
}

int tlw_max_dt(tlw_handle* h, const double* u, int32_t where, double cfl, double* dt_out) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!u || !dt_out) return fail(h, TLW_E_ARG, "null pointer");
    TLW_CUDA(h, cudaSetDevice(h->device));
    const double* du_in = u;
    // host arrays, and device arrays whose node records are not 32-byte aligned, through the handle's buffer
    if (where == TLW_WHERE_HOST || (uintptr_t)u % 32 != 0) {
        const cudaMemcpyKind in = where == TLW_WHERE_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
        if ((rc = ensure(h, h->d_in, state_doubles(h)))) return rc;
        TLW_CUDA(h, cudaMemcpyAsync(h->d_in, u, state_doubles(h) * sizeof(double), in, h->stream));
        du_in = h->d_in;
    }
    const unsigned long long zero = 0;
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->max_bits, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->stream));
    if (h->parabolic) {
        // the maxima, combined on the host exactly as par_finalize_dt_kernel does
        const unsigned long long zeros[2] = {0, 0};
        TLW_CUDA(h, cudaMemcpyAsync(h->d_visc, zeros, sizeof(zeros), cudaMemcpyHostToDevice, h->stream));
        dispatch<ParSpd>(h->N, h->stream, (const tlw_handle*)h, du_in);
        TLW_CUDA(h, cudaGetLastError());
        unsigned long long ba = 0, bv[2] = {0, 0};
        TLW_CUDA(h, cudaMemcpyAsync(&ba, &h->d_step->max_bits, sizeof(ba), cudaMemcpyDeviceToHost, h->stream));
        TLW_CUDA(h, cudaMemcpyAsync(bv, h->d_visc, sizeof(bv), cudaMemcpyDeviceToHost, h->stream));
        TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->max_bits, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->stream));
        TLW_CUDA(h, cudaMemcpyAsync(h->d_visc, zeros, sizeof(zeros), cudaMemcpyHostToDevice, h->stream));
        if ((rc = read_status(h))) return rc;
        double la, lv, lq;
        std::memcpy(&la, &ba, sizeof(la));
        std::memcpy(&lv, &bv[0], sizeof(lv));
        std::memcpy(&lq, &bv[1], sizeof(lq));
        if (!h->curved) lq = la;
        const double tiny = 4.9406564584124654e-324;
        if (!(la > tiny)) la = tiny;
        if (!(lv > tiny)) lv = tiny;
        if (!(lq > tiny)) lq = tiny;
        const double k = 2.0 * (2.0 * h->N + 1.0);
        *dt_out = std::fmin(cfl * (2.0 / (h->n * la)), cfl / ((lq + lv * k) * k));
        return TLW_OK;
    }
    if (h->curved)
        dispatch<CSpd>(h->N, h->stream, du_in, (const double*)h->d_Ja, (const double*)h->d_ijn, (int)h->E,
                       h->opts.gamma, h->d_step);
    else
        dispatch<Spd>(h->N, h->stream, du_in, (const double*)h->d_inv_jac, (int)h->E, h->opts.gamma, h->d_step,
                      true, false, indicator_args(h));
    TLW_CUDA(h, cudaGetLastError());
    unsigned long long bits = 0;
    TLW_CUDA(h, cudaMemcpyAsync(&bits, &h->d_step->max_bits, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->max_bits, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->stream));
    if ((rc = read_status(h))) return rc;
    double m;
    std::memcpy(&m, &bits, sizeof(m));
    const double tiny = 4.9406564584124654e-324;
    if (!(m > tiny)) m = tiny;
    *dt_out = cfl * (2.0 / (h->n * m));
    return TLW_OK;
}

int tlw_set_state(tlw_handle* h, const double* u, int32_t where, double t) {
    if (h) h->slots_valid = false;
    int rc = check_ready(h);
    if (rc) return rc;
    if (!u) return fail(h, TLW_E_ARG, "null pointer");
    TLW_CUDA(h, cudaSetDevice(h->device));
    const cudaMemcpyKind k = where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    TLW_CUDA(h, cudaMemcpyAsync(h->d_state[h->cur], u, state_doubles(h) * sizeof(double), k, h->stream));
    StepState* sp = h->d_step;
    const long long zero = 0;
    TLW_CUDA(h, cudaMemcpyAsync(&sp->t, &t, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&sp->steps, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->stream));
    if (where != TLW_WHERE_DEVICE) TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    return TLW_OK;
}

int tlw_get_state(tlw_handle* h, double* u, int32_t where, double* t_out) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (!u) return fail(h, TLW_E_ARG, "null pointer");
    TLW_CUDA(h, cudaSetDevice(h->device));
    const cudaMemcpyKind k = where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    TLW_CUDA(h, cudaMemcpyAsync(u, h->d_state[h->cur], state_doubles(h) * sizeof(double), k, h->stream));
    double t = 0;
    if (t_out) TLW_CUDA(h, cudaMemcpyAsync(&t, &h->d_step->t, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (where != TLW_WHERE_DEVICE || t_out) {
        if ((rc = read_status(h))) return rc;
    }
    if (t_out) *t_out = t;
    return TLW_OK;
}

namespace {
// the buffer pool, copy streams and events of tlw_step_host (created on its first call)
int ensure_host_stepping(tlw_handle* h) {
    if (!h->s_up) {
        TLW_CUDA(h, cudaStreamCreateWithFlags(&h->s_up, cudaStreamNonBlocking));
        TLW_CUDA(h, cudaStreamCreateWithFlags(&h->s_down, cudaStreamNonBlocking));
        for (cudaEvent_t* ev : {&h->ev_up, &h->ev_computed, &h->ev_prior})
            TLW_CUDA(h, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
        // (a wait on an event never recorded returns at once: nothing is in flight yet)
        for (cudaEvent_t& ev : h->ev_free) TLW_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        for (cudaEvent_t& ev : h->ev_dl) TLW_CUDA(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    if (!h->host_pool[0]) {
        // the handle's two state buffers and three more; the first upload into the state buffers waits for the
        // work other entry points have enqueued on them
        const size_t bytes = state_doubles(h) * sizeof(double);
        h->host_pool[0] = h->d_state[0];
        h->host_pool[1] = h->d_state[1];
        for (int k = 0; k < tlw_handle::HOST_POOL; ++k)
            if (!h->host_pool[k]) TLW_CUDA(h, cudaMalloc(&h->host_pool[k], bytes));
        TLW_CUDA(h, cudaEventRecord(h->ev_prior, h->stream));
        TLW_CUDA(h, cudaStreamWaitEvent(h->s_up, h->ev_prior, 0));
    }
    return TLW_OK;
}
}  // namespace

int tlw_step_host(tlw_handle* h, const double* u_in, double* u_out, double t, int32_t nsteps, double cfl,
                  double fixed_dt, double t_end) {
    int rc = check_ready(h, false);
    if (rc) return rc;
    if (!u_in || !u_out || nsteps < 1) return fail(h, TLW_E_ARG, "tlw_step_host: u_in, u_out, nsteps >= 1");
    if (h->nh > 0) return fail(h, TLW_E_STATE, "a partitioned mesh steps with tlw_dd_begin / _volume / _finish");
    TLW_CUDA(h, cudaSetDevice(h->device));
    if ((rc = ensure_host_stepping(h))) return rc;
    const size_t bytes = state_doubles(h) * sizeof(double);
    constexpr int P = tlw_handle::HOST_POOL, K = tlw_handle::HOST_CALLS;
    // call k takes pool buffers 2k and 2k + 1 (mod 5): A receives the upload, B is the steps' other buffer. A was
    // last used three calls back and B two calls back, so the upload of call k waits at most for the download of
    // call k - 3, and the uploads, steps and downloads of three consecutive calls overlap.
    const long long k = h->host_calls;
    const int ia = (int)((2 * k) % P), ib = (int)((2 * k + 1) % P);
    double* A = h->host_pool[ia];
    double* B = h->host_pool[ib];
    // 1. upload into A after its last use and after the downloads up to call k - 3 (in order on their stream; they
    //    have finished by then in a full pipeline); a u_in that call k - 1 or k - 2 downloads into is read after that
    //    download (the state round-tripping through the host)
    TLW_CUDA(h, cudaStreamWaitEvent(h->s_up, h->ev_free[ia], 0));
    if (k >= 3) TLW_CUDA(h, cudaStreamWaitEvent(h->s_up, h->ev_dl[(k - 3) % K], 0));
    for (long long j = k - 1; j >= 0 && j >= k - 2; --j)
        if (h->dl_out[j % K] == u_in) TLW_CUDA(h, cudaStreamWaitEvent(h->s_up, h->ev_dl[j % K], 0));
    TLW_CUDA(h, cudaMemcpyAsync(A, u_in, bytes, cudaMemcpyHostToDevice, h->s_up));
    TLW_CUDA(h, cudaEventRecord(h->ev_up, h->s_up));
    // the next upload also waits for the compute stream's work enqueued so far (other entry points between the
    // calls may have used any buffer of the pair that is current now)
    TLW_CUDA(h, cudaEventRecord(h->ev_prior, h->stream));
    TLW_CUDA(h, cudaStreamWaitEvent(h->s_up, h->ev_prior, 0));
    // 2. the steps from A, with B as the other buffer, after the upload and after B's last use
    TLW_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_up, 0));
    TLW_CUDA(h, cudaStreamWaitEvent(h->stream, h->ev_free[ib], 0));
    h->d_state[0] = A;
    h->d_state[1] = B;
    h->cur = 0;
    drop_graphs(h);   // they address the previous buffers
    h->slots_valid = false;
    StepState* sp = h->d_step;
    const long long zero = 0;
    TLW_CUDA(h, cudaMemcpyAsync(&sp->t, &t, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    TLW_CUDA(h, cudaMemcpyAsync(&sp->steps, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->stream));
    h->async_pending = false;
    if ((rc = tlw_step(h, nsteps, cfl, fixed_dt, t_end, 0))) return rc;
    const int ir = h->cur == 0 ? ia : ib, io = h->cur == 0 ? ib : ia;   // the result's buffer and the other
    TLW_CUDA(h, cudaEventRecord(h->ev_free[io], h->stream));
    TLW_CUDA(h, cudaEventRecord(h->ev_computed, h->stream));
    // 3. download the result
    TLW_CUDA(h, cudaStreamWaitEvent(h->s_down, h->ev_computed, 0));
    TLW_CUDA(h, cudaMemcpyAsync(u_out, h->d_state[h->cur], bytes, cudaMemcpyDeviceToHost, h->s_down));
    TLW_CUDA(h, cudaEventRecord(h->ev_free[ir], h->s_down));
    TLW_CUDA(h, cudaEventRecord(h->ev_dl[k % K], h->s_down));
    h->dl_out[k % K] = u_out;
    h->host_calls += 1;
    h->async_pending = true;
    return TLW_OK;
}

int tlw_step(tlw_handle* h, int32_t nsteps, double cfl, double fixed_dt, double t_end, int32_t use_graph) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (h->nh > 0) return fail(h, TLW_E_STATE, "a partitioned mesh steps with tlw_dd_begin / _volume / _finish");
    if (nsteps < 0) return fail(h, TLW_E_ARG, "nsteps");
    if (nsteps == 0) return TLW_OK;
    TLW_CUDA(h, cudaSetDevice(h->device));
    // parameters into the device step state (cfl, fixed_dt, t_end are contiguous after t)
    double params[3] = {t_end, cfl, fixed_dt};
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->t_end, params, sizeof(params), cudaMemcpyHostToDevice, h->stream));
    if (use_slots(h) && !h->slots_valid) {
        // one step with the full CFL pass; it leaves the per-element slots that later steps reduce
        enqueue_step(h, h->cur);
        h->cur ^= 1;
        h->slots_valid = true;
        if (--nsteps == 0) {
            TLW_CUDA(h, cudaGetLastError());
            return TLW_OK;
        }
    }
    if (!use_graph) {
        for (int s = 0; s < nsteps; ++s) {
            enqueue_step(h, h->cur);
            h->cur ^= 1;
        }
        TLW_CUDA(h, cudaGetLastError());
        return TLW_OK;
    }
    auto capture = [&](int from, int count, cudaGraphExec_t& exec) -> int {
        if (exec) return TLW_OK;
        cudaGraph_t g = nullptr;
        TLW_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int b = from;
        for (int s = 0; s < count; ++s) { enqueue_step(h, b); b ^= 1; }
        cudaError_t e1 = cudaStreamEndCapture(h->stream, &g);
        if (e1 != cudaSuccess) return fail(h, TLW_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e1));
        cudaError_t e2 = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) { exec = nullptr; return fail(h, TLW_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2)); }
        return TLW_OK;
    };
    // capture every variant on first use, so that no capture/instantiation lands inside a later call
    if ((rc = capture(0, 1, h->g_one[0])) || (rc = capture(1, 1, h->g_one[1])) || (rc = capture(0, 2, h->g_two[0])))
        return rc;
    int left = nsteps;
    if (h->cur == 1) {
        if ((rc = capture(1, 1, h->g_one[1]))) return rc;
        TLW_CUDA(h, cudaGraphLaunch(h->g_one[1], h->stream));
        h->cur = 0;
        --left;
    }
    if (left >= 2) {
        if ((rc = capture(0, 2, h->g_two[0]))) return rc;
        for (; left >= 2; left -= 2) TLW_CUDA(h, cudaGraphLaunch(h->g_two[0], h->stream));
    }
    if (left == 1) {
        if ((rc = capture(0, 1, h->g_one[0]))) return rc;
        TLW_CUDA(h, cudaGraphLaunch(h->g_one[0], h->stream));
        h->cur = 1;
    }
    return TLW_OK;
}

int tlw_step_timed(tlw_handle* h, int32_t nsteps, double cfl, double fixed_dt, double t_end, double* phase_ms) {
    int rc = check_ready(h);
    if (rc) return rc;
    if (h->nh > 0) return fail(h, TLW_E_STATE, "a partitioned mesh steps with tlw_dd_begin / _volume / _finish");
    if (nsteps < 0 || !phase_ms) return fail(h, TLW_E_ARG, "nsteps / phase_ms");
    TLW_CUDA(h, cudaSetDevice(h->device));
    double params[3] = {t_end, cfl, fixed_dt};
    TLW_CUDA(h, cudaMemcpyAsync(&h->d_step->t_end, params, sizeof(params), cudaMemcpyHostToDevice, h->stream));
    const int nstage = h->opts.time_discretization == TLW_LW ? 1 : 2;
    std::vector<cudaEvent_t> evs((size_t)nsteps * (2 + 3 * nstage));
    for (auto& e : evs) TLW_CUDA(h, cudaEventCreate(&e));
    size_t k = 0;
    std::vector<size_t> starts;
    for (int s = 0; s < nsteps; ++s) {
        starts.push_back(k);
        cudaEvent_t e_start = evs[k++], e_dt = evs[k++];
        PhaseEvents pe[2];
        for (int st = 0; st < nstage; ++st) pe[st] = {evs[k++], evs[k++], evs[k++]};
        cudaEventRecord(e_start, h->stream);
        enqueue_step(h, h->cur, e_dt, pe);
        h->cur ^= 1;
        if (use_slots(h)) h->slots_valid = true;
    }
    TLW_CUDA(h, cudaGetLastError());
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int p = 0; p < 5; ++p) phase_ms[p] = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        size_t b = starts[s];
        float ms;
        cudaEventElapsedTime(&ms, evs[b], evs[b + 1]);
        phase_ms[0] += ms;
        cudaEvent_t prev = evs[b + 1];
        for (int st = 0; st < nstage; ++st) {
            cudaEvent_t* pe = &evs[b + 2 + 3 * st];
            cudaEventElapsedTime(&ms, prev, pe[0]); phase_ms[1] += ms;
            cudaEventElapsedTime(&ms, pe[0], pe[1]); phase_ms[2] += ms;
            cudaEventElapsedTime(&ms, pe[1], pe[2]); phase_ms[3] += ms;
            prev = pe[2];
        }
        cudaEventElapsedTime(&ms, evs[b], prev);
        phase_ms[4] += ms;
    }
    for (auto& e : evs) cudaEventDestroy(e);
    return read_status(h);
}

int tlw_probe_fp64_tflops(int32_t device, double* tflops) {
    if (!tflops) return TLW_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return TLW_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int threads = 256, blocks = sms * 8, iters = 1 << 14;
    double* out = nullptr;
    if (cudaMalloc(&out, (size_t)threads * blocks * sizeof(double)) != cudaSuccess) return TLW_E_CUDA;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(a);
        fp64_probe_kernel<<<blocks, threads>>>(out, iters, 0.9999999, 1e-7);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && ms < best) best = ms;   // first launch is warm-up
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (err != cudaSuccess) return TLW_E_CUDA;
    *tflops = 2.0 * 16.0 * iters * (double)threads * blocks / (best * 1e-3) / 1e12;
    return TLW_OK;
}

int tlw_probe_reciprocal(int32_t device, const double* x, double* y, int64_t n) {
    if (!x || !y || n < 0) return TLW_E_ARG;
    if (n == 0) return TLW_OK;
    if (cudaSetDevice(device) != cudaSuccess) return TLW_E_CUDA;
    double* d = nullptr;
    if (cudaMalloc(&d, 2 * (size_t)n * sizeof(double)) != cudaSuccess) return TLW_E_CUDA;
    cudaError_t e = cudaMemcpy(d, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        reciprocal_probe_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4 * 148), 256>>>(d, d + n, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? TLW_OK : TLW_E_CUDA;
}

int tlw_get_time(tlw_handle* h, double* t, double* dt_last, int64_t* steps) {
    if (!h) return TLW_E_ARG;
    TLW_CUDA(h, cudaSetDevice(h->device));
    StepState st{};
    TLW_CUDA(h, cudaMemcpyAsync(&st, h->d_step, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    int rc = read_status(h);
    if (t) *t = st.t;
    if (dt_last) *dt_last = st.dt;
    if (steps) *steps = st.steps;
    return rc;
}

int64_t tlw_cache_size(tlw_handle* h, int32_t item) {
    if (!h || !h->have_mesh) return -1;
    switch (item) {
        case TLW_CACHE_U_TRACES:
        case TLW_CACHE_F_TRACES: return (int64_t)trace_doubles(h);
        case TLW_CACHE_U2: return h->d_U2 ? (int64_t)state_doubles(h) : -1;
        case TLW_CACHE_F2: return h->d_F2 ? (int64_t)(2 * state_doubles(h)) : -1;
        case TLW_CACHE_ALPHA: return h->d_alpha ? (int64_t)h->E : -1;
        case TLW_CACHE_FN_LOW: return h->d_tFn ? (int64_t)trace_doubles(h) : -1;
        default: return -1;
    }
}

int tlw_get_cache(tlw_handle* h, int32_t item, double* out, int32_t where) {
    if (!h || !out) return TLW_E_ARG;
    const int64_t count = tlw_cache_size(h, item);
    if (count < 0) return fail(h, TLW_E_ARG, "cache item not available");
    const double* src = item == TLW_CACHE_U_TRACES ? h->d_tU : item == TLW_CACHE_F_TRACES ? h->d_tF
                        : item == TLW_CACHE_U2 ? h->d_U2 : item == TLW_CACHE_F2 ? h->d_F2
                        : item == TLW_CACHE_ALPHA ? h->d_alpha : h->d_tFn;
    TLW_CUDA(h, cudaSetDevice(h->device));
    const cudaMemcpyKind k = where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    TLW_CUDA(h, cudaMemcpyAsync(out, src, count * sizeof(double), k, h->stream));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    return TLW_OK;
}

int tlw_synchronize(tlw_handle* h) {
    if (!h) return TLW_E_ARG;
    TLW_CUDA(h, cudaSetDevice(h->device));
    if (h->s_up) TLW_CUDA(h, cudaStreamSynchronize(h->s_up));
    if (h->s_down) TLW_CUDA(h, cudaStreamSynchronize(h->s_down));
    TLW_CUDA(h, cudaStreamSynchronize(h->stream));
    TLW_CUDA(h, cudaGetLastError());
    return read_status(h);
}

int tlw_get_stream(tlw_handle* h, void** stream) {
    if (!h || !stream) return TLW_E_ARG;
    *stream = (void*)h->stream;
    return TLW_OK;
}

int tlw_state_pointer(tlw_handle* h, double** dptr) {
    if (h) h->slots_valid = false;   // the caller may write the state through the pointer
    if (!h || !dptr) return TLW_E_ARG;
    if (!h->have_mesh) return fail(h, TLW_E_STATE, "no mesh");
    *dptr = h->d_state[h->cur];
    return TLW_OK;
}

const char* tlw_last_error(tlw_handle* h) { return h ? h->err.c_str() : "null handle"; }

}  // extern "C"
