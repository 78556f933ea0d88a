// tlw_handle.h -- internal: the handle behind tlw_handle* (shared by the translation units of libtlw that
// launch on a handle's mesh and buffers). Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/tlw.h"
#include "tlw_device.cuh"
#include "tlw_surface.cuh"

namespace tlw {

template <class T>
inline void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// device buffers of the discrete adjoint (allocated on first use by the adjoint entry points)
struct AdjointBuffers {
    int64_t E = 0;                          // element count the buffers were sized for
    int capacity_steps = 0;                 // dt sequence capacity
    int capacity_states = 0;                // states of one checkpoint segment
    int capacity_buffers = 0;               // segment buffers allocated (1 or 2)
    double* d_lam[2] = {nullptr, nullptr};  // adjoint state ping-pong
    double *d_bF = nullptr, *d_bU = nullptr, *d_bu = nullptr;   // face-trace adjoints [v, l, face, e]
    double* d_dts = nullptr;                // dt of every recorded forward step
    double* d_dts_given = nullptr;          // dt sequence given by the caller (fixed-dt solves)
    int capacity_given = 0;
    double* d_ckpt = nullptr;               // checkpoint states
    int capacity_ckpt = 0;
    // segment buffers (two when a run has several segments: one is recomputed while the reverse sweep reads
    // the other), each of capacity_states steps: the step input states (+1 slot: u(T), or scratch), U traces,
    // stage derivatives
    double* d_seg = nullptr;                // [buffers][capacity_states + 1] states
    double* d_segU = nullptr;               // [buffers][capacity_states] time-averaged U traces
    double* d_segD = nullptr;               // [buffers][capacity_states][depth] stage derivatives d_1..d_depth
    bool last_resident = false;             // the recorded run's last segment is in its buffer (no recompute)
    cudaStream_t s_rec = nullptr;           // reverse sweep: recompute stream (lowest priority)
    cudaStream_t s_adj = nullptr;           // reverse sweep: adjoint chain (highest priority)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
    cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    double* d_work = nullptr;               // scratch (objective partial sums)
    // MDRK: per step of a segment buffer the stage state u* and the stage-2 U traces (besides the step's state and
    // stage-1 U traces); scratch for steps outside the segment buffers; the stage adjoints (u*, (F2, G2), U2, and
    // the adjoint of u_new with the stage-2 jump term)
    double* d_segS = nullptr;               // [buffers][capacity_states] states u*
    double* d_segU2 = nullptr;              // [buffers][capacity_states] stage-2 U traces
    double *d_mus = nullptr, *d_mtU2 = nullptr;
    double *d_bus = nullptr, *d_bF2 = nullptr, *d_bU2 = nullptr, *d_lamacc = nullptr;
    double* d_final = nullptr;              // u(T) of the recorded run (one of the handle's state buffers)
    int rec_steps = 0, rec_ck = 0;          // recorded forward run: steps, checkpoint interval
    // the forward and reverse sweeps as CUDA graphs, keyed by (steps, interval); dropped whenever a buffer
    // they address is replaced
    cudaGraphExec_t g_fwd = nullptr, g_rev = nullptr;
    long long g_fwd_key = -1, g_rev_key = -1;
    bool const_uploaded = false;            // the adjoint translation unit's constant bank is set
};

inline void free_adjoint(AdjointBuffers& a) {
    if (a.g_fwd) cudaGraphExecDestroy(a.g_fwd);
    if (a.g_rev) cudaGraphExecDestroy(a.g_rev);
    dfree(a.d_lam[0]); dfree(a.d_lam[1]); dfree(a.d_bF); dfree(a.d_bU); dfree(a.d_bu); dfree(a.d_dts);
    dfree(a.d_dts_given); dfree(a.d_ckpt); dfree(a.d_seg); dfree(a.d_segU); dfree(a.d_segD); dfree(a.d_work);
    dfree(a.d_segS); dfree(a.d_segU2); dfree(a.d_mus); dfree(a.d_mtU2);
    dfree(a.d_bus); dfree(a.d_bF2); dfree(a.d_bU2); dfree(a.d_lamacc);
    for (cudaEvent_t ev : {a.ev_fork, a.ev_join, a.ev_join2, a.ev_ready[0], a.ev_ready[1], a.ev_free[0], a.ev_free[1]})
        if (ev) cudaEventDestroy(ev);
    if (a.s_rec) cudaStreamDestroy(a.s_rec);
    if (a.s_adj) cudaStreamDestroy(a.s_adj);
    a = AdjointBuffers{};
}

}  // namespace tlw

struct tlw_handle {
    tlw_opts opts{};
    int N = 0, n = 0, nn = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    tlw::Basis h_basis{};
    std::vector<double> nodes;
    tlw::Basis* d_basis = nullptr;
    tlw::StepState* d_step = nullptr;
    // mesh
    bool have_mesh = false;
    int64_t E = 0;
    double* d_inv_jac = nullptr;
    int *d_xl = nullptr, *d_xr = nullptr, *d_yl = nullptr, *d_yr = nullptr;
    int* d_nbr = nullptr;   // [4, E] element across each face when every face is a conforming interface
    // source terms (TreeMesh, FR volume integral): kind, node coordinates [2, i, j, e], MDRK stage 1's S2
    int source = 0;
    double* d_xnode = nullptr;
    double* d_S2 = nullptr;
    int nx = 0, ny = 0;
    int64_t nb = 0;
    int *d_b_elem = nullptr, *d_b_dir = nullptr, *d_bx = nullptr, *d_by = nullptr;
    int nbx = 0, nby = 0;
    double *d_levels = nullptr, *d_now = nullptr;
    bool have_bdata = false;
    // element-sized buffers
    double* d_state[2] = {nullptr, nullptr};
    int cur = 0;
    double* d_us = nullptr;
    double *d_in = nullptr, *d_in2 = nullptr, *d_out = nullptr;
    double *d_tU = nullptr, *d_tF = nullptr, *d_U2 = nullptr, *d_F2 = nullptr;
    // shock capturing
    bool sc = false;
    double *d_alpha = nullptr, *d_alpha_raw = nullptr, *d_tFn = nullptr;
    int *d_il = nullptr, *d_ir = nullptr;   // smoothing pairs: all interfaces, then the mortars' (small, large)
    int ni = 0, ni_if = 0;                  // pairs, of which interfaces
    // curvilinear shock capturing: subcell normals, calc_fn_low! normals, boundary-element flags, MUSCL geometry
    double *d_subn = nullptr, *d_subq = nullptr, *d_mgeom = nullptr;
    unsigned char* d_atb = nullptr;
    int reconstruction = 0;                 // 0 first-order subcells, 1 MUSCL (curvilinear meshes)
    double jac_first = 0.0;                 // inverse Jacobian of element 1 (TreeMesh interface cache)
    // Adaptive step control: per-element temporal errors, check scratch, tolerances of the trial in flight
    double* d_te = nullptr;
    double* d_check = nullptr;   // [blocks] partial sums, then the total
    unsigned* d_bad = nullptr;
    tlw::AdaptiveState* d_adapt = nullptr;   // the device controller (tlw_adaptive_begin / tlw_adaptive_run)
    bool te_request = false;
    double te_abstol = 0.0, te_reltol = 0.0;
    // per-element CFL slots of the state in d_state[cur] (plain LW step on a periodic conforming TreeMesh)
    unsigned long long* d_slots = nullptr;
    bool slots_valid = false;
    // compressible Navier-Stokes (TreeMesh, periodic, LW): BR1 gradients, viscous traces, viscous dt bound
    bool parabolic = false;
    double ns_mu = 0.0, ns_Pr = 0.72;
    double *d_gx = nullptr, *d_gy = nullptr, *d_tFv = nullptr;
    unsigned long long* d_visc = nullptr;
    // L2 mortars of a non-conforming TreeMesh: x-mortars [0, nmx), then y-mortars [nmx, nmx + nmy)
    int *d_ml = nullptr, *d_mu = nullptr, *d_mg = nullptr, *d_ms = nullptr;
    int nmx = 0, nmy = 0;
    // boundary condition per boundary (BC_*; null: all Dirichlet) and whether any is Dirichlet
    int* d_bkind = nullptr;
    bool bnd_dirichlet = true;
    // Navier-Stokes walls per boundary (WALL_*) and their data [3, l, B] (v1, v2, q or T)
    int* d_wkind = nullptr;
    double* d_wall = nullptr;
    // faces shared with other ranks' parts (domain decomposition): x-faces [0, nhx), y-faces [nhx, nh); local
    // element, face, position in the caller's order; send / receive buffers [halo][l][halo_values]; with shock
    // capturing also the raw alpha of each cut face's element [halo]
    int nh = 0, nhx = 0;
    int halo_values = 12;
    int dd_stage = 0;                       // split step: the MDRK stage in progress (0: stage 1, 1: stage 2)
    int *d_he = nullptr, *d_hf = nullptr, *d_hs = nullptr;
    double *d_send = nullptr, *d_recv = nullptr;
    double *d_asend = nullptr, *d_arecv = nullptr;
    // the caller's collectives run on s_comm; ev_lib / ev_comm hand the order over between it and the stream, so
    // that the exchange of the cut-face traces overlaps the part's x interfaces
    cudaStream_t s_comm = nullptr;
    cudaEvent_t ev_lib = nullptr, ev_comm = nullptr;
    // per element: the faces (0..3) through which it is the large element of a mortar, in mortar order
    // (bits 0-2 count, then 2 bits per mortar); for the positivity limiter's mortar pass
    int* d_mface = nullptr;
    // Zhang-Shu positivity limiter after each step (lim_count = 0: off)
    int lim_count = 0;
    double lim_thr[4] = {0.0, 0.0, 0.0, 0.0};
    int lim_var[4] = {0, 0, 0, 0};
    // conforming curvilinear mesh (instead of the TreeMesh arrays above; d_state etc. shared)
    bool curved = false;
    double* d_Ja = nullptr;                 // contravariant vectors [4, i, j, e]
    double* d_ijn = nullptr;                // inverse Jacobian per node [i, j, e]
    int *d_cp = nullptr, *d_cs = nullptr, *d_cf = nullptr;   // interfaces sorted by colour
    std::vector<int> color_off;             // colour c covers [color_off[c], color_off[c + 1])
    std::vector<signed char> face_used;     // [e * 4 + face]: 1 when an interface covers the face
    // boundary faces of the curvilinear mesh: xi faces [0, ncbx), then eta faces [ncbx, ncb); element, face,
    // slip-wall kind and the boundary's index in the caller's order (wall data)
    int ncb = 0, ncbx = 0;
    int *d_cbe = nullptr, *d_cbf = nullptr, *d_cbk = nullptr, *d_cbi = nullptr;
    // UnstructuredMesh2D (tlw_set_unstructured_mesh): the caller's outward normals [2, l, face, e] and the second
    // physical flux trace (G; d_tF holds F)
    bool unstructured = false;
    double* d_unorm = nullptr;
    double* d_tG = nullptr;
    // L2 mortars of the curvilinear mesh, sorted by colour: small elements (positions 1, 2), large element, and
    // small face | large face << 2 | large reversed << 4
    int ncm = 0;
    int *d_cms1 = nullptr, *d_cms2 = nullptr, *d_cml = nullptr, *d_cmc = nullptr;
    // shock capturing at the curvilinear mortars: smoothing pairs (small, large), lw_mortars.inverse_jacobian in
    // colour order [k][l], and the caller's mortar index of each colour-ordered mortar
    int *d_cmsl = nullptr, *d_cmsr = nullptr;
    int ncms = 0;
    double* d_cmj = nullptr;
    std::vector<int> mortar_order;
    std::vector<int> mortar_off;            // mortar colour c covers [mortar_off[c], mortar_off[c + 1])
    // host-buffer stepping (tlw_step_host): a pool of HOST_POOL state buffers taken round robin, two per call (the
    // upload target and the steps' other buffer), each with an event after its last use; the copy streams; per
    // call (ring of HOST_CALLS) the event after its download and its u_out; ev_prior on the compute stream at each
    // call (the next upload waits for the work enqueued before it); async_pending until another entry point has
    // ordered itself after the last download
    static constexpr int HOST_POOL = 5, HOST_CALLS = 4;
    double* host_pool[HOST_POOL] = {};
    cudaEvent_t ev_free[HOST_POOL] = {};
    cudaEvent_t ev_dl[HOST_CALLS] = {};
    const void* dl_out[HOST_CALLS] = {};
    cudaStream_t s_up = nullptr, s_down = nullptr;
    cudaEvent_t ev_up = nullptr, ev_computed = nullptr, ev_prior = nullptr;
    long long host_calls = 0;
    bool async_pending = false;
    // graphs: [start buffer] one step, two steps
    cudaGraphExec_t g_one[2] = {nullptr, nullptr};
    cudaGraphExec_t g_two[2] = {nullptr, nullptr};
    // discrete adjoint
    tlw::AdjointBuffers adj;
};
