/* tlw.h -- C ABI of libtlw, a B200 (sm_100a) implementation of TrixiLW's Lax-Wendroff / MDRK
 * flux-reconstruction right-hand side for the 2D compressible Euler equations on TreeMesh{2}.
 *
 * The entry points are what a Julia shim binds with `ccall` to replace the reference's
 *   rhs!(du_ode, u_ode, semi, t)         src/semidiscretization/semidiscretization_hyperbolic.jl:4-20
 *   rhs_mdrk1!/rhs_mdrk2!                src/semidiscretization/semidiscretization_hyperbolic.jl:22-56
 * and, below them, the mesh-level
 *   rhs!(du, u, t, dt, mesh::TreeMesh{2}, ..., ::LW, cache, tol)   src/solvers/dgsem_tree/dg_2d.jl:28-83
 *   rhs_mdrk1!/rhs_mdrk2!(..., mesh::TreeMesh{2}, ...)           src/solvers/dgsem_tree/multi_derivative_2d.jl:1-116
 * plus the CFL step loop of solve_lwfr (src/solvers/lwfr.jl:176-263, src/solvers/mdrk.jl:1-29) run on the
 * device. All arrays use the reference's Julia layout (column-major, leftmost index fastest):
 *   u, du: [v, i, j, element] with v = 1..4 (rho, rho v1, rho v2, rho e), i, j = 1..N+1.
 * Integer connectivity is accepted exactly as Trixi stores it (Int64, 1-based).
 *
 * Every function returns an int status (TLW_OK = 0). A handle is not thread-safe; it owns one CUDA
 * stream and all device memory it uses. Calls with TLW_WHERE_HOST pointers copy in and out and return
 * after the result is in host memory; calls with TLW_WHERE_DEVICE pointers are asynchronous on the
 * handle's stream. Kernels never trap: a square root of a negative number (the reference raises
 * DomainError there) sets a sticky status that the next synchronising call returns as
 * TLW_E_NONADMISSIBLE.
 */
#ifndef TLW_H
#define TLW_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TLW_ABI_VERSION 2

enum tlw_status {
    TLW_OK = 0,
    TLW_E_ARG = 1,             /* invalid argument / size / option */
    TLW_E_CUDA = 2,            /* CUDA runtime error (see tlw_last_error) */
    TLW_E_NONADMISSIBLE = 3,   /* negative pressure or density met in a square root (Julia DomainError) */
    TLW_E_STATE = 4,           /* call out of order (e.g. no mesh set) */
    TLW_E_UNSUPPORTED = 5      /* option combination not built */
};

enum tlw_time_discretization { TLW_LW = 0, TLW_MDRK = 1 };              /* src/basic_types.jl:4-6 */
enum tlw_surface_flux { TLW_FLUX_RUSANOV = 0, TLW_FLUX_HLL = 1 };        /* flux_lax_friedrichs / FluxHLL */
enum tlw_max_speed { TLW_SPEED_NAIVE = 0, TLW_SPEED_DAVIS = 1 };         /* Trixi max_abs_speed_naive / max_abs_speed */
enum tlw_where { TLW_WHERE_HOST = 0, TLW_WHERE_DEVICE = 1 };
enum tlw_stage { TLW_STAGE_LW = 0, TLW_STAGE_MDRK1 = 1, TLW_STAGE_MDRK2 = 2 };
enum tlw_cache_item {
    TLW_CACHE_U_TRACES = 0,    /* time-averaged U on the 4 faces, [v, l, face, element], face = -x,+x,-y,+y */
    TLW_CACHE_F_TRACES = 1,    /* normal time-averaged flux (F on x faces, G on y faces), same layout */
    TLW_CACHE_U2 = 2,          /* MDRK stage-1 U2 [v, i, j, element]   (MDRKElementCache.U2) */
    TLW_CACHE_F2 = 3,          /* MDRK stage-1 F2 [v, d, i, j, element] (MDRKElementCache.F2) */
    TLW_CACHE_ALPHA = 4,       /* shock capturing: blending factor per element (indicator.cache.alpha) */
    TLW_CACHE_FN_LOW = 5       /* shock capturing: first-order subcell flux next to each face, as the traces
                                  (element_cache.fn_low) */
};
enum tlw_volume_integral {
    TLW_VOLUME_FR = 0,                  /* VolumeIntegralFR(LW()/MDRK())                                  */
    TLW_VOLUME_FR_SHOCK_CAPTURING = 1   /* VolumeIntegralFRShockCapturing(IndicatorHennemannGassner(...;
                                           variable = density_pressure); volume_flux_fv = flux_lax_friedrichs,
                                           reconstruction = FirstOrderReconstruction()) (src/solvers/fr.jl:59-86) */
};

typedef struct tlw_opts {
    int32_t polydeg;               /* N, 1..7 */
    int32_t time_discretization;   /* TLW_LW | TLW_MDRK */
    int32_t surface_flux;          /* TLW_FLUX_RUSANOV | TLW_FLUX_HLL */
    int32_t max_speed;             /* TLW_SPEED_NAIVE (Trixi default of the reference's era) | TLW_SPEED_DAVIS */
    double gamma;                  /* CompressibleEulerEquations2D(gamma) */
    int32_t device;                /* CUDA device ordinal */
    int32_t volume_integral;       /* TLW_VOLUME_FR | TLW_VOLUME_FR_SHOCK_CAPTURING */
    double alpha_max;              /* indicator: alpha_max (Trixi default 0.5) */
    double alpha_min;              /* indicator: alpha_min (Trixi default 0.001) */
    int32_t alpha_smooth;          /* indicator: alpha_smooth (Trixi default true) */
    int32_t reserved[3];           /* zero */
} tlw_opts;

typedef struct tlw_handle tlw_handle;

int32_t tlw_abi_version(void);

/* Builds the solver state (basis, stream, device scalars). Replaces the cache construction
 * create_cache(mesh, equations, ::AbstractLWTimeDiscretization, dg, ...)
 * src/solvers/dgsem_tree/containers.jl:7-71 / src/semidiscretization/semidiscretization_hyperbolic.jl:58-84. */
int tlw_create(const tlw_opts* opts, tlw_handle** out);
int tlw_destroy(tlw_handle* h);

/* Uploads TreeMesh{2} connectivity (Trixi containers, 1-based Int64) and the per-element inverse
 * Jacobian (= 2 / element length). Call again after every AMR resize (src/callbacks/amr.jl:2-20).
 *   interface_neighbor_ids [2, n_interfaces]  (left, right)  Trixi interfaces.neighbor_ids
 *   interface_orientations [n_interfaces]     1 = x, 2 = y   Trixi interfaces.orientations
 *   boundary_* [n_boundaries]                 Trixi boundaries.neighbor_ids / orientations / neighbor_sides
 *   n_boundaries_per_direction [4]            boundaries grouped by direction 1..4 (dg_2d.jl:1385-1409)
 * Non-conforming meshes: add their mortars with tlw_set_tree_mortars. */
int tlw_set_tree_mesh(tlw_handle* h, int64_t n_elements, const double* inverse_jacobian, int64_t n_interfaces,
                      const int64_t* interface_neighbor_ids, const int64_t* interface_orientations,
                      int64_t n_boundaries, const int64_t* boundary_neighbor_ids,
                      const int64_t* boundary_orientations, const int64_t* boundary_neighbor_sides,
                      const int64_t* n_boundaries_per_direction);

/* Adaptive (error-controlled) stepping, src/solvers/adaptive.jl:47-172 (LW, hyperbolic; N >= 4 on a TreeMesh,
 * N >= 3 on a curvilinear mesh; FR or shock-capturing volume integral): one trial step u_trial = u + dt rhs(u)
 * from the current state at the given dt, with the LW volume kernels' temporal error estimate (abstol, reltol;
 * dg_2d.jl:1183-1265, dgsem_structured/dg_2d.jl:1595-1682 and 1983-2075). MDRK and the TreeMesh kernel of
 * depth 3 leave the reference's temporal_errors unset: TLW_E_UNSUPPORTED. *total_temporal_error = sqrt(sum_e errors / ndofs)
 * (load_temporal_errors!), *admissible = 0 when a square root of a negative number occurred (test_rhs!'s
 * DomainError) or a node of u_trial has rho <= 0 or p <= 0 (test_updated_solution). The state is not
 * changed until tlw_adaptive_accept(h, dt), which makes u_trial current and advances t by dt. Synchronous;
 * the controller (epsilon history, dt factor, rejection) stays with the caller, as in perform_step!. */
int tlw_adaptive_trial(tlw_handle* h, double dt, double abstol, double reltol, double* total_temporal_error,
                       int32_t* admissible);
int tlw_adaptive_accept(tlw_handle* h, double dt);

/* The same Adaptive stepping with the controller on the device (perform_step!'s epsilon history, dt_factor,
 * rejection and retry, set_dt! clamp; adaptive.jl:47-172), so that trials run back to back without a host
 * round trip. tlw_adaptive_begin starts a run from the current state and time to t_end with dt_initial and the
 * controller (beta1, beta2, beta3) (null: (0.6, -0.2, 0.0), lwfr.jl:162). tlw_adaptive_run enqueues n_trials
 * trials (each: trial step with the estimate, limiter, admissibility, the controller's decision, the accepted
 * state committed), then waits and reports the accepted steps so far (the handle's step count), the rejected
 * trials of accepted steps (the reference's nreject) and whether t_end is reached; trials after that are
 * no-ops. Synchronous; a mesh upload ends the run. The reference retries a rejected trial without a limit;
 * here, when repeated rejections bring the next dt to 1e-14 |t| or below, the run stops and tlw_adaptive_run
 * returns TLW_E_NONADMISSIBLE. */
int tlw_adaptive_begin(tlw_handle* h, double t_end, double dt_initial, const double* controller);
int tlw_adaptive_run(tlw_handle* h, int32_t n_trials, double abstol, double reltol, int64_t* steps,
                     int64_t* rejected, int32_t* finished);

/* Zhang-Shu positivity-preserving limiter, PositivityPreservingLimiterZhangShu(thresholds, variables) as a
 * stage limiter (src/callbacks/callbacks_stage/positivity_zhang_shu.jl:10-42, positivity_zhang_shu_dg2d.jl:8-176):
 * count (threshold, variable) pairs, applied in order; per pair the element pass and, on a TreeMesh with
 * mortars, the large-element mortar pass. count = 0 switches it off; at most TLW_LIMITER_MAX_PAIRS pairs.
 * Once set, tlw_step applies it after every step where solve_lwfr does (LW: twice, perform_step! and the
 * step loop, src/solvers/lwfr.jl:226,257; MDRK: once, the loop), tlw_adaptive_trial applies it to the trial
 * state before the admissibility check (adaptive.jl:131-132) and tlw_adaptive_accept once more (the loop).
 * Not with the adjoint entry points. tlw_apply_positivity_limiter applies it once to the current state
 * (solve_lwfr before its loop, lwfr.jl:251); asynchronous on the handle's stream. */
#define TLW_LIMIT_DENSITY 0           /* Trixi density(u, equations) */
#define TLW_LIMIT_PRESSURE 1          /* Trixi pressure(u, equations) */
#define TLW_LIMIT_DENSITY_PRESSURE 2  /* Trixi density_pressure(u, equations) */
#define TLW_LIMITER_MAX_PAIRS 4
int tlw_set_positivity_limiter(tlw_handle* h, int32_t count, const double* thresholds, const int32_t* variables);
int tlw_apply_positivity_limiter(tlw_handle* h);

/* Compressible Navier-Stokes (SemidiscretizationHyperbolicParabolic with CompressibleNavierStokesDiffusion2D,
 * conservative gradient variables, BR1) on the handle's conforming TreeMesh or curvilinear mesh, set after
 * tlw_set_tree_mesh / tlw_set_curved_mesh (which clear it): LW with the FR volume integral, N >= 3.
 * mu = dynamic viscosity, prandtl = Prandtl number; the handle's gamma. Replaces rhs! of
 * src/solvers/dgsem_tree/dg_2d_parabolic.jl:15-99 (TreeMesh kernels :725-1860, interface flux :1911-1949,
 * boundaries :1951-2084; P4estMesh kernels and surfaces of src/solvers/dgsem_p4est/dg_2d_parabolic.jl) and
 * compute_dt (src/solvers/lwfr.jl:192-210). A mesh with boundaries also needs tlw_set_parabolic_walls. */
int tlw_set_parabolic(tlw_handle* h, double mu, double prandtl);

/* Walls of the parabolic part, one per boundary (Trixi boundaries order), after tlw_set_parabolic:
 * BoundaryConditionNavierStokesWall(NoSlip(v), Adiabatic(q)) or (NoSlip(v), Isothermal(T))
 * (src/equations/compressible_navier_stokes_2d.jl:81-124). wall_data [3, l, boundary] = (v1, v2, q) or
 * (v1, v2, T) at the boundary's nodes, held until replaced (the reference evaluates the wall functions at the
 * step's t; re-send for walls that change in time). The gradient sees prim2cons(rho_inner, v, p_inner or
 * rho_inner T); the viscous boundary flux is the inner one with, for Adiabatic, the energy flux v . tau_n + q. */
#define TLW_WALL_NOSLIP_ADIABATIC 1
#define TLW_WALL_NOSLIP_ISOTHERMAL 2
int tlw_set_parabolic_walls(tlw_handle* h, const int32_t* kinds, const double* wall_data);

/* L2 mortars of a non-conforming TreeMesh{2} (after AMR), set after tlw_set_tree_mesh (which clears them):
 *   mortar_neighbor_ids [3, n_mortars]  (lower small, upper small, large element), 1-based  Trixi mortars.neighbor_ids
 *   mortar_large_sides  [n_mortars]     1: large element on the -side, 2: on the +side   Trixi mortars.large_sides
 *   mortar_orientations [n_mortars]     1 = x, 2 = y                                     Trixi mortars.orientations
 * The LW traces are carried over the mortar as prolong2mortars! / calc_mortar_flux! do
 * (src/solvers/dgsem_tree/dg_2d.jl:1456-1646), with Trixi's L2 mortar operators. Not with shock capturing. */
int tlw_set_tree_mortars(tlw_handle* h, int64_t n_mortars, const int64_t* mortar_neighbor_ids,
                         const int64_t* mortar_large_sides, const int64_t* mortar_orientations);

/* Conforming curvilinear mesh (StructuredMesh{2}, or P4estMesh{2} / UnstructuredMesh2D without mortars), in
 * place of a TreeMesh; LW with the FR volume integral, periodic or fully connected (no boundaries).
 * Replaces the volume and surface kernels of src/solvers/dgsem_structured/dg_2d.jl:1379-2105, 2107-2391
 * and src/solvers/dgsem_p4est/dg_2d.jl:8-191.
 *   contravariant_vectors [2, 2, n, n, element]  Trixi elements.contravariant_vectors (Ja^a_d at [d, a, ...])
 *   inverse_jacobian      [n, n, element]         Trixi elements.inverse_jacobian (positive)
 *   interface k: primary element / face, secondary element / face (1-based elements; faces 0: -xi (i = 1),
 *   1: +xi (i = n), 2: -eta (j = 1), 3: +eta (j = n)) and whether the secondary's face index runs backwards
 *   (P4est node_indices :i_backward). The normal is the primary's outward contravariant vector; a
 *   StructuredMesh interface takes the right / upper element as primary (its -xi / -eta face), which is the
 *   normal the StructuredMesh code uses (dgsem_structured/dg_2d.jl:2233-2267). Every element face must
 *   belong to exactly one interface. */
int tlw_set_curved_mesh(tlw_handle* h, int64_t n_elements, const double* contravariant_vectors,
                        const double* inverse_jacobian, int64_t n_interfaces, const int64_t* primary_elements,
                        const int32_t* primary_faces, const int64_t* secondary_elements,
                        const int32_t* secondary_faces, const int32_t* secondary_reversed);
/* UnstructuredMesh2D in Trixi's conventions (src/solvers/dgsem_unstructured_2d/dg_2d.jl:14-280, containers.jl), in
 * place of a TreeMesh: LW with the FR or the shock-capturing volume integral (first-order or MUSCL subcells, Rusanov),
 * conforming and without boundaries, which is what the reference runs on it (its rhs! is LW only, and its
 * calc_boundary_flux!, :421-450, calls the boundary condition with arguments no method accepts).
 *   contravariant_vectors [2, 2, n, n, element], inverse_jacobian [n, n, element]: as for tlw_set_curved_mesh
 *   normal_directions     [2, n, 4, element]  Trixi elements.normal_directions (outward, by side)
 *   interface k: element_ids [2, k] (primary, secondary; 1-based), element_side_ids [2, k] (sides 1: bottom (j = 1),
 *   2: right (i = n), 3: top (j = n), 4: left (i = 1)), start_index [k] and index_increment [k] (1 and 1, or n and
 *   -1) of the secondary's node index along the primary's.
 * The interface flux takes the primary's outward normal from normal_directions at its node, dots both sides'
 * physical time-averaged fluxes with it, and with shock capturing blends by compute_alp (the admissibility of
 * both sides' first-order subcell updates from the time-averaged U, J^{-1} of the primary face node). */
int tlw_set_unstructured_mesh(tlw_handle* h, int64_t n_elements, const double* contravariant_vectors,
                              const double* inverse_jacobian, const double* normal_directions, int64_t n_interfaces,
                              const int64_t* element_ids, const int64_t* element_side_ids, const int64_t* start_index,
                              const int64_t* index_increment);

/* Source terms (SemidiscretizationHyperbolic(...; source_terms), calc_source and its time-derivative stencils,
 * src/solvers/dgsem_tree/dg_2d.jl:89-175, used by every LW kernel and by mdrk_kernel_1! / _2!,
 * multi_derivative_2d.jl:321-400 and :484-550, and the structured kernels, dgsem_structured/dg_2d.jl:578-2058), after
 * the mesh upload (and again after a new mesh): kind 0 none,
 * 1 Trixi's source_terms_convergence_test for CompressibleEulerEquations2D (the source of
 * initial_condition_convergence_test's manufactured solution); node_coordinates [2, i, j, e] as Trixi's
 * cache.elements.node_coordinates. The source is evaluated at the step's t (tlw_step: the device time; tlw_rhs:
 * its t argument; MDRK stage 2 at t + dt/2 on the TreeMesh, at t on curvilinear meshes, as the reference's
 * structured kernels take it). TreeMesh or curvilinear mesh, FR volume integral, Euler, LW or MDRK; not with
 * Adaptive. */
int tlw_set_source_terms(tlw_handle* h, int32_t kind, const double* node_coordinates);

/* Domain decomposition (the reference's MPI path, src/solvers/dgsem_tree/dg_2d_parallel.jl:23-200, with the same
 * message per cut face node: the u face value, U trace and F.n trace, 3 nv doubles, dg_parallel.jl:12-13). A rank
 * uploads its part of the TreeMesh with tlw_set_tree_mesh (local elements, the interfaces between them, its
 * boundaries) and lists its cut faces here: elements 1-based local, faces 0: -x, 1: +x, 2: -y, 3: +y, in the
 * order of its send / receive buffers ([halo][l][tlw_dd_halo_values] doubles, tlw_dd_buffers; a neighbour's
 * send buffer segment lands in this rank's receive buffer at the same positions). LW or MDRK, conforming
 * TreeMesh, Euler, with the FR volume integral or shock capturing. A step is then
 *   tlw_dd_begin(h, cfl, fixed_dt, t_end)  this part's CFL maximum into *max_bits (a non-negative double's bits);
 *                                          with shock capturing also the raw alpha of each cut face's element
 *                                          into the alpha send buffer (tlw_dd_alpha_buffers, [halo] doubles)
 *   caller: allreduce(MAX) of *max_bits over the ranks (uint64); with shock capturing send / receive the
 *           alpha buffers (same segments, one double per cut face)
 *   tlw_dd_volume(h)                       (the alpha smoothing across the part's interfaces and cut faces) dt,
 *                                          the volume kernel, this part's cut-face traces into send, then the x
 *                                          faces inside the part (they overlap the exchange)
 *   caller: send / receive the halo buffers
 *   tlw_dd_finish(h)                       the x cut faces, y interfaces, boundaries and cut faces; the new state
 *                                          becomes current
 * all asynchronous. The caller enqueues its collectives on the comm stream (tlw_dd_comm_stream): each tlw_dd_*
 * call first waits for what the caller enqueued there, and the comm stream continues after tlw_dd_begin's work
 * and after tlw_dd_volume's packing, so the exchange runs beside the part's x interfaces (the reference overlaps
 * its MPI exchange with the local interface fluxes the same way, dg_2d_parallel.jl:209-320).
 * tlw_step / tlw_step_timed / tlw_rhs refuse a handle with cut faces. */
int tlw_set_halo(tlw_handle* h, int64_t n_halo, const int64_t* elements, const int32_t* faces);
int tlw_dd_buffers(tlw_handle* h, double** send, double** recv, unsigned long long** max_bits);
int tlw_dd_begin(tlw_handle* h, double cfl, double fixed_dt, double t_end);
int tlw_dd_volume(tlw_handle* h);
int tlw_dd_finish(tlw_handle* h);
/* Rounds of tlw_dd_volume / exchange / tlw_dd_finish per step: 1 for LW, 2 for MDRK (stage 1 produces u*, stage 2
 * the new state; each stage exchanges its own traces, the reference's two MPI exchanges of an MDRK step). */
int32_t tlw_dd_stages(tlw_handle* h);
/* Doubles per cut face node in the halo buffers: 12 (u, U, F.n), or 20 with shock capturing (and the element's
 * first-order subcell flux next to the face, fn_low, and its smoothed alpha, padded to 20), so that a cut face is blended as an
 * interface inside one part is (compute_alp, src/solvers/dgsem_tree/dg_2d.jl:1879-1901) and the decomposed run
 * equals the undecomposed one; the reference's calc_mpi_interface_flux! (dg_2d_parallel.jl:370-420) applies the
 * plain LW flux there. */
int32_t tlw_dd_halo_values(tlw_handle* h);
/* The alpha send / receive buffers of the shock-capturing split step ([halo] doubles, null without shock
 * capturing), exchanged between tlw_dd_begin and tlw_dd_volume. */
int tlw_dd_alpha_buffers(tlw_handle* h, double** send, double** recv);
/* The stream the caller's collectives of the split step go on (a cudaStream_t; created by tlw_set_halo). */
int tlw_dd_comm_stream(tlw_handle* h, void** stream);

/* L2 mortars of a curvilinear mesh after an AMR step (the reference's P4estMesh path: prolong2mortars! and
 * calc_mortar_flux!, src/solvers/dgsem_p4est/dg_2d.jl:395-603, with Trixi's mortar_fluxes_to_elements!), after
 * tlw_set_curved_mesh and before tlw_set_curved_boundaries. Mortar k: the small elements at positions 1 and 2
 * (1-based; position 1 at the start of the large face's forward index) on small_faces[k], the large element on
 * large_faces[k] (faces 0: -xi, 1: +xi, 2: -eta, 3: +eta), and whether the large face's index runs backwards
 * along the mortar (P4est node_indices :i_backward); the small faces run forward. As the reference, the large
 * side's normal flux is its instantaneous Trixi.flux(u, -n_large / 2), and the large face receives -2 times the
 * L2 projection of the small faces' fluxes. LW or MDRK, FR or shock-capturing volume integral, Euler; the
 * positivity limiter then runs the P4estMesh limit_mortars! (src/callbacks/callbacks_stage/positivity_zhang_shu_dg2d.jl:
 * 178-260) after its element pass. With shock capturing the blending factors are smoothed over the mortars too
 * and each small node's flux goes through get_blended_flux (dg_2d.jl:227-250, 589-593) with the J^{-1} of
 * tlw_set_curved_mortar_jacobian (zeros until it is called). */
int tlw_set_curved_mortars(tlw_handle* h, int64_t n_mortars, const int64_t* small1, const int64_t* small2,
                           const int32_t* small_faces, const int64_t* large, const int32_t* large_faces,
                           const int32_t* large_reversed);

/* lw_mortars.inverse_jacobian (dgsem_p4est/containers.jl:23-33), [n_mortars][n] in the order of
 * tlw_set_curved_mortars, as the reference holds it: zeros from create_cache, then after each AMR step what
 * load_inverse_jacobian!(lw_mortars.inverse_jacobian, mesh, eachmortar(dg, cache), dg, cache) loads
 * (callbacks/amr.jl:203; that loader reads the interface arrays, so mortar k gets the J^{-1} of interface k's
 * primary face nodes). Only the shock-capturing blend at the mortars reads it; null resets it to zeros. A
 * shim passes cache.lw_mortars.inverse_jacobian unchanged. */
int tlw_set_curved_mortar_jacobian(tlw_handle* h, const double* inverse_jacobian);

/* Subcell reconstruction of the blended elements under shock capturing on a curvilinear mesh (the reference's
 * VolumeIntegralFRShockCapturing(...; reconstruction), src/solvers/dgsem_tree/dg_2d.jl:251-365):
 * TLW_RECONSTRUCTION_FIRST_ORDER (FirstOrderReconstruction, the default) or TLW_RECONSTRUCTION_MUSCL
 * (MUSCLReconstruction: calcflux_muscl!, src/solvers/dgsem_structured/dg_2d.jl:176-311) or
 * TLW_RECONSTRUCTION_MUSCL_HANCOCK (MUSCLHancockReconstruction: calcflux_mh!, :313-538, the half step with the time
 * step fv_kernel! is given: dt, dt / 2 in MDRK stage 1); both first order on elements with a boundary face. Shock capturing on a curvilinear mesh follows the P4estMesh{2} path: LW or MDRK (both
 * stages blend with the indicator of u^n and take their subcells from u^n), Rusanov surface flux, the blended interface flux of get_blended_flux / zhang_shu_flux_fix (src/solvers/dgsem_p4est/
 * dg_2d.jl:199-250). TreeMesh shock capturing takes first-order subcells only. */
#define TLW_RECONSTRUCTION_FIRST_ORDER 0
#define TLW_RECONSTRUCTION_MUSCL 1
#define TLW_RECONSTRUCTION_MUSCL_HANCOCK 2
int tlw_set_reconstruction(tlw_handle* h, int32_t reconstruction);

/* Boundary faces of the curvilinear mesh (P4estMesh boundaries: element, face), after tlw_set_curved_mesh
 * (which clears them): elements 1-based, faces 0: -xi, 1: +xi, 2: -eta, 3: +eta (a face no interface covers),
 * kinds TLW_BC_SLIP_WALL_VERTICAL / _HORIZONTAL (the normal-direction slip walls of src/equations/equations.jl:
 * 137-169) or TLW_BC_DIRICHLET (the normal-direction time-averaged Dirichlet condition, :64-93, with exterior
 * data from tlw_set_boundary_data in this order; the MDRK stage 1 halves its time averages as the P4estMesh path
 * does), called as calc_boundary_flux! of src/solvers/dgsem_p4est/dg_2d.jl:285-393 does. The boundaries keep the
 * caller's order for tlw_set_boundary_data and tlw_set_parabolic_walls (Navier-Stokes: slip walls only). */
int tlw_set_curved_boundaries(tlw_handle* h, int64_t n_boundaries, const int64_t* elements, const int32_t* faces,
                              const int32_t* kinds);
/* Number of interface colours (launches per interface pass) of the curvilinear mesh; 0 for a TreeMesh. */
int32_t tlw_curved_colors(tlw_handle* h);

/* Boundary condition of each boundary (Trixi boundaries order) of a TreeMesh, after tlw_set_tree_mesh (which
 * resets all to Dirichlet): TLW_BC_DIRICHLET, the time-averaged Dirichlet condition below, or the LW slip walls
 * boundary_condition_slip_wall_vertical / _horizontal (src/equations/equations.jl:95-135), which mirror the
 * normal momentum of u, U and the normal flux trace and need no exterior data. */
#define TLW_BC_DIRICHLET 0
#define TLW_BC_SLIP_WALL_VERTICAL 1
#define TLW_BC_SLIP_WALL_HORIZONTAL 2
int tlw_set_boundary_kinds(tlw_handle* h, const int32_t* kinds);

/* Exterior states of the time-averaged Dirichlet boundary condition (src/equations/equations.jl:6-37):
 *   levels [v, q, l, boundary]: boundary_value_function(x_l, t + 0.5*dt_scaled*(x_q + 1)) at the N+1 GLL
 *                              time levels q (dt_scaled = scaling_factor * dt)
 *   now    [v, l, boundary]:    boundary_value_function(x_l, t)
 * Held until replaced; required before any rhs when the mesh has Dirichlet boundaries. */
int tlw_set_boundary_data(tlw_handle* h, const double* levels, const double* now, int32_t where);

/* One right-hand side evaluation: du = rhs(u) exactly as the reference's rhs!/rhs_mdrk1!/rhs_mdrk2!
 * (du already multiplied by -J^{-1}, ready for u_new = u + dt*du). For TLW_STAGE_MDRK2, `us` is the
 * stage state u* = u + dt*du1 (cache.element_cache.mdrk_cache.us); U2/F2 come from the preceding
 * TLW_STAGE_MDRK1 call on the same handle. Device arrays (where = TLW_WHERE_DEVICE) are used in place when they
 * are 32-byte aligned (one node's four doubles per access) and copied through the handle's buffers otherwise. */
int tlw_rhs(tlw_handle* h, int32_t stage, double* du, const double* u, const double* us, double t, double dt,
            int32_t where);

/* cfl * max_dt(u) (Trixi max_dt for TreeMesh{2}; src/solvers/lwfr.jl:176-190). Synchronous. */
int tlw_max_dt(tlw_handle* h, const double* u, int32_t where, double cfl, double* dt_out);

/* Device-resident time stepping (the LWIntegrator loop of solve_lwfr, CFLBased). */
int tlw_set_state(tlw_handle* h, const double* u, int32_t where, double t);
int tlw_get_state(tlw_handle* h, double* u, int32_t where, double* t_out);
/* Runs up to nsteps steps of perform_step!(..., ::CFLBased, ::LW|::MDRK): dt = cfl * max_dt(u) (or
 * fixed_dt when > 0), clamped to t_end, u <- u + dt * rhs(u). dt never leaves the device. The steps are
 * replayed from a captured CUDA graph when use_graph != 0. Asynchronous. */
int tlw_step(tlw_handle* h, int32_t nsteps, double cfl, double fixed_dt, double t_end, int32_t use_graph);
/* Host-buffer stepping: uploads the state u_in (host, [v, i, j, element]) at time t, runs nsteps steps as
 * tlw_step does (without graphs) and downloads the result into u_out (host). Asynchronous: it returns after
 * enqueueing, and the caller keeps u_in and u_out untouched until tlw_synchronize (or until a later call that
 * waits on them returns). Consecutive calls overlap: the upload of the next call and the download of the
 * previous one run on copy streams of their own beside the steps, so a stream of independent states (an
 * ensemble, or requests served one after another) moves through the GPU at the host link's bandwidth. With
 * pinned (page-locked) host buffers the copies run asynchronously; pageable ones make the copies wait. A u_in
 * equal to the u_out of an earlier call (the state round-tripping through the host) is read after that download:
 * each upload waits for the downloads up to three calls back, and for the last two calls' where u_in is their u_out. The
 * handle's current state afterwards is the last call's result. (No counterpart in the reference, whose
 * solution vectors stay in host memory; this is the host-side path of the drop-in at full link speed.) */
int tlw_step_host(tlw_handle* h, const double* u_in, double* u_out, double t, int32_t nsteps, double cfl,
                  double fixed_dt, double t_end);
/* As tlw_step without graphs, with CUDA events between the phases of each step. Synchronous. On return
 * phase_ms[0..4] hold the summed device time of: CFL reduction (max speed + dt), volume kernel(s),
 * x interfaces + x boundaries, y interfaces + y boundaries, and the whole steps. (Measurement entry: no
 * counterpart in the reference.) */
int tlw_step_timed(tlw_handle* h, int32_t nsteps, double cfl, double fixed_dt, double t_end, double* phase_ms);
/* Measures the device's dense FP64 FMA throughput (TFLOP/s) with a bounded register-resident loop.
 * Roofline calibration only (no counterpart in the reference). */
int tlw_probe_fp64_tflops(int32_t device, double* tflops);
/* y[k] = the kernels' reciprocal of x[k] (the 1/rho of every Euler flux) for n host values, on the given
 * device; for accuracy tests of that routine against IEEE division (no counterpart in the reference). */
int tlw_probe_reciprocal(int32_t device, const double* x, double* y, int64_t n);
/* Synchronous: current time, last dt and number of accepted steps. */
int tlw_get_time(tlw_handle* h, double* t, double* dt_last, int64_t* steps);

/* Element/interface caches of the last rhs (layouts in tlw_cache_item). Synchronous. U2 and F2 are those of the
 * last tlw_rhs MDRK stage 1: the device step loop passes only u_t between its stages (a TreeMesh without shock
 * capturing or source terms) and rebuilds U2 and F2 in stage 2. */
int tlw_get_cache(tlw_handle* h, int32_t item, double* out, int32_t where);
int64_t tlw_cache_size(tlw_handle* h, int32_t item);

/* Waits for the handle's stream; returns TLW_E_NONADMISSIBLE if a kernel flagged a bad state. */
int tlw_synchronize(tlw_handle* h);
/* The handle's cudaStream_t (for event timing / interop). */
int tlw_get_stream(tlw_handle* h, void** stream);
/* Device address of the current state (valid until the next tlw_step / tlw_set_tree_mesh). */
int tlw_state_pointer(tlw_handle* h, double** dptr);
const char* tlw_last_error(tlw_handle* h);

/* LW rhs for callers that must not allocate device memory (no counterpart in the reference: the
 * reference's Julia rhs! allocates nothing per call because its caches are built once; this entry point
 * gives a caller whose device memory is owned by another pool, or who cannot accept cudaMalloc's implicit
 * synchronisation, the same rhs without a handle). Periodic TreeMesh{2} only (no boundaries, no mortars).
 * All pointers are device pointers; u and du 32-byte aligned (TLW_E_ARG otherwise): u, du [v, i, j, element]; inverse_jacobian
 * [element]; x_left/x_right, y_left/y_right the 0-based element ids of the x- and y-oriented interfaces.
 * The face-trace scratch is a static device array of TLW_NOALLOC_SCRATCH_BYTES: meshes with
 * n_elements * 2 * 4 * (N+1) * 4 * 8 bytes of traces beyond it are rejected with TLW_E_ARG. Calls on a
 * device share that array and the static dt and status words beside it, so calls that overlap on the GPU
 * race. The first call on a device sets the device up. Runs on `stream`
 * (a cudaStream_t, 0 = default), waits for that stream and returns after the result is in du: TLW_OK,
 * TLW_E_NONADMISSIBLE (DomainError), TLW_E_ARG or TLW_E_CUDA. */
#define TLW_NOALLOC_SCRATCH_BYTES (32u << 20)
int tlw_rhs_lw_noalloc(int32_t polydeg, double gamma, int32_t surface_flux, int32_t max_speed, int64_t n_elements,
                       const double* inverse_jacobian, int32_t n_x_interfaces, const int32_t* x_left,
                       const int32_t* x_right, int32_t n_y_interfaces, const int32_t* y_left,
                       const int32_t* y_right, const double* u, double* du, double dt, void* stream);

/* ---- Differentiable form: discrete adjoint of the LW step (periodic TreeMesh{2}, N = 3..5, LW, FR volume
 * integral, Rusanov surface flux with either speed estimate) -----------------------------------------------
 * No counterpart in the reference. What is differentiated is the reference's forward map of one step at a
 * fixed dt, u_new = u + dt * rhs(u) (src/solvers/dgsem_tree/dg_2d.jl:28-83, src/solvers/lwfr.jl:212-230);
 * the dt sequence of a run is recorded on the forward sweep and held fixed on the reverse sweep. */
/* lam_out = (d u_new / d u)^T lam_in for one step from u at the given dt. Synchronous. */
int tlw_adjoint_step(tlw_handle* h, double* lam_out, const double* lam_in, const double* u, double dt, int32_t where);
/* Forward sweep of nsteps CFL steps from u0 (dt = cfl * max_dt(u) each step) that records the dt sequence
 * and checkpoints the state every checkpoint_every steps; u(T) into uT_out (optional). Uses the handle's
 * state buffers (the state set by tlw_set_state is overwritten). Synchronous. */
int tlw_forward_record(tlw_handle* h, const double* u0, int32_t nsteps, double cfl, int32_t checkpoint_every,
                       double* uT_out, int32_t where);
/* Reverse sweep of the recorded run: grad_out = (d u(T) / d u0)^T lam_T, the states between checkpoints
 * recomputed segment by segment. phase_ms (optional, 2 doubles): device time of the recomputation and of
 * the adjoint steps (adds synchronisations). Synchronous. */
int tlw_adjoint_sweep(tlw_handle* h, const double* lam_T, double* grad_out, int32_t where, double* phase_ms);
/* Both sweeps for the objective
 * J = 1/2 sum_nodes (rho(T) - rho_target)^2 (rho_target [i, j, element], one value per node), and the
 * gradient dJ/du0 [v, i, j, element]. uT_out (optional) receives u(T). phase_ms (optional, 3 doubles): device
 * time of the forward sweep (with the objective), of the recomputation and of the adjoint steps. */
int tlw_adjoint_solve(tlw_handle* h, const double* u0, int32_t nsteps, double cfl, int32_t checkpoint_every,
                      const double* rho_target, double* grad_out, double* J_out, double* uT_out, int32_t where,
                      double* phase_ms);
/* The dt of the first n steps of the recorded forward sweep (host array). */
int tlw_adjoint_dt_sequence(tlw_handle* h, double* dts, int32_t n);
/* Forward solve of nsteps LW steps from u0 at the given dt sequence (host array), u(T) into uT_out. Synchronous. */
int tlw_solve_dts(tlw_handle* h, const double* u0, int32_t nsteps, const double* dts, double* uT_out, int32_t where);

/* ---- Batched form: many independent periodic TreeMesh{2} LW runs (N = 3, 4, 5, uneven sizes) ----------
 * No counterpart in the reference, which runs one semidiscretization per `solve_lwfr` call
 * (src/solvers/lwfr.jl:233-270); each instance here advances exactly as that loop would advance it alone:
 * its own CFL dt (compute_dt, src/solvers/lwfr.jl:176-190), its own final time (set_dt! clamp and
 * isfinished, src/solvers/lwfr.jl:76-90 and 146-148), its own step count. A step of the batch is one graph replay.
 * Order: tlw_batch_create, tlw_batch_add_tree_mesh per instance, tlw_batch_finalize, tlw_batch_set_state per
 * instance, optionally tlw_batch_autotune, then tlw_batch_step / tlw_batch_get_state. Opts: LW, FR volume
 * integral, any surface flux / speed; opts->polydeg is ignored (each instance has its own). */
typedef struct tlw_batch tlw_batch;
int tlw_batch_create(const tlw_opts* opts, tlw_batch** out);
int tlw_batch_destroy(tlw_batch* b);
/* Adds one instance: its degree (3..5), its periodic mesh (arrays as in tlw_set_tree_mesh, without
 * boundaries). *index_out receives the instance id (0, 1, ... in call order). */
int tlw_batch_add_tree_mesh(tlw_batch* b, int32_t polydeg, int64_t n_elements, const double* inverse_jacobian,
                            int64_t n_interfaces, const int64_t* interface_neighbor_ids,
                            const int64_t* interface_orientations, int32_t* index_out);
/* Groups the instances by degree and allocates the concatenated device arrays. */
int tlw_batch_finalize(tlw_batch* b);
/* State [v, i, j, element] of one instance, its start time, CFL number and final time; resets its step count.
 * Synchronous. */
int tlw_batch_set_state(tlw_batch* b, int32_t instance, const double* u, int32_t where, double t, double cfl,
                        double t_end);
/* Synchronous: state, time and accepted steps of one instance; TLW_E_NONADMISSIBLE if any kernel flagged a
 * bad state since the last check. */
int tlw_batch_get_state(tlw_batch* b, int32_t instance, double* u, int32_t where, double* t_out,
                        int64_t* steps_out);
/* Enqueues nsteps batch steps (asynchronous). Instances past their final time take dt = 0 steps. */
int tlw_batch_step(tlw_batch* b, int32_t nsteps, int32_t use_graph);
int tlw_batch_synchronize(tlw_batch* b);
int tlw_batch_get_stream(tlw_batch* b, void** stream);
/* Times the launch variants on this batch (elements per CTA of the volume kernel per degree group, the
 * element-centric surface pass or the x / y interface sweeps and their CTA size, degree groups serial or
 * concurrent) and keeps the fastest; every variant gives the same bits. choices_out (optional, 2 * groups + 1
 * ints): per group (volume variant, interface CTA size or 0 for the surface pass), then the concurrency flag.
 * The current state is not changed. */
int tlw_batch_autotune(tlw_batch* b, int32_t trials, int32_t* choices_out);
int32_t tlw_batch_num_groups(tlw_batch* b);
const char* tlw_batch_last_error(tlw_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* TLW_H */
