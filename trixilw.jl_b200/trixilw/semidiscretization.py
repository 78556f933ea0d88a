"""Host-side mirror of the reference's semidiscretization API for the LW / MDRK rhs.

Mirrors (names, argument meaning and error behaviour):
  LW, MDRK                               src/basic_types.jl:4-6
  CFLBased, Adaptive                     src/basic_types.jl:10-16
  VolumeIntegralFR                       src/solvers/fr.jl:15-19
  SemidiscretizationHyperbolic(...)      src/semidiscretization/semidiscretization_hyperbolic.jl:58-84
  semidiscretize(semi, td, tspan)        src/semidiscretization/semidiscretization.jl:4-15
  rhs!(du_ode, u_ode, semi, t, tol)      src/semidiscretization/semidiscretization_hyperbolic.jl:4-20
  rhs_mdrk1!/rhs_mdrk2!                  src/semidiscretization/semidiscretization_hyperbolic.jl:22-56
  trixi2lw / lw_fourier_cfl              src/auxiliary/auxiliary.jl:14-23

Python cannot spell ``rhs!``; the functions are ``rhs``, ``rhs_mdrk1``, ``rhs_mdrk2``. dt is read from
``semi.cache["dt"][0]`` exactly as the reference reads ``cache.dt[1]``. Every evaluation runs in libtlw
on the GPU; a non-admissible state raises :class:`DomainError` as the reference's sqrt does.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import DomainError, check, lib
from .basis import gauss_lobatto
from .equations import CompressibleEulerEquations2D
from .mesh import RefinedTreeMesh, TreeMesh


class LW:
    """Lax-Wendroff time discretization."""
    code = _lib.TLW_LW

    def __repr__(self):
        return "Lax-Wendroff"


class MDRK:
    """Two-stage multi-derivative Runge-Kutta time discretization."""
    code = _lib.TLW_MDRK

    def __repr__(self):
        return "Multi-Derivative Runge-Kutta"


@dataclass
class CFLBased:
    cfl_number: float


class Adaptive:
    """Error-controlled stepping (src/solvers/adaptive.jl:47-172): the LW step's temporal error estimate,
    the PI controller with (beta1, beta2, beta3) = (0.6, -0.2, 0.0) (src/solvers/lwfr.jl:162) and rejection
    below a factor of 0.81. LW, hyperbolic; N >= 4 on a TreeMesh, N >= 3 on a curvilinear mesh.

    on_device: the controller runs on the device too (tlw_adaptive_begin / tlw_adaptive_run), so trials follow
    one another without a host round trip; chunk trials per call. Time-dependent boundary data and interval
    callbacks keep the controller on the host (they act between steps)."""

    def __init__(self, on_device: bool = False, chunk: int = 32):
        self.on_device = on_device
        self.chunk = chunk


@dataclass
class VolumeIntegralFR:
    time_discretization: object = field(default_factory=LW)


@dataclass
class FluxLaxFriedrichs:
    """flux_lax_friedrichs = FluxPlusDissipation(flux_central, DissipationLocalLaxFriedrichs(speed)).
    max_abs_speed: "naive" (Trixi max_abs_speed_naive, the default of the reference's Trixi era) or
    "davis" (Trixi max_abs_speed)."""
    max_abs_speed: str = "naive"
    code = _lib.TLW_FLUX_RUSANOV


@dataclass
class FluxHLL:
    """FluxHLL(min_max_speed_naive) with the LW 8-argument method (src/equations/compressible_euler_2d.jl:24-40)."""
    max_abs_speed: str = "naive"
    code = _lib.TLW_FLUX_HLL


flux_lax_friedrichs = FluxLaxFriedrichs()
flux_hll = FluxHLL()


@dataclass
class IndicatorHennemannGassner:
    """Trixi IndicatorHennemannGassner(equations, basis; alpha_max, alpha_min, alpha_smooth, variable);
    only variable = density_pressure is built."""
    alpha_max: float = 0.5
    alpha_min: float = 0.001
    alpha_smooth: bool = True
    variable: str = "density_pressure"

    def __post_init__(self):
        if self.variable != "density_pressure":
            raise NotImplementedError("only the density_pressure indicator variable is built")


class FirstOrderReconstruction:
    """FirstOrderReconstruction(): first-order subcells of the blended elements."""


class MUSCLReconstruction:
    """MUSCLReconstruction(): minmod-limited MUSCL subcells (curvilinear meshes)."""


class MUSCLHancockReconstruction:
    """MUSCLHancockReconstruction(): MUSCL subcells with the Hancock half step (curvilinear meshes)."""


@dataclass
class VolumeIntegralFRShockCapturing:
    """VolumeIntegralFRShockCapturing(indicator; volume_integralFR, volume_flux_fv, reconstruction)
    (src/solvers/fr.jl:59-86). Built: volume_flux_fv = flux_lax_friedrichs; reconstruction =
    FirstOrderReconstruction() (every mesh), MUSCLReconstruction() or MUSCLHancockReconstruction() (curvilinear
    meshes), given as an instance or by name."""
    indicator: IndicatorHennemannGassner = field(default_factory=IndicatorHennemannGassner)
    volume_integralFR: VolumeIntegralFR = field(default_factory=VolumeIntegralFR)
    volume_flux_fv: object = field(default_factory=FluxLaxFriedrichs)
    reconstruction: object = "FirstOrderReconstruction"

    def __post_init__(self):
        name = self.reconstruction if isinstance(self.reconstruction, str) else type(self.reconstruction).__name__
        codes = {"FirstOrderReconstruction": _lib.TLW_RECONSTRUCTION_FIRST_ORDER,
                 "MUSCLReconstruction": _lib.TLW_RECONSTRUCTION_MUSCL,
                 "MUSCLHancockReconstruction": _lib.TLW_RECONSTRUCTION_MUSCL_HANCOCK}
        if name not in codes:
            raise NotImplementedError(f"{name} subcells are not built")
        self.reconstruction_code = codes[name]

    @property
    def time_discretization(self):
        return self.volume_integralFR.time_discretization


@dataclass
class DGSEM:
    polydeg: int
    surface_flux: object = field(default_factory=FluxLaxFriedrichs)
    volume_integral: object = field(default_factory=VolumeIntegralFR)


def get_time_discretization(solver: DGSEM):
    return solver.volume_integral.time_discretization


class BoundaryConditionPeriodic:
    pass


boundary_condition_periodic = BoundaryConditionPeriodic()


class BoundaryConditionDirichlet:
    """Time-averaged Dirichlet condition (src/equations/equations.jl:6-37). ``boundary_value_function``
    is called as f(x, y, t, equations) on arrays and returns conservative states [..., 4]."""

    def __init__(self, boundary_value_function, time_independent=None):
        self.boundary_value_function = boundary_value_function
        if time_independent is None:
            time_independent = bool(getattr(boundary_value_function, "time_independent", False))
        self.time_independent = time_independent


class BoundaryConditionSlipWall:
    """TrixiLW's LW slip walls (src/equations/equations.jl:95-135): the exterior u, U and normal flux are
    the inner ones with the wall-normal momentum mirrored; no exterior data."""

    time_independent = True

    def __init__(self, code: int, name: str):
        self.code = code
        self.name = name

    def __repr__(self):
        return self.name


boundary_condition_slip_wall_vertical = BoundaryConditionSlipWall(_lib.TLW_BC_SLIP_WALL_VERTICAL,
                                                                  "boundary_condition_slip_wall_vertical")
boundary_condition_slip_wall_horizontal = BoundaryConditionSlipWall(_lib.TLW_BC_SLIP_WALL_HORIZONTAL,
                                                                    "boundary_condition_slip_wall_horizontal")

DIRECTIONS = ("x_neg", "x_pos", "y_neg", "y_pos")   # Trixi directions 1..4


def digest_boundary_conditions(bc):
    """One condition per direction (x_neg, x_pos, y_neg, y_pos), as Trixi's digest_boundary_conditions: a
    single condition for all, or a mapping / named tuple with those four keys."""
    if isinstance(bc, dict):
        missing = [d for d in DIRECTIONS if d not in bc]
        if missing:
            raise ValueError(f"boundary conditions missing for {missing}")
        return tuple(bc[d] for d in DIRECTIONS)
    if hasattr(bc, "_fields"):
        return digest_boundary_conditions(bc._asdict())
    return (bc,) * 4


# ---- walls of the parabolic part (Trixi BoundaryConditionNavierStokesWall) ------------------------------
class NoSlip:
    """NoSlip(boundary_value_function): f(x, y, t, equations) -> (v1, v2) of the wall."""

    def __init__(self, boundary_value_function):
        self.boundary_value_function = boundary_value_function


class Adiabatic:
    """Adiabatic(boundary_value_normal_flux_function): f(x, y, t, equations) -> normal heat flux q."""

    def __init__(self, boundary_value_normal_flux_function):
        self.boundary_value_normal_flux_function = boundary_value_normal_flux_function


class Isothermal:
    """Isothermal(boundary_value_function): f(x, y, t, equations) -> wall temperature T (= p / rho)."""

    def __init__(self, boundary_value_function):
        self.boundary_value_function = boundary_value_function


class BoundaryConditionNavierStokesWall:
    """BoundaryConditionNavierStokesWall(boundary_condition_velocity, boundary_condition_heat_flux) as TrixiLW
    imposes it with conservative gradient variables (src/equations/compressible_navier_stokes_2d.jl:81-124)."""

    def __init__(self, boundary_condition_velocity: NoSlip, boundary_condition_heat_flux):
        if not isinstance(boundary_condition_velocity, NoSlip):
            raise NotImplementedError("NoSlip velocity walls are built")
        if not isinstance(boundary_condition_heat_flux, (Adiabatic, Isothermal)):
            raise NotImplementedError("Adiabatic or Isothermal heat conditions are built")
        self.boundary_condition_velocity = boundary_condition_velocity
        self.boundary_condition_heat_flux = boundary_condition_heat_flux

    @property
    def code(self) -> int:
        return (_lib.TLW_WALL_NOSLIP_ADIABATIC if isinstance(self.boundary_condition_heat_flux, Adiabatic)
                else _lib.TLW_WALL_NOSLIP_ISOTHERMAL)

    def data(self, x, y, t, equations) -> np.ndarray:
        """[..., 3] = (v1, v2, q or T) at the points (x, y)."""
        v1, v2 = self.boundary_condition_velocity.boundary_value_function(x, y, t, equations)
        h = self.boundary_condition_heat_flux
        third = (h.boundary_value_normal_flux_function(x, y, t, equations) if isinstance(h, Adiabatic)
                 else h.boundary_value_function(x, y, t, equations))
        return np.stack(np.broadcast_arrays(v1, v2, third, x), axis=-1)[..., :3].astype(np.float64)


def lw_fourier_cfl(N: int) -> float:
    """LW Fourier CFL limits for N = 1..4 (src/auxiliary/auxiliary.jl:14). N >= 5 is not tabulated by
    the reference; callers must supply their own CFL there."""
    table = (1.000, 0.333, 0.170, 0.103)
    if not 1 <= N <= 4:
        raise KeyError(f"lw_fourier_cfl undefined for N={N} (the reference tabulates N = 1..4)")
    return table[N - 1]


def trixi2lw(cfl_number: float, solver: DGSEM) -> float:
    """src/auxiliary/auxiliary.jl:17-23: cfl * nnodes * lw_fourier_cfl(N)."""
    N = solver.polydeg
    return cfl_number * (N + 1) * lw_fourier_cfl(N)


class _Handle:
    def __init__(self, opts):
        L = lib()
        self.ptr = ctypes.c_void_p()
        rc = L.tlw_create(ctypes.byref(opts), ctypes.byref(self.ptr))
        if rc != 0:
            raise _lib.TlwError(rc, "tlw_create failed (CUDA device unavailable or invalid options)")

    def __del__(self):
        try:
            if self.ptr:
                lib().tlw_destroy(self.ptr)
                self.ptr = ctypes.c_void_p()
        except Exception:
            pass


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _i64p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


class SemidiscretizationHyperbolic:
    """SemidiscretizationHyperbolic(mesh, time_discretization, equations, initial_condition, solver;
    boundary_conditions=boundary_condition_periodic, source_terms=nothing). Builds the libtlw handle and uploads the
    mesh. source_terms: None or source_terms_convergence_test (TreeMesh, FR volume integral, LW or MDRK)."""

    def __init__(self, mesh: TreeMesh, time_discretization, equations: CompressibleEulerEquations2D,
                 initial_condition, solver: DGSEM, boundary_conditions=boundary_condition_periodic, device: int = 0,
                 source_terms=None):
        if source_terms is not None and getattr(source_terms, "kind", None) != 1:
            raise NotImplementedError("device source terms: source_terms_convergence_test")
        self.source_terms = source_terms
        self.curved = self._curved_form(mesh, solver.polydeg)
        self.mesh = mesh
        self.equations = equations
        self.initial_condition = initial_condition
        self.solver = solver
        self.time_discretization = time_discretization
        self.polydeg = solver.polydeg
        self.nnodes = solver.polydeg + 1
        self.boundary_conditions = boundary_conditions
        self._bcs = digest_boundary_conditions(boundary_conditions) if mesh.n_boundaries > 0 else ()
        for d, bc in zip(DIRECTIONS, self._bcs):
            if not isinstance(bc, (BoundaryConditionDirichlet, BoundaryConditionSlipWall)):
                raise ValueError(f"{d}: a non-periodic TreeMesh needs BoundaryConditionDirichlet or a slip wall")

        self.cache = {"dt": [math.nan]}
        sf = solver.surface_flux
        opts = _lib.TlwOpts()
        opts.polydeg = solver.polydeg
        opts.time_discretization = time_discretization.code
        opts.surface_flux = sf.code
        opts.max_speed = _lib.TLW_SPEED_DAVIS if getattr(sf, "max_abs_speed", "naive") == "davis" else _lib.TLW_SPEED_NAIVE
        opts.gamma = equations.gamma
        opts.device = device
        self.device = int(device)
        vi = solver.volume_integral
        if isinstance(vi, VolumeIntegralFRShockCapturing):
            opts.volume_integral = _lib.TLW_VOLUME_FR_SHOCK_CAPTURING
            opts.alpha_max = vi.indicator.alpha_max
            opts.alpha_min = vi.indicator.alpha_min
            opts.alpha_smooth = 1 if vi.indicator.alpha_smooth else 0
        else:
            opts.volume_integral = _lib.TLW_VOLUME_FR
        self._handle = _Handle(opts)
        self._upload_mesh()
        if isinstance(vi, VolumeIntegralFRShockCapturing):
            check(self.handle, lib().tlw_set_reconstruction(self.handle, vi.reconstruction_code))
        self._bdata_key = None
        self.node_coordinates = (self.curved.xy if self.curved is not None
                                 else mesh.node_coordinates(self.polydeg))
        if mesh.n_boundaries:
            self._bnd_xy = mesh.boundary_node_coordinates(self.polydeg)
            self._upload_boundary_kinds()
        self._upload_source_terms()

    def _upload_source_terms(self):
        """The source kind and the node coordinates in Trixi's [2, i, j, e] order."""
        if self.source_terms is None:
            return
        xy = self.node_coordinates
        self._xnode = np.ascontiguousarray(np.transpose(xy, (3, 2, 1, 0)), dtype=np.float64)
        check(self.handle, lib().tlw_set_source_terms(self.handle, int(self.source_terms.kind), _ptr(self._xnode)))

    @property
    def handle(self):
        return self._handle.ptr

    @staticmethod
    def _curved_form(mesh, polydeg: int):
        """The curvilinear form of a mesh (None for a TreeMesh)."""
        from .curved_mesh import CurvedMesh, RefinedStructuredMesh, StructuredMesh
        if isinstance(mesh, (StructuredMesh, RefinedStructuredMesh)):
            return mesh.curved(polydeg)
        if isinstance(mesh, CurvedMesh):
            return mesh
        if isinstance(mesh, (TreeMesh, RefinedTreeMesh)):
            return None
        raise NotImplementedError("TreeMesh{2}, StructuredMesh{2}, UnstructuredMesh2D and curvilinear meshes (with L2 "
                                  "mortars) are built")

    def remesh(self, mesh):
        """The re-upload after an AMR step (what the drop-in does behind the reference's resize! of the integrator
        and its caches, src/callbacks/amr.jl:2-208): the handle takes the new mesh's connectivity and element count,
        sizes its buffers anew and drops its captured graphs; the state is set again by the caller (Trixi projects
        it onto the new mesh on the host). Boundary conditions, the reconstruction and the positivity limiter carry
        over; the mortar inverse Jacobian of the curvilinear shock-capturing blend goes back to zeros."""
        curved = self._curved_form(mesh, self.polydeg)
        if (curved is None) != (self.curved is None):
            raise ValueError("remesh keeps the mesh family (TreeMesh or curvilinear)")
        if mesh.n_boundaries:
            bcs = digest_boundary_conditions(self.boundary_conditions)
        self.curved = curved
        self.mesh = mesh
        self._upload_mesh()
        vi = self.solver.volume_integral
        if isinstance(vi, VolumeIntegralFRShockCapturing):
            check(self.handle, lib().tlw_set_reconstruction(self.handle, vi.reconstruction_code))
        self.node_coordinates = self.curved.xy if self.curved is not None else mesh.node_coordinates(self.polydeg)
        self._bdata_key = None
        self._bcs = bcs if mesh.n_boundaries else ()
        if mesh.n_boundaries:
            self._bnd_xy = mesh.boundary_node_coordinates(self.polydeg)
            self._upload_boundary_kinds()
        self._upload_source_terms()

    def _upload_mesh(self):
        if self.curved is not None and getattr(self.curved, "unstructured", False):
            c = self.curved
            Ja = np.ascontiguousarray(c.Ja, dtype=np.float64)
            ij = np.ascontiguousarray(c.inverse_jacobian_nodes, dtype=np.float64)
            nd = np.ascontiguousarray(c.normal_directions, dtype=np.float64)      # (E, 4, n, 2) = [2, n, 4, E]
            arrs = (np.ascontiguousarray(c.element_ids.T, dtype=np.int64),         # [2, I] column-major
                    np.ascontiguousarray(c.element_side_ids.T, dtype=np.int64),
                    np.ascontiguousarray(c.start_index, dtype=np.int64),
                    np.ascontiguousarray(c.index_increment, dtype=np.int64))
            self._keep = (Ja, ij, nd) + arrs
            check(self.handle, lib().tlw_set_unstructured_mesh(self.handle, c.n_elements, _ptr(Ja), _ptr(ij), _ptr(nd),
                                                               c.n_interfaces, *[_ptr(a) for a in arrs]))
            return
        if self.curved is not None:
            c = self.curved
            Ja = np.ascontiguousarray(c.Ja, dtype=np.float64)                     # [E, j, i, 4] = [4, i, j, E]
            ij = np.ascontiguousarray(c.inverse_jacobian_nodes, dtype=np.float64)  # [E, j, i] = [i, j, E]
            arrs = (np.ascontiguousarray(c.primary_elements, dtype=np.int64),
                    np.ascontiguousarray(c.primary_faces, dtype=np.int32),
                    np.ascontiguousarray(c.secondary_elements, dtype=np.int64),
                    np.ascontiguousarray(c.secondary_faces, dtype=np.int32),
                    np.ascontiguousarray(c.secondary_reversed, dtype=np.int32))
            self._keep = (Ja, ij) + arrs
            i32p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            rc = lib().tlw_set_curved_mesh(self.handle, c.n_elements, dp(Ja), dp(ij), c.n_interfaces,
                                           _i64p(arrs[0]), i32p(arrs[1]), _i64p(arrs[2]), i32p(arrs[3]),
                                           i32p(arrs[4]))
            check(self.handle, rc)
            if getattr(c, "n_mortars", 0):
                mk = (np.ascontiguousarray(c.mortar_small1, dtype=np.int64),
                      np.ascontiguousarray(c.mortar_small2, dtype=np.int64),
                      np.ascontiguousarray(c.mortar_small_faces, dtype=np.int32),
                      np.ascontiguousarray(c.mortar_large, dtype=np.int64),
                      np.ascontiguousarray(c.mortar_large_faces, dtype=np.int32),
                      np.ascontiguousarray(c.mortar_large_reversed, dtype=np.int32))
                self._mkeep = mk
                check(self.handle, lib().tlw_set_curved_mortars(self.handle, c.n_mortars, *[_ptr(a) for a in mk]))
            return
        m = self.mesh
        ij = np.ascontiguousarray(m.inverse_jacobian, dtype=np.float64)
        nid = np.ascontiguousarray(m.interface_neighbor_ids, dtype=np.int64)
        nor = np.ascontiguousarray(m.interface_orientations, dtype=np.int64)
        bid = np.ascontiguousarray(m.boundary_neighbor_ids, dtype=np.int64)
        bor = np.ascontiguousarray(m.boundary_orientations, dtype=np.int64)
        bsi = np.ascontiguousarray(m.boundary_neighbor_sides, dtype=np.int64)
        bpd = np.ascontiguousarray(m.n_boundaries_per_direction, dtype=np.int64)
        self._keep = (ij, nid, nor, bid, bor, bsi, bpd)
        rc = lib().tlw_set_tree_mesh(self.handle, m.n_elements, ij.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     m.n_interfaces, _i64p(nid), _i64p(nor), m.n_boundaries, _i64p(bid), _i64p(bor),
                                     _i64p(bsi), _i64p(bpd))
        check(self.handle, rc)
        if getattr(m, "n_mortars", 0):
            mids = np.ascontiguousarray(m.mortar_neighbor_ids, dtype=np.int64)
            msd = np.ascontiguousarray(m.mortar_large_sides, dtype=np.int64)
            mor = np.ascontiguousarray(m.mortar_orientations, dtype=np.int64)
            self._mkeep = (mids, msd, mor)
            check(self.handle, lib().tlw_set_tree_mortars(self.handle, m.n_mortars, _i64p(mids), _i64p(msd), _i64p(mor)))

    # ---- array helpers -----------------------------------------------------------------------------
    def ndofs(self) -> int:
        return self.mesh.ndofs(self.polydeg)

    def wrap_array(self, u_ode: np.ndarray) -> np.ndarray:
        """View of the flat state as [element, j, i, v] (the reference's u[v, i, j, element])."""
        n = self.nnodes
        return u_ode.reshape(self.mesh.n_elements, n, n, 4)

    def compute_coefficients(self, t: float) -> np.ndarray:
        xy = self.node_coordinates
        u = self.initial_condition(xy[0], xy[1], t, self.equations)   # [i, j, E, 4]
        return np.ascontiguousarray(np.transpose(u, (2, 1, 0, 3))).reshape(-1)

    # ---- boundary data ------------------------------------------------------------------------------
    def _direction_ranges(self):
        last = np.cumsum(self.mesh.n_boundaries_per_direction)
        return [(int(b - c), int(b)) for b, c in zip(last, self.mesh.n_boundaries_per_direction)]

    def _upload_boundary_kinds(self):
        kinds = np.zeros(self.mesh.n_boundaries, dtype=np.int32)
        for (a, b), bc in zip(self._direction_ranges(), self._bcs):
            kinds[a:b] = bc.code if isinstance(bc, BoundaryConditionSlipWall) else _lib.TLW_BC_DIRICHLET
        self._kinds = kinds
        if self.curved is not None:
            c = self.curved
            self._cbkeep = (np.ascontiguousarray(c.boundary_elements, dtype=np.int64),
                            np.ascontiguousarray(c.boundary_faces, dtype=np.int32), kinds)
            check(self.handle, lib().tlw_set_curved_boundaries(self.handle, c.n_boundaries, _ptr(self._cbkeep[0]),
                                                               _ptr(self._cbkeep[1]), _ptr(kinds)))
            return
        check(self.handle, lib().tlw_set_boundary_kinds(self.handle, _ptr(kinds)))

    def time_dependent_boundaries(self) -> bool:
        return any(isinstance(bc, BoundaryConditionDirichlet) and not bc.time_independent for bc in self._bcs)

    def _prepare_boundaries(self, t: float, dt: float, scaling_factor: float):
        if self.mesh.n_boundaries == 0:
            return
        dirichlet = [(r, bc) for r, bc in zip(self._direction_ranges(), self._bcs)
                     if isinstance(bc, BoundaryConditionDirichlet) and r[1] > r[0]]
        if not dirichlet:
            return
        const = not self.time_dependent_boundaries()
        key = ("const", scaling_factor) if const else (t, dt, scaling_factor)
        if key == self._bdata_key or (const and self._bdata_key is not None):
            return
        nodes, _ = gauss_lobatto(self.polydeg)
        n = self.nnodes
        dts = scaling_factor * dt
        levels = np.zeros((self.mesh.n_boundaries, n, n, 4))  # [B, l, q, v] == [v, q, l, B] column-major
        now = np.zeros((self.mesh.n_boundaries, n, 4))
        for (a, b), bc in dirichlet:
            x, y = self._bnd_xy[0][:, a:b], self._bnd_xy[1][:, a:b]        # [l, B_d]
            for q in range(n):
                ts = t + 0.5 * dts * (nodes[q] + 1.0) if bc.time_independent is False else t
                levels[a:b, :, q, :] = np.transpose(bc.boundary_value_function(x, y, ts, self.equations), (1, 0, 2))
            now[a:b] = np.transpose(bc.boundary_value_function(x, y, t, self.equations), (1, 0, 2))
        levels = np.ascontiguousarray(levels)
        now = np.ascontiguousarray(now)
        check(self.handle, lib().tlw_set_boundary_data(self.handle, _ptr(levels), _ptr(now), _lib.TLW_WHERE_HOST))
        self._bdata_key = key

    # ---- rhs entry points ---------------------------------------------------------------------------
    def _rhs(self, stage: int, du_ode, u_ode, us_ode, t, dt):
        where = _lib.TLW_WHERE_HOST
        for a in (du_ode, u_ode) + ((us_ode,) if us_ode is not None else ()):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.size == 4 * self.ndofs()):
                raise ValueError("state arrays must be contiguous float64 vectors of length 4*ndofs")
        self._prepare_boundaries(t, dt, 0.5 if stage == _lib.TLW_STAGE_MDRK1 else 1.0)
        rc = lib().tlw_rhs(self.handle, stage, _ptr(du_ode), _ptr(u_ode),
                           _ptr(us_ode) if us_ode is not None else None, float(t), float(dt), where)
        check(self.handle, rc)

    def get_cache(self, item: int) -> np.ndarray:
        L = lib()
        size = L.tlw_cache_size(self.handle, item)
        if size < 0:
            raise ValueError("cache item not available")
        out = np.empty(size)
        check(self.handle, L.tlw_get_cache(self.handle, item, _ptr(out), _lib.TLW_WHERE_HOST))
        return out

    def set_mortar_inverse_jacobian(self, inverse_jacobian=None):
        """lw_mortars.inverse_jacobian [n_mortars, n] of a curvilinear mesh with mortars, read by the
        shock-capturing blend at the mortars (None: zeros, as the reference holds it before an AMR step)."""
        if inverse_jacobian is None:
            check(self.handle, lib().tlw_set_curved_mortar_jacobian(self.handle, None))
            return
        a = np.ascontiguousarray(inverse_jacobian, dtype=np.float64).reshape(-1)
        if a.size != getattr(self.mesh, "n_mortars", 0) * self.nnodes:
            raise ValueError("inverse_jacobian: n_mortars x nnodes values")
        check(self.handle, lib().tlw_set_curved_mortar_jacobian(self.handle, _ptr(a)))

    def max_dt(self, u_ode: np.ndarray, cfl: float) -> float:
        dt = ctypes.c_double()
        check(self.handle, lib().tlw_max_dt(self.handle, _ptr(u_ode), _lib.TLW_WHERE_HOST, float(cfl), ctypes.byref(dt)))
        return dt.value


def rhs(du_ode, u_ode, semi: SemidiscretizationHyperbolic, t, tolerances=None):
    """rhs!(du_ode, u_ode, semi, t, tolerances) with dt = semi.cache["dt"][0]."""
    semi._rhs(_lib.TLW_STAGE_LW, du_ode, u_ode, None, t, semi.cache["dt"][0])


def rhs_mdrk1(du_ode, u_ode, semi: SemidiscretizationHyperbolic, t, tolerances=None):
    """rhs_mdrk1!(du_ode, u_ode, semi, t): stage 1; keeps U2/F2 in the handle for stage 2."""
    semi._rhs(_lib.TLW_STAGE_MDRK1, du_ode, u_ode, None, t, semi.cache["dt"][0])


def rhs_mdrk2(du_ode, u_ode, semi: SemidiscretizationHyperbolic, t, us_ode, tolerances=None):
    """rhs_mdrk2!(du_ode, u_ode, semi, t): stage 2 at the stage state ``us_ode`` (the reference reads it
    from cache.element_cache.mdrk_cache.us, which perform_step! filled with uprev + dt*du)."""
    semi._rhs(_lib.TLW_STAGE_MDRK2, du_ode, u_ode, us_ode, t, semi.cache["dt"][0])


@dataclass
class LWUpdate:
    f: object
    u0_ode: np.ndarray
    du_ode: np.ndarray
    tspan: tuple
    p: SemidiscretizationHyperbolic


class SemidiscretizationHyperbolicParabolic(SemidiscretizationHyperbolic):
    """SemidiscretizationHyperbolicParabolic(mesh, [time_discretization,] (equations, equations_parabolic),
    initial_condition, solver; boundary_conditions=(hyperbolic, parabolic)): compressible Navier-Stokes on a
    conforming TreeMesh{2} (BR1 gradients of the conservative variables), LW. On a non-periodic mesh the
    parabolic conditions are BoundaryConditionNavierStokesWall, one per direction (x_neg, x_pos, y_neg, y_pos);
    their wall data are taken at t = 0 (the lid-driven cavity's walls do not change in time)."""

    def __init__(self, mesh, *args, device: int = 0, boundary_conditions=None, **kw):
        if len(args) == 4:   # the reference's form with the time discretization second
            _, equations, initial_condition, solver = args
        else:
            equations, initial_condition, solver = args
        eq, eq_par = equations
        bc_hyp, bc_par = boundary_conditions if boundary_conditions is not None else (
            boundary_condition_periodic, boundary_condition_periodic)
        self.equations_parabolic = eq_par
        self._bcs_par = digest_boundary_conditions(bc_par) if mesh.n_boundaries > 0 else ()
        for d, bc in zip(DIRECTIONS, self._bcs_par):
            if not isinstance(bc, BoundaryConditionNavierStokesWall):
                raise ValueError(f"{d}: the parabolic part needs a BoundaryConditionNavierStokesWall")
        super().__init__(mesh, get_time_discretization(solver), eq, initial_condition, solver, device=device,
                         boundary_conditions=bc_hyp, **kw)
        self.boundary_conditions_parabolic = bc_par
        self._upload_parabolic()

    def remesh(self, mesh):
        """As SemidiscretizationHyperbolic.remesh, with the parabolic terms and walls uploaded again."""
        if mesh.n_boundaries:
            self._bcs_par = digest_boundary_conditions(self.boundary_conditions_parabolic)
        super().remesh(mesh)
        self._upload_parabolic()

    def _upload_parabolic(self):
        eq_par = self.equations_parabolic
        check(self.handle, lib().tlw_set_parabolic(self.handle, eq_par.mu, eq_par.Pr))
        if self.mesh.n_boundaries == 0:
            return
        n = self.nnodes
        kinds = np.zeros(self.mesh.n_boundaries, dtype=np.int32)
        data = np.zeros((self.mesh.n_boundaries, n, 3))     # [B, l, 3] == [3, l, B] column-major
        xy = self.mesh.boundary_node_coordinates(self.polydeg)
        for (a, b), bc in zip(self._direction_ranges(), self._bcs_par):
            kinds[a:b] = bc.code
            if b > a:
                data[a:b] = np.transpose(bc.data(xy[0][:, a:b], xy[1][:, a:b], 0.0, self.equations), (1, 0, 2))
        self._wkeep = (kinds, np.ascontiguousarray(data))
        check(self.handle, lib().tlw_set_parabolic_walls(self.handle, _ptr(kinds), _ptr(self._wkeep[1])))



def semidiscretize(semi: SemidiscretizationHyperbolic, time_discretization, tspan) -> LWUpdate:
    u0 = semi.compute_coefficients(tspan[0])
    return LWUpdate(rhs, u0, np.empty_like(u0), (float(tspan[0]), float(tspan[1])), semi)


__all__ = [
    "LW", "MDRK", "CFLBased", "Adaptive", "VolumeIntegralFR", "VolumeIntegralFRShockCapturing",
    "IndicatorHennemannGassner", "DGSEM", "FluxLaxFriedrichs", "FluxHLL",
    "flux_lax_friedrichs", "flux_hll", "BoundaryConditionDirichlet", "boundary_condition_periodic",
    "boundary_condition_slip_wall_vertical", "boundary_condition_slip_wall_horizontal", "NoSlip", "Adiabatic",
    "Isothermal", "BoundaryConditionNavierStokesWall",
    "SemidiscretizationHyperbolic", "SemidiscretizationHyperbolicParabolic", "semidiscretize", "rhs", "rhs_mdrk1", "rhs_mdrk2", "lw_fourier_cfl",
    "trixi2lw", "get_time_discretization", "DomainError", "LWUpdate",
]
