"""Definitions of the small golden cases (inputs + oracle outputs). tests/golden/make_golden.py writes
them to tests/golden/*.npz; tests check the oracle (CPU) and the CUDA library (GPU) against them."""
import numpy as np

CASES = {
    # name: (time discretization, N, level, initial condition, domain, periodic)
    "lw_vortex_N3_L2": ("lw", 3, 2, "vortex", (-10.0, 10.0), True),
    "lw_vortex_N4_L2": ("lw", 4, 2, "vortex", (-10.0, 10.0), True),
    "lw_vortex_N5_L2": ("lw", 5, 2, "vortex", (-10.0, 10.0), True),
    "mdrk_vortex_N4_L2": ("mdrk", 4, 2, "vortex", (-10.0, 10.0), True),
    "lw_riemann_N4_L2": ("lw", 4, 2, "riemann", (0.0, 1.0), False),
    # shock capturing (HG indicator alpha_max = 0.5, first-order subcells)
    "sc_lw_riemann_N4_L3": ("lw", 4, 3, "riemann", (0.0, 1.0), False),
    "sc_mdrk_riemann_N3_L3": ("mdrk", 3, 3, "riemann", (0.0, 1.0), False),
}

SHOCK_CAPTURING = {"sc_lw_riemann_N4_L3", "sc_mdrk_riemann_N3_L3"}


def setup(name, tl):
    td, N, level, icname, (lo, hi), periodic = CASES[name]
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((lo, lo), (hi, hi), level, periodicity=periodic)
    ic = tl.IsentropicVortex(5.0, center=(0.5, 0.3)) if icname == "vortex" else tl.FourQuadrantRiemann()
    xy = mesh.node_coordinates(N)
    u = np.ascontiguousarray(np.transpose(ic(xy[0], xy[1], 0.0, eq), (2, 1, 0, 3))).reshape(-1)
    return td, N, eq, mesh, ic, u


def boundary_data(mesh, N, ic, eq, t=0.0):
    """[v, q, l, B] levels and [v, l, B] now for a time-independent boundary function."""
    if mesh.n_boundaries == 0:
        return None, None
    from trixilw.semidiscretization import BoundaryConditionDirichlet  # noqa: F401  (layout documented there)
    bxy = mesh.boundary_node_coordinates(N)
    n = N + 1
    now = np.ascontiguousarray(np.transpose(ic(bxy[0], bxy[1], t, eq), (1, 0, 2)))     # [B, l, v]
    levels = np.ascontiguousarray(np.repeat(now[:, :, None, :], n, axis=2))           # [B, l, q, v]
    return levels, now


def run_case(name, oracle_mod, tl):
    td, N, eq, mesh, ic, u = setup(name, tl)
    o = oracle_mod.Oracle(mesh, N)
    if name in SHOCK_CAPTURING:
        o.set_shock_capturing(True, 0.5, 0.001, True)
    levels, now = boundary_data(mesh, N, ic, eq)
    if levels is not None:
        o.set_boundary_data(levels, now)
    cfl = 0.98 * (N + 1) * 0.103
    dt = o.max_dt(u, cfl)
    out = {"u": u, "dt": np.array([dt])}
    if td == "lw":
        out["du"] = o.rhs(u, 0.0, dt)
        out["U"] = o.get(0)
        out["F"] = o.get(1)
        if name in SHOCK_CAPTURING:
            out["alpha"] = o.get(6)
            out["fn_low"] = o.get(7)
    else:
        du1 = o.rhs(u, 0.0, dt, kind=1)
        out["du1"] = du1
        out["U1"] = o.get(0)
        out["F1"] = o.get(1)
        out["U2"] = o.get(2)
        out["F2"] = o.get(3)
        us = u + dt * du1
        out["du2"] = o.rhs(u, 0.0, dt, kind=2, us=us)
        out["U"] = o.get(0)
        out["F"] = o.get(1)
        if name in SHOCK_CAPTURING:
            out["alpha"] = o.get(6)
            out["fn_low"] = o.get(7)
    return out
