"""Compressible Navier-Stokes on a curvilinear mesh with walls: the lid-driven cavity on [0, 1]^2 warped by
x += 0.05 sin(pi x) sin(pi y) (same for y), as a P4estMesh{2} runs it (the reference has no StructuredMesh
parabolic path): slip walls for the advective part (normal-direction form, src/equations/equations.jl:137-169)
and no-slip adiabatic walls with the lid at v1 = 1 for the parabolic part
(src/solvers/dgsem_p4est/dg_2d_parabolic.jl). CPU: the oracle's rest state, conservation, invariance under
P4est-like element rotations and the viscous decay rate of a shear wave on a warped mesh; GPU: libtlw against
the oracle (1e-12 relative L2 per variable), and the 64 x 64, N = 4 cavity for 2000 steps."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1
GAMMA = 1.4
MA = 0.1
P0 = 1.0 / (MA ** 2 * GAMMA)


def cavity_warp(xi, eta):
    """[-1, 1]^2 -> [0, 1]^2, then x += 0.05 sin(pi x) sin(pi y), y likewise (the boundary stays straight)."""
    X = 0.5 * (xi + 1.0)
    Y = 0.5 * (eta + 1.0)
    s = 0.05 * np.sin(np.pi * X) * np.sin(np.pi * Y)
    return X + s, Y + s


def periodic_warp(xi, eta):
    """[-1, 1]^2 -> [-10, 10]^2 with the interior warped by 5 % of the side, periodic-compatible."""
    X = 10.0 * xi
    Y = 10.0 * eta
    s = np.sin(np.pi * (X + 10.0) / 10.0) * np.sin(np.pi * (Y + 10.0) / 10.0)
    return X + 1.0 * s, Y + 1.0 * s


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def cavity_mesh(tl, cells=6):
    return tl.StructuredMesh((cells, cells), cavity_warp, periodicity=False)


def flat(U):
    return np.ascontiguousarray(np.transpose(U, (2, 1, 0, 3))).reshape(-1)


def rest(cm, N):
    return np.tile(np.array([1.0, 0.0, 0.0, P0 / (GAMMA - 1.0)]), cm.n_elements * (N + 1) ** 2)


def stirred(tl, cm, amp=0.1):
    """The cavity state with a smooth density bump, a rotating velocity field and a pressure bump."""
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    x, y = cm.xy
    rho = 1.0 + 0.2 * np.exp(-20 * ((x - 0.6) ** 2 + (y - 0.45) ** 2))
    v1 = amp * np.sin(np.pi * x) * np.cos(np.pi * (y - 0.5))
    v2 = -amp * np.cos(np.pi * (x - 0.5)) * np.sin(np.pi * y) + 0.3 * amp
    p = P0 * (1.0 + 0.02 * np.exp(-15 * ((x - 0.35) ** 2 + (y - 0.6) ** 2)))
    return flat(eq.prim2cons(rho, v1, v2, p))


SLIP = (1, 1, 2, 2)


def slip_kinds(cm):
    return np.repeat(np.asarray(SLIP, dtype=np.int32), cm.n_boundaries_per_direction)


def walls(cm, N, lid=1.0):
    data = np.zeros((cm.n_boundaries, N + 1, 3))
    data[cm.n_boundaries_per_direction[:3].sum():, :, 0] = lid
    return np.full(cm.n_boundaries, 1, dtype=np.int32), data


def oracle_for(oracle_mod, cm, N, mu=None, lid=1.0):
    o = oracle_mod.Oracle(cm, N)
    if cm.n_boundaries:
        o.set_curved_boundaries(cm.boundary_elements, cm.boundary_faces, slip_kinds(cm))
    if mu is not None:
        o.set_parabolic(mu)
        if cm.n_boundaries:
            o.set_walls(*walls(cm, N, lid))
    return o


def quad(cm, N, du):
    from trixilw.basis import gauss_lobatto
    _, w = gauss_lobatto(N)
    return np.einsum("ejiv,eji,j,i->v", du.reshape(-1, N + 1, N + 1, 4), cm.jacobian_nodes(), w, w)


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_slip_walls_rest_and_conservation(oracle_mod, tl, N):
    cm = cavity_mesh(tl).curved(N)
    o = oracle_for(oracle_mod, cm, N)
    u0 = rest(cm, N)
    assert np.abs(o.rhs(u0, 0.0, 1e-4)).max() < 1e-9 * u0.max()
    u = stirred(tl, cm)
    du = o.rhs(u, 0.0, o.max_dt(u, 0.3))
    tot = quad(cm, N, du)
    assert abs(tot[0]) < 1e-11 and abs(tot[3]) < 1e-9 * P0


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_navier_stokes_walls(oracle_mod, tl, N):
    cm = cavity_mesh(tl).curved(N)
    o = oracle_for(oracle_mod, cm, N, mu=0.01, lid=0.0)
    u0 = rest(cm, N)
    assert np.abs(o.rhs(u0, 0.0, 1e-4)).max() < 1e-9 * u0.max()
    o.set_walls(*walls(cm, N, 1.0))
    du = o.rhs(u0, 0.0, 1e-4)
    tot = quad(cm, N, du)
    assert abs(tot[0]) < 1e-11 and tot[1] > 0.0


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_navier_stokes_invariant_under_element_rotations(oracle_mod, tl, N):
    cm = cavity_mesh(tl, 5).curved(N)
    turns = np.random.default_rng(10 + N).integers(0, 4, cm.n_elements)
    rm = tl.rotate_elements(cm, turns)
    u = stirred(tl, cm)
    o, o2 = oracle_for(oracle_mod, cm, N, mu=0.01), oracle_for(oracle_mod, rm, N, mu=0.01)
    dt = o.max_dt(u, 0.3)
    du = o.rhs(u, 0.0, dt)
    du2 = o2.rhs(tl.rotate_state(u, N, turns), 0.0, dt)
    assert np.all(rel_l2(du2, tl.rotate_state(du, N, turns)) < 1e-11)


def test_oracle_curved_shear_wave_decays_at_the_viscous_rate(oracle_mod, tl):
    """A small shear wave on a warped periodic mesh decays as exp(-mu/rho k^2 t) (linearised Navier-Stokes)."""
    N, mu, T = 4, 0.2, 2.0
    cm = tl.StructuredMesh((8, 8), periodic_warp).curved(N)
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    k = 2 * np.pi / 20.0
    x, y = cm.xy
    one = np.ones_like(x)
    u = flat(eq.prim2cons(one, 0 * one, 1e-3 * np.sin(k * (x + 10.0)), one))
    o = oracle_for(oracle_mod, cm, N, mu=mu)
    s, t = o.steps(u, 10 ** 6, 0.5, 0.0, T, nthreads=NTH)
    assert t == T
    uu = u.reshape(-1, N + 1, N + 1, 4)
    v2 = uu[..., 2] / uu[..., 0]
    ref = 1e-3 * np.sin(k * (np.transpose(x, (2, 1, 0)) + 10.0)) * np.exp(-mu * k * k * T)
    assert np.abs(v2 - ref).max() < 2e-4 * 1e-3


def test_curved_mesh_boundaries(tl):
    m = cavity_mesh(tl, 4)
    cm = m.curved(3)
    assert cm.n_boundaries == 16 and list(cm.n_boundaries_per_direction) == [4, 4, 4, 4]
    assert cm.n_interfaces == 2 * 4 * 3
    xy = cm.boundary_node_coordinates(3)
    np.testing.assert_allclose(xy[0, :, :4], 0.0, atol=1e-15)     # x_neg
    np.testing.assert_allclose(xy[1, :, -4:], 1.0, atol=1e-15)    # y_pos
    # every element face is covered once by an interface or a boundary
    cover = np.zeros((cm.n_elements, 4), dtype=int)
    for e, f in zip(cm.primary_elements - 1, cm.primary_faces):
        cover[e, f] += 1
    for e, f in zip(cm.secondary_elements - 1, cm.secondary_faces):
        cover[e, f] += 1
    for e, f in zip(cm.boundary_elements - 1, cm.boundary_faces):
        cover[e, f] += 1
    assert np.all(cover == 1)


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, mu=None, lid=1.0):
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    bc = {"x_neg": tl.boundary_condition_slip_wall_vertical, "x_pos": tl.boundary_condition_slip_wall_vertical,
          "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    if mu is None:
        return tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.ConstantState(), solver, boundary_conditions=bc)
    eq_par = tl.CompressibleNavierStokesDiffusion2D(eq, mu=mu, Prandtl=0.72,
                                                    gradient_variables=tl.GradientVariablesConservative())
    heat = tl.Adiabatic(lambda x, y, t, e: 0.0)
    cavity = tl.BoundaryConditionNavierStokesWall(tl.NoSlip(lambda x, y, t, e: (0.0, 0.0)), heat)
    lidbc = tl.BoundaryConditionNavierStokesWall(tl.NoSlip(lambda x, y, t, e: (lid, 0.0)), heat)
    par = {"x_neg": cavity, "y_neg": cavity, "y_pos": lidbc, "x_pos": cavity}
    return tl.SemidiscretizationHyperbolicParabolic(mesh, tl.LW(), (eq, eq_par), tl.ConstantState(), solver,
                                                    boundary_conditions=(bc, par))


@pytest.mark.gpu
@pytest.mark.parametrize("N,mu,rotated", [(3, None, False), (4, None, True), (3, 0.01, False), (4, 0.01, False),
                                          (4, 0.01, True), (5, 0.01, False)])
def test_gpu_curved_walls_match_oracle(oracle_mod, tl, N, mu, rotated):
    cm = cavity_mesh(tl, 6).curved(N)
    if rotated:
        turns = np.random.default_rng(N).integers(0, 4, cm.n_elements)
        cm = tl.rotate_elements(cm, turns)
    semi = make_semi(tl, cm, N, mu)
    u0 = stirred(tl, cm)
    o = oracle_for(oracle_mod, cm, N, mu)
    dt = o.max_dt(u0, 0.3)
    semi.cache["dt"][0] = dt
    du_gpu = np.empty_like(u0)
    tl.rhs(du_gpu, u0, semi, 0.0)
    du_cpu = o.rhs(u0, 0.0, dt)
    assert np.all(rel_l2(u0 + dt * du_gpu, u0 + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-10)
    assert semi.max_dt(u0, 0.3) == pytest.approx(dt, rel=1e-14)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(8, 0.3, use_graph=True)
    integ.sync_time()
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 8, 0.3, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 8 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)


@pytest.mark.gpu
def test_gpu_warped_lid_driven_cavity_runs(tl):
    """The warped 64 x 64 cavity at N = 4 (Re = 1000 with lid speed 1 and side 1: mu = 0.001; Ma = 0.1,
    Pr = 0.72) for 2000 steps: admissible, mass conserved, the lid drags the layer below it. The steps use a
    fixed dt of the advective scale (5e-5, inside the viscous limit): the reference's parabolic max_dt reads
    inverse_jacobian[element] of the P4estMesh's per-node inverse area Jacobian (about 16384 here) and
    gives dt near 1e-9, with which 2000 steps leave the fluid at rest."""
    N = 4
    mesh = cavity_mesh(tl, 64)
    cm = mesh.curved(N)
    semi = make_semi(tl, mesh, N, mu=0.001)
    u0 = rest(cm, N)
    ode = tl.semidiscretize(semi, tl.LW(), (0.0, 1e9))
    integ = tl.LWIntegrator(ode)
    integ.set_state(u0, 0.0)
    assert semi.max_dt(u0, 0.98 * 5 * 0.103) < 1e-7
    integ.step(2000, 0.98 * 5 * 0.103, fixed_dt=5e-5, use_graph=True)
    integ.sync_time()
    assert integ.iter == 2000 and integ.t == pytest.approx(0.1)
    u = integ.get_state()
    assert np.all(np.isfinite(u))
    np.testing.assert_allclose(quad(cm, N, u)[0], quad(cm, N, u0)[0], rtol=1e-12)
    x, y = cm.xy
    xs = np.transpose(x, (2, 1, 0)).reshape(-1)
    ys = np.transpose(y, (2, 1, 0)).reshape(-1)
    uu = u.reshape(-1, 4)
    v1 = uu[:, 1] / uu[:, 0]
    assert v1[(np.abs(xs - 0.5) < 0.05) & (ys > 0.99)].mean() > 0.02
    assert v1[ys > 0.98].mean() > 0.01      # the whole lid layer moves with the lid
