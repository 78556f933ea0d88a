"""UnstructuredMesh2D (the reference's src/solvers/dgsem_unstructured_2d path): a periodic warped quadrilateral mesh
whose element frames are turned, so that interfaces pair every combination of sides and many secondary indices
run backwards (start_index n, index_increment -1). CPU: the oracle's restatement (free stream, conservation,
agreement with the P4estMesh conventions where the two coincide, use of the caller's normals, FR invariance under
element rotations, the reference's dependence of the blended flux on which element is primary); GPU: libtlw against the oracle, plain and with shock capturing, and the C ABI's refusals."""
import os

import numpy as np
import pytest

from test_curved import quad, rel_l2, vortex_state, warp
from test_curved_sc import blast_state

NTH = os.cpu_count() or 1


def unstructured(tl, N, cells=(5, 4), seed=1, rotate=True):
    cm = tl.StructuredMesh(cells, warp).curved(N)
    turns = np.random.default_rng(seed + N).integers(0, 4, cm.n_elements) if rotate else np.zeros(cm.n_elements, int)
    rm = tl.rotate_elements(cm, turns) if rotate else cm
    return cm, rm, tl.UnstructuredMesh2D.from_curved(rm), turns


def sc_oracle(oracle_mod, mesh, N, alpha_max=1.0, rec=0):
    o = oracle_mod.Oracle(mesh, N)
    o.set_shock_capturing(True, alpha_max=alpha_max, alpha_min=0.001, alpha_smooth=True, reconstruction=rec)
    return o


# ---------------------------------------------------------------------------------------------- CPU
def test_mesh_conventions(tl):
    _, rm, um, _ = unstructured(tl, 4)
    n = 5
    assert um.n_interfaces == 2 * um.n_elements
    assert set(np.unique(um.element_side_ids)) == {1, 2, 3, 4}
    assert np.any(um.index_increment == -1) and np.any(um.index_increment == 1)
    assert np.all(um.start_index[um.index_increment == -1] == n)
    # each element side belongs to exactly one interface
    used = np.zeros((um.n_elements, 4), int)
    for k in range(um.n_interfaces):
        for s in (0, 1):
            used[um.element_ids[s, k] - 1, um.element_side_ids[s, k] - 1] += 1
    assert np.all(used == 1)
    # the normals computed from the sides are the outward contravariant vectors at the side nodes
    Ja = rm.Ja   # [E, j, i, 4]
    nd = um.normal_directions
    np.testing.assert_allclose(nd[:, 0, :, 0], -Ja[:, 0, :, 2], atol=1e-12)      # bottom: -Ja^2
    np.testing.assert_allclose(nd[:, 1, :, 1], Ja[:, :, n - 1, 1], atol=1e-12)   # right: +Ja^1
    np.testing.assert_allclose(nd[:, 2, :, 1], Ja[:, n - 1, :, 3], atol=1e-12)   # top: +Ja^2
    np.testing.assert_allclose(nd[:, 3, :, 0], -Ja[:, :, 0, 0], atol=1e-12)      # left: -Ja^1


@pytest.mark.parametrize("N", [3, 4, 6])
def test_oracle_free_stream_and_conservation(oracle_mod, tl, N):
    _, rm, um, _ = unstructured(tl, N)
    o = oracle_mod.Oracle(um, N)
    u = np.tile(np.array([1.0, 0.3, -0.2, 2.5]), um.n_elements * (N + 1) ** 2)
    assert np.abs(o.rhs(u, 0.0, 0.05)).max() < 1e-11
    u = vortex_state(tl, um)
    du = o.rhs(u, 0.0, o.max_dt(u, 0.4))
    assert np.all(np.abs(quad(um, N, du)) < 1e-11)


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_fr_agrees_with_the_p4est_conventions(oracle_mod, tl, N):
    """With the FR volume integral and normals that are the contravariant vectors, dotting the secondary's flux
    with the primary's normal (unstructured) or with its own negated normal (P4estMesh) differs only by roundoff."""
    _, rm, um, _ = unstructured(tl, N)
    u = vortex_state(tl, um)
    o_u, o_p = oracle_mod.Oracle(um, N), oracle_mod.Oracle(rm, N)
    dt = o_p.max_dt(u, 0.4)
    assert o_u.max_dt(u, 0.4) == dt
    assert np.all(rel_l2(u + dt * o_u.rhs(u, 0.0, dt), u + dt * o_p.rhs(u, 0.0, dt)) < 1e-14)


def test_oracle_uses_the_callers_normals(oracle_mod, tl):
    """Scaling the given normal_directions scales the interface normal fluxes: the rhs changes."""
    N = 4
    _, rm, um, _ = unstructured(tl, N)
    u = vortex_state(tl, um)
    scaled = tl.UnstructuredMesh2D(um.xy, N, um.element_ids, um.element_side_ids, um.start_index,
                                   um.index_increment, um.area, normal_directions=1.5 * um.normal_directions)
    o, o2 = oracle_mod.Oracle(um, N), oracle_mod.Oracle(scaled, N)
    dt = o.max_dt(u, 0.4)
    assert np.all(rel_l2(o2.rhs(u, 0.0, dt), o.rhs(u, 0.0, dt)) > 1e-3)


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_fr_invariant_under_element_rotations(oracle_mod, tl, N):
    """The same mesh with and without turned element frames gives the same FR rhs."""
    cm, rm, um, turns = unstructured(tl, N, cells=(6, 6))
    um0 = tl.UnstructuredMesh2D.from_curved(cm)
    u = vortex_state(tl, cm, beta=4.0)
    ur = tl.rotate_state(u, N, turns)
    o0, o1 = oracle_mod.Oracle(um0, N), oracle_mod.Oracle(um, N)
    dt = o0.max_dt(u, 0.4)
    assert np.all(rel_l2(ur + dt * o1.rhs(ur, 0.0, dt), tl.rotate_state(u + dt * o0.rhs(u, 0.0, dt), N, turns)) < 1e-13)


def test_oracle_shock_capturing_depends_on_which_element_is_primary(oracle_mod, tl):
    """The reference's compute_alp tests the primary's first-order subcell update as U - c (Fn - fn_inner) with its
    fn_low oriented along +xi / +eta, which has the sign of the outward flux only when the primary's side is its
    right or top one; on its bottom or left side the test sees -Fn - fn_inner and the node often falls back to the
    first-order flux. Swapping primary and secondary of every interface therefore leaves the FR rhs unchanged (up
    to roundoff) but changes the shock-capturing one, even on a smooth state with alpha = 0 everywhere."""
    N = 3
    _, rm, um, _ = unstructured(tl, N, cells=(6, 6))
    sw = tl.UnstructuredMesh2D(um.xy, N, um.element_ids[::-1], um.element_side_ids[::-1], um.start_index,
                               um.index_increment, um.area)
    u = vortex_state(tl, um, beta=4.0)
    o, o2 = oracle_mod.Oracle(um, N), oracle_mod.Oracle(sw, N)
    dt = o.max_dt(u, 0.4)
    assert np.all(rel_l2(u + dt * o2.rhs(u, 0.0, dt), u + dt * o.rhs(u, 0.0, dt)) < 1e-14)
    s, s2 = sc_oracle(oracle_mod, um, N, alpha_max=0.0), sc_oracle(oracle_mod, sw, N, alpha_max=0.0)
    d = rel_l2(u + dt * s2.rhs(u, 0.0, dt), u + dt * s.rhs(u, 0.0, dt))
    assert np.all(s.get(6) == 0.0) and np.all(d > 1e-6)


@pytest.mark.parametrize("N,rec", [(3, 0), (4, 0), (6, 0), (4, 1)])
def test_oracle_shock_capturing_blast(oracle_mod, tl, N, rec):
    """The blast with the Sedov elixir's settings (alpha_max 1, first-order subcells; also MUSCL): blending active,
    conservation, and admissible steps."""
    _, rm, um, _ = unstructured(tl, N, cells=(8, 8))
    o = sc_oracle(oracle_mod, um, N, rec=rec)
    u = blast_state(um)
    dt = o.max_dt(u, 0.2)
    du = o.rhs(u, 0.0, dt)
    alpha = o.get(6)
    assert alpha.max() > 0.1 and (alpha == 0.0).sum() > 0
    assert np.all(np.abs(quad(um, N, du)) < 1e-11 * np.abs(quad(um, N, u)).max())
    mass0 = quad(um, N, u)
    s, _ = o.steps(u, 10, 0.2, 0.0, 1e9, nthreads=NTH)
    assert s == 10 and np.all(np.isfinite(u))
    np.testing.assert_allclose(quad(um, N, u), mass0, rtol=1e-12, atol=1e-12)


def test_oracle_refuses_what_the_reference_cannot_run(oracle_mod, tl):
    _, rm, um, _ = unstructured(tl, 4)
    o = oracle_mod.Oracle(um, 4)
    u = vortex_state(tl, um)
    with pytest.raises(RuntimeError):
        o.rhs(u, 0.0, 1e-3, kind=1)      # MDRK


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, sc=False, rec=None):
    eq = tl.CompressibleEulerEquations2D(1.4)
    vi = tl.VolumeIntegralFR(tl.LW())
    if sc:
        kw = {"reconstruction": rec} if rec is not None else {}
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=1.0), vi, **kw)
    return tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.ConstantState(), tl.DGSEM(N, tl.flux_lax_friedrichs, vi))


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 6])
def test_gpu_rhs_and_steps_match_oracle(oracle_mod, tl, N):
    _, rm, um, _ = unstructured(tl, N, cells=(6, 5))
    semi = make_semi(tl, um, N)
    u = vortex_state(tl, um)
    o = oracle_mod.Oracle(um, N)
    dt = o.max_dt(u, 0.4)
    assert semi.max_dt(u, 0.4) == pytest.approx(dt, rel=1e-14)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    ref = o.rhs(u, 0.0, dt)
    assert np.all(rel_l2(u + dt * du, u + dt * ref) < 1e-12)
    assert np.all(rel_l2(du, ref) < 1e-10)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u, 0.0)
    integ.step(6, 0.4)
    integ.sync_time()
    u_cpu = u.copy()
    s, t = o.steps(u_cpu, 6, 0.4, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 6 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("N,rec", [(3, 0), (4, 0), (6, 0), (4, 1)])
def test_gpu_shock_capturing_matches_oracle(oracle_mod, tl, N, rec):
    from trixilw import _lib
    _, rm, um, _ = unstructured(tl, N, cells=(8, 8))
    semi = make_semi(tl, um, N, sc=True, rec=tl.MUSCLReconstruction() if rec == 1 else None)
    u = blast_state(um)
    o = sc_oracle(oracle_mod, um, N, rec=rec)
    dt = o.max_dt(u, 0.2)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    ref = o.rhs(u, 0.0, dt)
    assert np.all(rel_l2(u + dt * du, u + dt * ref) < 1e-12)
    np.testing.assert_allclose(semi.get_cache(_lib.TLW_CACHE_ALPHA), o.get(6), rtol=1e-10, atol=1e-14)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u, 0.0)
    integ.step(8, 0.2)
    u_cpu = u.copy()
    s, _ = o.steps(u_cpu, 8, 0.2, 0.0, 1e9, nthreads=NTH)
    assert s == 8
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)


@pytest.mark.gpu
def test_gpu_unstructured_refusals(tl):
    """MDRK and boundaries are refused with TLW_E_UNSUPPORTED (the reference cannot run them on this mesh)."""
    _, rm, um, _ = unstructured(tl, 4)
    eq = tl.CompressibleEulerEquations2D(1.4)
    solver = tl.DGSEM(4, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.MDRK()))
    with pytest.raises(tl.TlwError) as ex:
        tl.SemidiscretizationHyperbolic(um, tl.MDRK(), eq, tl.ConstantState(), solver)
    from trixilw import _lib
    assert ex.value.code == _lib.TLW_E_UNSUPPORTED
