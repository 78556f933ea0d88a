"""Shock capturing across the L2 mortars of a curvilinear mesh (the reference's P4estMesh{2} path after an AMR
step, as its AMR shock elixirs run it): the blending factors smoothed over the mortars, get_blended_flux at every
small mortar node (dgsem_p4est/dg_2d.jl:506-603) with lw_mortars.inverse_jacobian either zero (before an AMR
step) or given. The oracle's properties on the CPU; libtlw against the oracle on the GPU."""
import os

import numpy as np
import pytest

from test_curved import quad, rel_l2, vortex_state
from test_curved_mortar import refined
from test_curved_sc import RECONSTRUCTIONS, blast_state

NTH = os.cpu_count() or 1


def sc_oracle(oracle_mod, cm, N, rec, alpha_max=0.5):
    o = oracle_mod.Oracle(cm, N)
    o.set_shock_capturing(True, alpha_max=alpha_max, alpha_min=0.001, alpha_smooth=True, reconstruction=rec)
    return o


def mortar_jacobian(cm, N):
    """A nonzero lw_mortars.inverse_jacobian: the J^{-1} of each mortar's first small element along its face."""
    n = N + 1
    ij = np.asarray(cm.inverse_jacobian_nodes).reshape(cm.n_elements, n, n)   # [e, j, i]
    out = np.empty((cm.n_mortars, n))
    for k in range(cm.n_mortars):
        e = int(cm.mortar_small1[k]) - 1
        f = int(cm.mortar_small_faces[k])
        for l in range(n):
            i, j = ((0, l), (N, l), (l, 0), (l, N))[f]
            out[k, l] = ij[e, j, i]
    return out


def evolved_blast(oracle_mod, cm, N, rec, steps=4):
    """The blast after a few oracle steps (nonzero MUSCL slopes, a smeared front crossing the mortars)."""
    o = sc_oracle(oracle_mod, cm, N, rec)
    u = blast_state(cm, p_in=3.0, center=(-2.0, -2.0), r0=5.0)
    o.steps(u, steps, 0.2, 0.0, 1e9, nthreads=NTH)
    return u


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [3, 4])
def test_oracle_sc_mortar_without_blending_is_the_fr_rhs(oracle_mod, tl, N):
    """alpha_max = 0 on a smooth state: no element is blended and get_blended_flux returns the LW flux (zero
    J^{-1} keeps the mortars' subcell test updates at u, and at the interfaces they stay admissible), so the
    rhs is the plain FR mortar rhs."""
    cm = refined(tl).curved(N)
    u = vortex_state(tl, cm)
    o = sc_oracle(oracle_mod, cm, N, 0, alpha_max=0.0)
    plain = oracle_mod.Oracle(cm, N)
    dt = plain.max_dt(u, 0.2)
    np.testing.assert_allclose(o.rhs(u, 0.0, dt), plain.rhs(u, 0.0, dt), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("rec", [0, 2])
@pytest.mark.parametrize("given_jacobian", [False, True])
def test_oracle_sc_mortar_conservation(oracle_mod, tl, rec, given_jacobian):
    """The blended mortar flux is single-valued and the large face takes its L2 projection: the periodic rhs
    conserves every variable, with blending at the mortars."""
    N = 4
    cm = refined(tl).curved(N)
    u = evolved_blast(oracle_mod, cm, N, rec)
    o = sc_oracle(oracle_mod, cm, N, rec)
    if given_jacobian:
        o.set_curved_mortar_jacobian(mortar_jacobian(cm, N))
    du = o.rhs(u, 0.0, o.max_dt(u, 0.2))
    alpha = o.get(6)
    large = np.asarray(cm.mortar_large) - 1
    assert alpha[large].max() > 0.05                  # blending reaches the mortars
    assert np.all(np.abs(quad(cm, N, du)) < 1e-10)


@pytest.mark.parametrize("rec", [0, 2])
def test_oracle_sc_mortar_flux_fix_fires_on_both_sides(oracle_mod, tl, rec):
    """With four times the small elements' J^{-1} as lw_mortars.inverse_jacobian the subcell test updates at the
    mortars leave the admissible set, and zhang_shu_flux_fix (dgsem_p4est/dg_2d.jl:199-225) changes the blended
    flux on the small side and on the large side; with a zero J^{-1} it never does. The rhs still conserves."""
    N = 4
    cm = refined(tl).curved(N)
    u = evolved_blast(oracle_mod, cm, N, rec)
    o = sc_oracle(oracle_mod, cm, N, rec)
    dt = o.max_dt(u, 0.2)
    o.rhs(u, 0.0, dt)
    assert np.all(o.get(8) == 0)
    o.set_curved_mortar_jacobian(4.0 * mortar_jacobian(cm, N))
    du = o.rhs(u, 0.0, dt)
    fixes = o.get(8)
    assert fixes[0] > 0 and fixes[1] > 0
    assert fixes.max() <= 2 * cm.n_mortars * (N + 1)
    assert np.all(np.abs(quad(cm, N, du)) < 1e-10)


def test_oracle_sc_mortar_smoothing_reaches_across(oracle_mod, tl):
    """Smoothing over the mortars: each small element's alpha is at least half its large neighbour's raw
    (unsmoothed) alpha, and the other way round."""
    N = 4
    cm = refined(tl).curved(N)
    u = evolved_blast(oracle_mod, cm, N, 1)
    o = sc_oracle(oracle_mod, cm, N, 1)
    raw = oracle_mod.Oracle(cm, N)
    raw.set_shock_capturing(True, alpha_max=0.5, alpha_min=0.001, alpha_smooth=False, reconstruction=1)
    dt = o.max_dt(u, 0.2)
    o.rhs(u, 0.0, dt)
    raw.rhs(u, 0.0, dt)
    a, r = o.get(6), raw.get(6)
    g = np.asarray(cm.mortar_large) - 1
    assert r[g].max() > 0.05
    for s in (cm.mortar_small1, cm.mortar_small2):
        s = np.asarray(s) - 1
        assert np.all(a[s] >= 0.5 * r[g]) and np.all(a[g] >= 0.5 * r[s])


# ---------------------------------------------------------------------------------------------- GPU
def sc_semi(tl, mesh, N, rec, td="lw"):
    eq = tl.CompressibleEulerEquations2D(1.4)
    t = tl.LW() if td == "lw" else tl.MDRK()
    vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5, alpha_min=0.001),
                                           tl.VolumeIntegralFR(t), reconstruction=RECONSTRUCTIONS[rec](tl))
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, vi)
    return tl.SemidiscretizationHyperbolic(mesh, t, eq, tl.ConstantState(), solver)


@pytest.mark.gpu
@pytest.mark.parametrize("N,rec,given_jacobian", [(3, 0, False), (4, 0, True), (4, 1, False), (4, 2, True),
                                                  (5, 2, False)])
def test_gpu_sc_mortar_rhs_matches_oracle(oracle_mod, tl, N, rec, given_jacobian):
    from trixilw import _lib
    cm = refined(tl).curved(N)
    u = evolved_blast(oracle_mod, cm, N, rec)
    o = sc_oracle(oracle_mod, cm, N, rec)
    semi = sc_semi(tl, cm, N, rec)
    if given_jacobian:
        mj = mortar_jacobian(cm, N)
        o.set_curved_mortar_jacobian(mj)
        semi.set_mortar_inverse_jacobian(mj)
    dt = o.max_dt(u, 0.2)
    du_cpu = o.rhs(u, 0.0, dt)
    semi.cache["dt"][0] = dt
    du_gpu = np.empty_like(u)
    tl.rhs(du_gpu, u, semi, 0.0)
    # the indicator's sigmoid is ill-conditioned near its threshold: small blending factors of the evolved
    # state agree to about 1e-13 absolute
    np.testing.assert_allclose(semi.get_cache(_lib.TLW_CACHE_ALPHA), o.get(6), rtol=1e-10, atol=1e-12)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("N,rec", [(3, 0), (4, 2), (5, 1)])
def test_gpu_sc_mortar_flux_fix_matches_oracle(oracle_mod, tl, N, rec):
    """The mortar nodes' zhang_shu_flux_fix branches on the GPU: four times the small elements' J^{-1} makes
    the fix fire on both sides of many small-mortar nodes (counted by the oracle), and the rhs matches."""
    cm = refined(tl).curved(N)
    u = evolved_blast(oracle_mod, cm, N, rec)
    mj = 4.0 * mortar_jacobian(cm, N)
    o = sc_oracle(oracle_mod, cm, N, rec)
    o.set_curved_mortar_jacobian(mj)
    semi = sc_semi(tl, cm, N, rec)
    semi.set_mortar_inverse_jacobian(mj)
    dt = o.max_dt(u, 0.2)
    du_cpu = o.rhs(u, 0.0, dt)
    fixes = o.get(8)
    assert fixes[0] > 0 and fixes[1] > 0
    semi.cache["dt"][0] = dt
    du_gpu = np.empty_like(u)
    tl.rhs(du_gpu, u, semi, 0.0)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("td", ["lw", "mdrk"])
def test_gpu_sc_mortar_steps_with_limiter_match_oracle(oracle_mod, tl, td):
    """10 CFL steps (N = 4, MUSCL-Hancock, given mortar J^{-1}) with the positivity limiter, LW and MDRK."""
    N, rec = 4, 2
    cm = refined(tl).curved(N)
    u0 = evolved_blast(oracle_mod, cm, N, rec)
    mj = mortar_jacobian(cm, N)
    semi = sc_semi(tl, cm, N, rec, td)
    semi.set_mortar_inverse_jacobian(mj)
    from trixilw import limiters
    t = tl.LW() if td == "lw" else tl.MDRK()
    integ = tl.LWIntegrator(tl.semidiscretize(semi, t, (0.0, 1e9)))
    limiters.install(semi, (tl.PositivityPreservingLimiterZhangShu((1e-6, 1e-6), (tl.density, tl.pressure)),))
    integ.set_state(u0, 0.0)
    integ.step(10, 0.2, use_graph=False)
    integ.sync_time()
    o = sc_oracle(oracle_mod, cm, N, rec)
    o.set_curved_mortar_jacobian(mj)
    o.set_positivity_limiter((1e-6, 1e-6), (0, 1))
    u_cpu = u0.copy()
    s, tt = o.steps(u_cpu, 10, 0.2, 0.0, 1e9, nthreads=NTH, kind=0 if td == "lw" else 1)
    assert s == integ.iter == 10 and integ.t == pytest.approx(tt, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)
