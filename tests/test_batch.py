"""Batched form (tlw_batch_*): each instance of a batch must advance exactly like a single-instance run of
the same problem (same kernels, same per-instance dt), and like the oracle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFL_LIMIT = {3: 0.170, 4: 0.103, 5: 0.070}


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def make_instances(tl, seed, count, sides=(4, 8, 16), degrees=(3, 4, 5)):
    """Isentropic vortices on periodic [-10, 10]^2 with strength ~ U[1, 5], centre ~ U[-2, 2]^2."""
    from trixilw.batch import compute_coefficients
    rng = np.random.default_rng(seed)
    eq = tl.CompressibleEulerEquations2D(1.4)
    out = []
    for k in range(count):
        N = degrees[k % len(degrees)]
        side = int(rng.choice(sides))
        mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), int(np.log2(side)))
        ic = tl.IsentropicVortex(rng.uniform(1.0, 5.0), center=tuple(rng.uniform(-2.0, 2.0, 2)))
        out.append({"mesh": mesh, "polydeg": N, "ic": ic, "u0": compute_coefficients(mesh, N, ic, eq),
                    "cfl": 0.98 * (N + 1) * CFL_LIMIT[N]})
    return eq, out


def single_run(tl, eq, inst, nsteps, t_end=1e9):
    solver = tl.DGSEM(inst["polydeg"], tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(inst["mesh"], tl.LW(), eq, inst["ic"], solver)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, t_end)))
    integ.set_state(inst["u0"], 0.0)
    integ.step(nsteps, inst["cfl"], use_graph=True)
    integ.sync_time()
    return integ.get_state(), integ.t, integ.iter


def run_batch(tl, eq, insts, nsteps, use_graph=True, autotune=False, t_end=None):
    b = tl.LWBatch(eq)
    for inst in insts:
        b.add(inst["mesh"], inst["polydeg"])
    b.finalize()
    for i, inst in enumerate(insts):
        b.set_state(i, inst["u0"], 0.0, inst["cfl"], t_end[i] if t_end else float("inf"))
    if autotune:
        b.autotune(trials=2)
    b.step(nsteps, use_graph=use_graph)
    b.synchronize()
    res = [b.get_state(i) for i in range(len(insts))]
    b.close()
    return res


def test_batch_matches_single_instance_runs(tl):
    eq, insts = make_instances(tl, 1, 9)
    res = run_batch(tl, eq, insts, 6)
    for inst, (u, t, steps) in zip(insts, res):
        u1, t1, s1 = single_run(tl, eq, inst, 6)
        assert steps == s1 == 6
        assert t == t1
        np.testing.assert_array_equal(u, u1)


def test_batch_matches_oracle(tl, oracle_mod):
    eq, insts = make_instances(tl, 2, 3, sides=(4, 8))
    res = run_batch(tl, eq, insts, 5)
    for inst, (u, t, steps) in zip(insts, res):
        o = oracle_mod.Oracle(inst["mesh"], inst["polydeg"])
        uc = inst["u0"].copy()
        s, tc = o.steps(uc, 5, inst["cfl"], 0.0, 1e9, kind=0, nthreads=os.cpu_count() or 1)
        assert s == steps == 5
        assert t == pytest.approx(tc, rel=1e-13)
        assert np.all(rel_l2(u, uc) < 1e-12)


def test_batch_graph_stream_and_autotune_bitwise(tl):
    eq, insts = make_instances(tl, 3, 6, sides=(4, 8, 16))
    a = run_batch(tl, eq, insts, 5, use_graph=True)
    b = run_batch(tl, eq, insts, 5, use_graph=False)
    c = run_batch(tl, eq, insts, 5, use_graph=True, autotune=True)
    for (ua, ta, sa), (ub, tb, sb), (uc, tc, sc) in zip(a, b, c):
        assert sa == sb == sc == 5 and ta == tb == tc
        np.testing.assert_array_equal(ua, ub)
        np.testing.assert_array_equal(ua, uc)


def test_batch_final_time_per_instance(tl):
    eq, insts = make_instances(tl, 4, 4, sides=(4, 8))
    t_end = [0.05, 0.2, 1e9, 0.1]
    res = run_batch(tl, eq, insts, 40, t_end=t_end)
    for inst, te, (u, t, steps) in zip(insts, t_end, res):
        u1, t1, s1 = single_run(tl, eq, inst, 40, t_end=te)
        assert steps == s1 and t == t1
        if te < 1e8:
            assert t == pytest.approx(te, abs=1e-14) and steps < 40
        np.testing.assert_array_equal(u, u1)


def test_batch_domain_error(tl):
    eq, insts = make_instances(tl, 5, 2, sides=(4,))
    bad = insts[1]["u0"].copy().reshape(-1, 4)
    bad[0, 3] = -1.0          # negative energy at a face node of element 1: negative pressure
    insts[1]["u0"] = bad.reshape(-1)
    b = tl.LWBatch(eq)
    for inst in insts:
        b.add(inst["mesh"], inst["polydeg"])
    b.finalize()
    for i, inst in enumerate(insts):
        b.set_state(i, inst["u0"], 0.0, inst["cfl"])
    b.step(1)
    with pytest.raises(tl.DomainError):
        b.synchronize()
    b.close()
