#!/usr/bin/env python
"""Throughput benchmark of the LW-FR time step (TrixiLW hot path) on B200.

Workload (default): isentropic vortex, periodic TreeMesh [-10,10]^2 with 512 x 512 elements, N = 4,
compressible Euler, FP64, Lax-Wendroff with CFL-based dt (cfl = 0.98 * (N+1) * 0.103) computed on the
device every step. A step is one perform_step! (dt reduction + rhs + update) over all 6.55 M nodes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Under torchrun with N > 1 ranks the default workload is one mesh split over the ranks (domain decomposition:
space-filling-curve ranges, cut-face trace exchange and a MAX all-reduce of the CFL maximum over NCCL; strong
scaling); --replicas runs N independent copies instead.

One JSON line on rank 0. `value`: whole-job DOF-updates/s with the state resident in HBM (CUDA events on
the library's stream around K graph-replayed steps, max over ranks). `e2e`: the same metric through
the C ABI with host buffers (per step: pinned host -> device upload of u, one step, device -> host
download of u). `--impl reference` times the CPU oracle port (the reference itself is Julia and cannot
run on these machines) on the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "trixilw.jl_b200"))

METRIC = "LW-FR DOF-updates/s on 1 B200 (% HBM roofline); batched & adjoint vs plain"
UNIT = "DOF-updates/s"

DEFAULT_WORKLOAD = "vortex_tree512_N4_lw"
# time discretizations of the domain-decomposed split step
DECOMPOSED_TD = ("lw", "mdrk")
# name -> (refinement level, N, time discretization, initial condition)
WORKLOADS = {
    "vortex_tree512_N4_lw": (9, 4, "lw", "vortex"),
    "vortex_tree512_N3_lw": (9, 3, "lw", "vortex"),
    "vortex_tree512_N5_lw": (9, 5, "lw", "vortex"),
    "vortex_tree256_N4_lw": (8, 4, "lw", "vortex"),
    "vortex_tree512_N4_mdrk": (9, 4, "mdrk", "vortex"),
    "riemann_tree512_N4_lw": (9, 4, "lw", "riemann"),
    # StructuredMesh{2} 512 x 512 on [-10, 10]^2 warped by x += sin(pi (x+10)/10) sin(pi (y+10)/10) (same for y)
    "vortex_warped512_N4_lw": (9, 4, "lw", "warped"),
    # compressible Navier-Stokes lid-driven cavity (Re 1000, Ma 0.1, Pr 0.72): [0, 1]^2 with 64 x 64 elements
    # warped by x += 0.05 sin(pi x) sin(pi y) (same for y), slip walls + no-slip adiabatic walls, lid v1 = 1
    "cavity_warped64_N4_ns": (6, 4, "lw", "cavity"),
    # shock capturing on the warped 512 x 512 StructuredMesh (the reference's P4estMesh path): a circular blast
    # (rho 1 / 0.125, p 10 / 1 at radius 3 around (0.5, -0.7)), Hennemann-Gassner blending (alpha_max 0.5) with
    # MUSCL subcells
    "blast_warped512_N4_muscl": (9, 4, "lw", "blast"),
}


class Blast:
    """Circular blast at rest: (rho, p) = (1, 10) inside radius 3 around (0.5, -0.7), (0.125, 1) outside."""

    time_independent = True

    def __call__(self, x, y, t, eq):
        import numpy as np
        x, y = np.broadcast_arrays(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64))
        inside = (x - 0.5) ** 2 + (y + 0.7) ** 2 < 9.0
        z = np.zeros(x.shape)
        return eq.prim2cons(np.where(inside, 1.0, 0.125), z, z, np.where(inside, 10.0, 1.0))
CAVITY_MU, CAVITY_PR, CAVITY_P0 = 0.001, 0.72, 1.0 / (0.1 ** 2 * 1.4)
# batched form: 512 independent vortex instances (per-instance seed 0..511: side from {8, 16, 32, 64}
# elements, degree from {3, 4, 5}, strength ~ U[1, 5], centre ~ U[-2, 2]^2), 50 LW steps
BATCH_WORKLOADS = {"batched512_vortex_lw": 512}
# differentiable form: 128 x 128 TreeMesh, N = 4, 200 LW steps, checkpoints every 20 steps
ADJOINT_WORKLOADS = {"adjoint128_vortex_lw": (7, 4, 200, 20)}
FALLBACK_HBM_GBS = 6650.0


def alg_bytes_per_element_step(N: int, td: str, curved: bool = False) -> float:
    """Algorithmic HBM bytes of one rhs/step per element (two-pass model): 8 nv (2n^2 + 28n - 8);
    an MDRK step is 2 B + 8 nv 6 n^2. Curvilinear meshes add the metric terms (Ja, 4 doubles, and J^-1 per
    node) read by the volume and CFL passes and, per interface node, Ja of the primary and J^-1 of both
    sides: 8 (2 * 5 n^2 + 2 n * 6)."""
    n, nv = N + 1, 4
    b = 8 * nv * (2 * n * n + 28 * n - 8)
    if curved:
        b += 8 * (2 * 5 * n * n + 2 * n * 6)
    return 2 * b + 8 * nv * 6 * n * n if td == "mdrk" else b


def volume_kernel_bytes_per_element(N: int, td: str, curved: bool = False, sc: bool = False) -> float:
    """Algorithmic bytes of one LW volume-kernel launch per element: read u (nv n^2), write u_new
    (nv n^2), write the face traces of U and F.n (2 x 4 faces x n x nv); curvilinear: read Ja and J^-1
    (5 n^2); shock capturing: write the fn_low traces (4 faces x n x nv), and on curvilinear meshes read the
    subcell normals (2 directions x n lines x (n - 1) faces x 2, and 2 x n x 2 for the calc_fn_low! normal)."""
    n, nv = N + 1, 4
    b = 2 * nv * n * n + 2 * 4 * n * nv + (5 * n * n if curved else 0)
    if sc:
        b += 4 * n * nv + (4 * n * (n - 1) + 4 * n if curved else 0)
    return 8.0 * b


def mdrk_volume_bytes_per_element(N: int) -> float:
    """Algorithmic bytes of the two compact MDRK stage kernels of a step per element: stage 1 reads u^n and writes
    u*, u_t and the U, F.n face traces; stage 2 reads u*, u^n and u_t and writes u^{n+1} and the face traces."""
    n, nv = N + 1, 4
    return 8.0 * (7 * nv * n * n + 2 * 2 * 4 * n * nv)


def mdrk_volume_flops_per_node(N: int) -> float:
    """Algorithmic FP64 flops per node of the two MDRK stage kernels of a step (FMA = 2, divides not counted):
    2 (8 n nv + 5 F_pair + 120) with F_pair = 17, the survey's count for two stages of two line contractions and
    five flux pairs each. (The compact stages recompute stage 1's five flux pairs in stage 2 instead of storing
    U2 and F2; those flops are not algorithmic and not counted.)"""
    n, nv = N + 1, 4
    return 2 * (8 * n * nv + 5 * 17 + 120)


def surface_pass_bytes_per_element(N: int) -> float:
    """Algorithmic (unique) bytes of one element-centric surface launch per element: read the element's own U
    and F.n face traces (2 x 4 faces x n x nv), read its 4(n - 1) face nodes of u for the jumps, read-modify-write
    the same face nodes of the output, write two CFL slots. The neighbours' traces and face nodes are the
    neighbours' own bytes, counted once there."""
    n, nv = N + 1, 4
    nb = 4 * (n - 1)
    return 8.0 * (2 * 4 * n * nv + 3 * nb * nv + 2)


def ns_volume_bytes_per_element(N: int) -> float:
    """Algorithmic bytes of the Navier-Stokes launches before the surfaces, per element on a curvilinear mesh:
    the BR1 gradient (read u, Ja, J^-1; write both gradients) and the parabolic LW volume kernel (read u, both
    gradients, Ja, J^-1; write u_new and the U, F.n, Fv.n face traces)."""
    n, nv = N + 1, 4
    grad = nv * n * n + 5 * n * n + 2 * nv * n * n
    vol = 3 * nv * n * n + 5 * n * n + nv * n * n + 3 * 4 * n * nv
    return 8.0 * (grad + vol)


def volume_flops_per_node(N: int) -> float:
    """Algorithmic FP64 flops per node of the LW volume kernel (FMA = 2, divides not counted):
    N >= 4: 20 n nv + 17 * 17 + 300; N = 3: 16 n nv + 11 * 17 + 200."""
    n, nv = N + 1, 4
    if N >= 4:
        return 20 * n * nv + 17 * 17 + 300
    return 16 * n * nv + 11 * 17 + 200


def host_link(nbytes: int, stream) -> dict:
    """The host link for one state: a pinned upload alone, a download alone, and both at once on two streams
    (best of five, CUDA events)."""
    import torch

    n = nbytes // 8
    h_in = torch.empty(n, dtype=torch.float64, pin_memory=True)
    h_out = torch.empty(n, dtype=torch.float64, pin_memory=True)
    d_a = torch.empty(n, dtype=torch.float64, device="cuda")
    d_b = torch.empty(n, dtype=torch.float64, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(up, down):
        best = float("inf")
        for r in range(6):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s1.wait_stream(stream)
            s2.wait_stream(stream)
            if up:
                with torch.cuda.stream(s1):
                    d_a.copy_(h_in, non_blocking=True)
            if down:
                with torch.cuda.stream(s2):
                    h_out.copy_(d_b, non_blocking=True)
            stream.wait_stream(s1)
            stream.wait_stream(s2)
            e1.record(stream)
            torch.cuda.synchronize()
            if r:
                best = min(best, e0.elapsed_time(e1))
        return best

    up, down, both = timed(True, False), timed(False, True), timed(True, True)
    return {"h2d_ms": up, "d2h_ms": down, "both_ms": both, "h2d_gbs": nbytes / up / 1e6,
            "d2h_gbs": nbytes / down / 1e6, "both_gbs": 2 * nbytes / both / 1e6}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(kernel_tag: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if one exists."""
    path = os.path.join(ROOT, "profiles", f"{kernel_tag}.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch_full_size:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1", "0x1"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def warp_mapping(xi, eta):
    """[-1, 1]^2 -> [-10, 10]^2 with a periodic sinusoidal warp of 5 % of the side."""
    import numpy as np
    X = 10.0 * xi
    Y = 10.0 * eta
    s = np.sin(np.pi * (X + 10.0) / 10.0) * np.sin(np.pi * (Y + 10.0) / 10.0)
    return X + s, Y + s


def cavity_mapping(xi, eta):
    """[-1, 1]^2 -> [0, 1]^2, then x += 0.05 sin(pi x) sin(pi y) and y likewise (the sides stay straight)."""
    import numpy as np
    X = 0.5 * (xi + 1.0)
    Y = 0.5 * (eta + 1.0)
    s = 0.05 * np.sin(np.pi * X) * np.sin(np.pi * Y)
    return X + s, Y + s


def cavity_ic(tl):
    return tl.ConstantState(rho=1.0, v1=0.0, v2=0.0, p=CAVITY_P0)


def make_mesh(tl, level, icname):
    if icname == "cavity":
        m = 1 << level
        return tl.StructuredMesh((m, m), cavity_mapping, periodicity=False)
    if icname in ("warped", "blast"):
        m = 1 << level
        return tl.StructuredMesh((m, m), warp_mapping)
    if icname == "vortex":
        return tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
    return tl.TreeMesh((0.0, 0.0), (1.0, 1.0), level, periodicity=False)


def build_semi(tl, level, N, td, icname, device):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    if icname == "warped":
        return tl.SemidiscretizationHyperbolic(make_mesh(tl, level, icname), tdo, eq, tl.IsentropicVortex(5.0),
                                               solver, device=device)
    if icname == "blast":
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), tl.VolumeIntegralFR(tdo),
                                               reconstruction=tl.MUSCLReconstruction())
        return tl.SemidiscretizationHyperbolic(make_mesh(tl, level, icname), tdo, eq, Blast(),
                                               tl.DGSEM(N, tl.flux_lax_friedrichs, vi), device=device)
    if icname == "cavity":
        eq_par = tl.CompressibleNavierStokesDiffusion2D(eq, mu=CAVITY_MU, Prandtl=CAVITY_PR,
                                                        gradient_variables=tl.GradientVariablesConservative())
        slip = {"x_neg": tl.boundary_condition_slip_wall_vertical, "x_pos": tl.boundary_condition_slip_wall_vertical,
                "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
        heat = tl.Adiabatic(lambda x, y, t, e: 0.0)
        wall = tl.BoundaryConditionNavierStokesWall(tl.NoSlip(lambda x, y, t, e: (0.0, 0.0)), heat)
        lid = tl.BoundaryConditionNavierStokesWall(tl.NoSlip(lambda x, y, t, e: (1.0, 0.0)), heat)
        walls = {"x_neg": wall, "x_pos": wall, "y_neg": wall, "y_pos": lid}
        return tl.SemidiscretizationHyperbolicParabolic(make_mesh(tl, level, icname), tdo, (eq, eq_par),
                                                        cavity_ic(tl), solver, device=device,
                                                        boundary_conditions=(slip, walls))
    if icname == "vortex":
        mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
        ic = tl.IsentropicVortex(5.0)
        semi = tl.SemidiscretizationHyperbolic(mesh, tdo, eq, ic, solver, device=device)
    else:
        # four-quadrant Riemann problem: Hennemann-Gassner blending (alpha_max = 0.5) with first-order
        # subcells, Dirichlet(initial condition) boundaries
        mesh = tl.TreeMesh((0.0, 0.0), (1.0, 1.0), level, periodicity=False)
        ic = tl.FourQuadrantRiemann()
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), tl.VolumeIntegralFR(tdo))
        solver = tl.DGSEM(N, tl.flux_lax_friedrichs, vi)
        semi = tl.SemidiscretizationHyperbolic(mesh, tdo, eq, ic, solver, device=device,
                                               boundary_conditions=tl.BoundaryConditionDirichlet(ic))
        semi._prepare_boundaries(0.0, 0.0, 1.0)
    return semi


# The Riemann workload with alpha_max = 0.5 loses admissibility above CFL ~ 0.3 (as the reference's scheme
# does without a positivity limiter); it is run at 0.15.
RIEMANN_CFL = 0.15


def cfl_for(N):
    """0.98 of the LW stability limit: trixi2lw(0.98) = 0.98 (N+1) lw_fourier_cfl(N) for N <= 4
    (src/auxiliary/auxiliary.jl:14-23). The reference tabulates no limit for N = 5; 0.98 * 6 * 0.07 is
    used there (a value below the N = 4 limit, stable on the vortex)."""
    table = {1: 1.000, 2: 0.333, 3: 0.170, 4: 0.103}
    return 0.98 * (N + 1) * table.get(N, 0.07)


def cpu_oracle_rate(level, N, td, icname, steps_hint, budget_s=20.0, warmup=1):
    """Oracle port (C++/OpenMP, all host threads) on the same workload: DOF-updates/s over a bounded
    number of steps (steps_hint, or as many as fit in about budget_s seconds, at least one) after `warmup`
    untimed steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    import trixilw as tl

    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = make_mesh(tl, level, icname)
    ic = (tl.FourQuadrantRiemann() if icname == "riemann" else cavity_ic(tl) if icname == "cavity"
          else Blast() if icname == "blast" else tl.IsentropicVortex(5.0))
    xy = mesh.curved(N).xy if icname in ("warped", "cavity", "blast") else mesh.node_coordinates(N)
    u = np.ascontiguousarray(np.transpose(ic(xy[0], xy[1], 0.0, eq), (2, 1, 0, 3))).reshape(-1)
    o = pyoracle.Oracle(mesh, N)
    if icname == "cavity":
        cm = mesh.curved(N)
        per = cm.n_boundaries_per_direction
        o.set_curved_boundaries(cm.boundary_elements, cm.boundary_faces,
                                np.repeat(np.array([1, 1, 2, 2], dtype=np.int32), per))
        o.set_parabolic(CAVITY_MU, CAVITY_PR)
        data = np.zeros((cm.n_boundaries, N + 1, 3))
        data[per[:3].sum():, :, 0] = 1.0
        o.set_walls(np.ones(cm.n_boundaries, dtype=np.int32), data)
    elif mesh.n_boundaries:
        bxy = mesh.boundary_node_coordinates(N)
        now = np.ascontiguousarray(np.transpose(ic(bxy[0], bxy[1], 0.0, eq), (1, 0, 2)))
        o.set_boundary_data(np.repeat(now[:, :, None, :], N + 1, axis=2), now)
    threads = os.cpu_count() or 1
    kind = 0 if td == "lw" else 1
    cfl = RIEMANN_CFL if icname in ("riemann", "blast") else cfl_for(N)
    if icname == "riemann":
        o.set_shock_capturing(True, 0.5, 0.001, True)
    if icname == "blast":
        o.set_shock_capturing(True, 0.5, 0.001, True, reconstruction=1)
    t0 = time.perf_counter()
    o.steps(u, max(1, warmup), cfl, 0.0, 1e9, kind=kind, nthreads=threads)
    one = (time.perf_counter() - t0) / max(1, warmup)
    nsteps = max(1, min(steps_hint, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    o.steps(u, nsteps, cfl, 0.0, 1e9, kind=kind, nthreads=threads)
    el = time.perf_counter() - t0
    return mesh.ndofs(N) * nsteps / el, threads, nsteps, el


def workload_config(workload, N, E, ndofs, td, cfl, world):
    """The `config` of a plain-workload line, the same for both arms."""
    return {"workload": workload, "polydeg": N, "elements": E, "ndofs": ndofs, "time_discretization": td,
            "cfl": cfl, "dt": "device CFL reduction every step",
            "l2": "inputs larger than L2 (state %.0f MB per array)" % (8 * 4 * ndofs / 1e6),
            "parallelism": f"replicas{world}" if world > 1 else "single"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    if args.workload in BATCH_WORKLOADS:
        return run_reference_batched(args, world)
    if args.workload in ADJOINT_WORKLOADS:
        return run_reference_adjoint(args, world)
    level, N, td, icname = WORKLOADS[args.workload]
    # W warm-up steps, then K timed steps of the full workload (fewer when K steps would take over 2 minutes)
    rate, threads, nsteps, el = cpu_oracle_rate(level, N, td, icname, steps_hint=max(1, args.steps), budget_s=120.0,
                                                warmup=max(args.warmup, 3))
    E = 1 << (2 * level)
    ndofs = E * (N + 1) ** 2
    cfl = RIEMANN_CFL if icname in ("riemann", "blast") else cfl_for(N)
    sample = f"{nsteps} full steps of the {args.workload} workload ({ndofs} DOF) in {el:.2f} s"
    out = {
        "metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": nsteps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * el / nsteps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, N, E, ndofs, td, cfl, 1),
        "implementation": "CPU oracle port (C++/OpenMP, all host threads) of the TrixiLW LW / MDRK step; the Julia "
                          "reference cannot run on these machines",
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_reference_adjoint(args, world):
    """Oracle port: forward sweep with stored states, then the reverse sweep of oracle adjoint steps (all host
    threads), on the same 128 x 128, N = 4 problem; as many steps as fit in about a minute."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    import trixilw as tl
    from trixilw.batch import compute_coefficients
    level, N, nsteps, ck = ADJOINT_WORKLOADS[args.workload]
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
    u0 = compute_coefficients(mesh, N, tl.IsentropicVortex(5.0), eq)
    u0 = u0 + 1e-3 * np.random.default_rng(0).standard_normal(u0.size)
    threads = os.cpu_count() or 1
    o = pyoracle.Oracle(mesh, N)
    cfl = cfl_for(N)
    t0 = time.perf_counter()
    states, dts, u = [], [], u0
    while len(dts) < nsteps and time.perf_counter() - t0 < 20.0:
        dt = o.max_dt(u, cfl)
        states.append(u)
        dts.append(dt)
        u = o.step_fixed(u, dt, nthreads=threads)
    t_fwd = time.perf_counter() - t0
    lam = np.zeros_like(u)
    lam[0::4] = u[0::4] - 1.0
    t1 = time.perf_counter()
    for x, dt in zip(reversed(states), reversed(dts)):
        lam = o.adjoint_step(x, dt, lam, nthreads=threads)
    t_adj = time.perf_counter() - t1
    k = len(dts)
    ndofs = mesh.ndofs(N)
    rate = ndofs * k / (t_fwd + t_adj)
    sample = (f"{k} of {nsteps} steps of the {args.workload} problem: forward {t_fwd:.2f} s, reverse {t_adj:.2f} s "
              "(states stored, no recomputation)")
    out = {
        "metric": METRIC, "value": rate, "unit": UNIT + " (forward steps differentiated per second)",
        "impl": "reference", "n_gpus": world, "steps": k, "warmup": 0, "ms_per_step": 1e3 * (t_fwd + t_adj) / k,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "implementation": "CPU oracle port (C++/OpenMP) of the LW step and "
                   "of its discrete adjoint; the reference has no adjoint and its Julia code cannot run here",
                   "gradient_cost_vs_forward": (t_fwd + t_adj) / t_fwd},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_reference_batched(args, world):
    """Oracle port over the uneven batch: instances one after another (each with all host threads), as many
    instances as fit in about a minute, 5 steps each."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    import trixilw as tl
    _, insts = batch_instances(tl, BATCH_WORKLOADS[args.workload])
    threads = os.cpu_count() or 1
    done, el, used = 0, 0.0, 0
    for inst in insts:
        o = pyoracle.Oracle(inst["mesh"], inst["polydeg"])
        u = inst["u0"].copy()
        t0 = time.perf_counter()
        o.steps(u, 5, inst["cfl"], 0.0, 1e9, kind=0, nthreads=threads)
        el += time.perf_counter() - t0
        done += 5 * inst["mesh"].ndofs(inst["polydeg"])
        used += 1
        if el > 60.0:
            break
    rate = done / el
    sample = f"5 steps of each of the first {used} of {len(insts)} instances in {el:.2f} s"
    out = {
        "metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": 5,
        "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "instances": len(insts), "implementation": "CPU oracle port "
                   "(C++/OpenMP) of the TrixiLW LW rhs, instances in sequence; the Julia reference cannot run here"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    import trixilw as tl
    from trixilw import _lib

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    level, N, td, icname = WORKLOADS[args.workload]
    semi = build_semi(tl, level, N, td, icname, local_rank)
    ndofs = semi.ndofs()
    cfl = RIEMANN_CFL if icname in ("riemann", "blast") else cfl_for(N)
    u0 = semi.compute_coefficients(0.0)
    upd = tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9))
    integ = tl.LWIntegrator(upd)
    integ.set_state(u0, 0.0)
    L = _lib.lib()
    sp = ctypes.c_void_p()
    L.tlw_get_stream(semi.handle, ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local_rank))

    # warm-up (also captures the CUDA graphs)
    integ.step(max(args.warmup, 3) if args.warmup > 0 else 3, cfl)
    check = L.tlw_synchronize(semi.handle)
    _lib.check(semi.handle, check)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[local_rank]) \
        if os.environ.get("CUDA_VISIBLE_DEVICES") else local_rank
    sampler = ClockSampler(gpu_index)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    integ.step(args.steps, cfl)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    _lib.check(semi.handle, L.tlw_synchronize(semi.handle))
    # per-phase device time of K further steps (events between the kernels of each step)
    phase = (ctypes.c_double * 5)()
    _lib.check(semi.handle, L.tlw_step_timed(semi.handle, args.steps, cfl, 0.0, 1e9, phase))
    clocks = sampler.stop()
    ms_max = ms
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = ndofs * args.steps * world / (ms_max * 1e-3)

    # end-to-end through the C ABI with host buffers. (a) tlw_step_host: a stream of independent states in
    # pinned host memory, each uploaded, advanced one step and downloaded, the copies of consecutive calls
    # overlapped (two alternating inputs and outputs); host wall clock from idle to idle. (b) the state
    # round-tripping through the host with the synchronous calls (tlw_set_state, tlw_step, tlw_get_state).
    n_e2e = max(3, min(args.steps, 20))
    ins = [integ.pinned_state() for _ in range(2)]
    outs = [integ.pinned_state() for _ in range(2)]
    ins[0][:] = u0
    integ.step_host(ins[0], outs[0], 0.0, 1, cfl)
    integ.synchronize()
    ins[1][:] = outs[0]
    for k in range(2):
        integ.step_host(ins[k], outs[k], 0.0, 1, cfl)
    integ.synchronize()
    barrier()
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for k in range(n_e2e):
        integ.step_host(ins[k % 2], outs[k % 2], 0.0, 1, cfl)
    integ.synchronize()
    ms_e2e = 1e3 * (time.perf_counter() - w0)
    barrier()
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = ndofs * n_e2e * world / (ms_e2e * 1e-3)
    uh = ins[0]
    ub = uh.ctypes.data_as(ctypes.c_void_p)
    tt = ctypes.c_double()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n_e2e):
        _lib.check(semi.handle, L.tlw_set_state(semi.handle, ub, _lib.TLW_WHERE_HOST, tt.value))
        _lib.check(semi.handle, L.tlw_step(semi.handle, 1, cfl, 0.0, 1e9, 1))
        _lib.check(semi.handle, L.tlw_get_state(semi.handle, ub, _lib.TLW_WHERE_HOST, ctypes.byref(tt)))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_rt = ndofs * n_e2e / (e0.elapsed_time(e1) * 1e-3)
    state_bytes = 8 * 4 * ndofs
    link = host_link(state_bytes, stream)

    if rank == 0:
        E = semi.mesh.n_elements
        curved = icname in ("warped", "cavity", "blast")
        ns = icname == "cavity"
        sc = icname in ("riemann", "blast")
        peak, peak_kind = measured_peaks()
        vol_ms = phase[1] / args.steps
        plain_mdrk = td == "mdrk" and not (ns or sc or curved)
        vol_bytes = (ns_volume_bytes_per_element(N) if ns else mdrk_volume_bytes_per_element(N) if plain_mdrk
                     else volume_kernel_bytes_per_element(N, td, curved, sc)) * E
        achieved = vol_bytes / (vol_ms * 1e-3) / 1e9
        fp = ctypes.c_double()
        fp64_peak = fp.value if L.tlw_probe_fp64_tflops(local_rank, ctypes.byref(fp)) == 0 else None
        vol_flops = (None if (ns or sc) else mdrk_volume_flops_per_node(N) * ndofs if plain_mdrk
                     else volume_flops_per_node(N) * ndofs)
        tag = (f"par_volume_kernel_N{N}_cavity{1 << level}" if ns
               else f"lw_volume_kernel_N{N}_blast_muscl{1 << level}" if icname == "blast"
               else f"mdrk_volume_kernels_N{N}_{'warped' if curved else 'tree'}{1 << level}" if td == "mdrk"
               else f"lw_volume_kernel_sc_N{N}_tree{1 << level}" if sc
               else f"lw_volume_kernel_N{N}_{'warped' if curved else 'tree'}{1 << level}")
        traffic = profile_traffic(tag)
        step_alg = alg_bytes_per_element_step(N, td, curved) * E
        # the binding roof of the volume kernel: the slower of its byte floor (HBM) and its flop floor (FP64)
        t_hbm = vol_bytes / (peak * 1e9)
        t_fp64 = vol_flops / (fp64_peak * 1e12) if (vol_flops and fp64_peak) else 0.0
        fp64_bound = t_fp64 > t_hbm
        hbm_rec = {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                   "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                   "alg_bytes_per_launch": vol_bytes, "floor_ms": 1e3 * t_hbm}
        fp64_rec = ({"achieved": vol_flops / (vol_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": (vol_flops / (vol_ms * 1e-3) / 1e12) / fp64_peak if fp64_peak else None,
                     "peak_source": "measured live (register FMA loop)", "alg_flops_per_launch": vol_flops,
                     "floor_ms": 1e3 * t_fp64} if vol_flops else
                    {"achieved": None, "peak": fp64_peak, "unit": "TFLOP/s",
                     "note": "no algorithmic flop model for the Navier-Stokes or the shock-capturing kernels"})
        binding = fp64_rec if fp64_bound else hbm_rec
        # a TreeMesh whose every face is an interface or a boundary runs one element-centric surface launch per
        # stage (surface_kernel); other meshes run the x and y sweeps
        surf_pass = not curved and not ns and getattr(semi.mesh, "n_mortars", 0) == 0
        stages = 2 if td == "mdrk" else 1
        surf_ms = (phase[2] + phase[3]) / args.steps
        phases_rec = {"cfl_dt": phase[0] / args.steps, "volume": phase[1] / args.steps, "surfaces": surf_ms,
                      "step": phase[4] / args.steps}
        surf_rec = None
        if surf_pass:
            sb = surface_pass_bytes_per_element(N) * E
            sgbs = sb / (surf_ms / stages * 1e-3) / 1e9
            surf_rec = {"kernel": f"surface_kernel<{N}>", "ms_per_launch": surf_ms / stages,
                        "alg_bytes_per_launch": sb, "achieved": sgbs, "unit": "GB/s", "frac": sgbs / peak,
                        "traffic": profile_traffic(f"surface_kernel_N{N}_tree{1 << level}")}
        else:
            phases_rec.update({"x_faces": phase[2] / args.steps, "y_faces": phase[3] / args.steps})
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.workload, N, E, ndofs, td, cfl, world),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                    "steps": n_e2e, "api": "tlw_step_host (pinned host in/out, one step per call, calls overlapped)",
                    "round_trip": {"value": e2e_rt, "unit": UNIT,
                                   "api": "tlw_set_state + tlw_step + tlw_get_state (synchronous, serial copies)"},
                    # the host link bounds it: a state up and a state down per step, at best concurrently
                    "link": {**link, "bound_value": ndofs / (link["both_ms"] * 1e-3),
                             "frac": e2e / (ndofs / (link["both_ms"] * 1e-3))}},
            "roofline": {"kernel": (f"grad_volume_kernel + curved_grad_*_kernel + par_volume_kernel<{N}, MODE_STEP, CURVED>"
                                    if ns else f"lw_volume_kernel<{N}, MODE_STEP, SC, CURVED, MUSCL>" if icname == "blast"
                                    else (f"mdrk1_volume_kernel<{N}, MODE_STEP{', CURVED' if curved else ', compact'}> + "
                                          f"mdrk2_volume_kernel<{N}, MODE_STEP{', CURVED' if curved else ', compact'}>")
                                    if td == "mdrk"
                                    else f"lw_volume_kernel<{N}, MODE_STEP{', SC' if sc else ''}{', CURVED' if curved else ''}>"),
                         "bound": "fp64" if fp64_bound else "hbm",
                         "achieved": binding["achieved"], "peak": binding["peak"], "unit": binding["unit"],
                         "frac": binding["frac"], "traffic": traffic,
                         "peak_source": binding["peak_source"], "ms_per_launch": vol_ms,
                         "binding_floor_ms": 1e3 * max(t_hbm, t_fp64),
                         "hbm": hbm_rec, "fp64": fp64_rec,
                         "step": {"alg_bytes_per_step": step_alg,
                                  "achieved_gbs": step_alg * args.steps / (ms_max * 1e-3) / 1e9,
                                  "frac": step_alg * args.steps / (ms_max * 1e-3) / 1e9 / peak},
                         "phase_ms_per_step": phases_rec,
                         **({"surface": surf_rec} if surf_rec else {})},
            "clocks": clocks,
            "gpu_launches": args.steps * ((8 + 2 * int(L.tlw_curved_colors(semi.handle))) if ns else
                                          (5 + int(L.tlw_curved_colors(semi.handle))) if icname == "blast" else
                                          (2 + 2 * stages + (1 if icname == "riemann" else 0))),
        }
        if world == 1 and not args.no_cpu_baseline:
            rate, threads, nsteps, el = cpu_oracle_rate(level, N, td, icname, steps_hint=args.steps)
            out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                   "sample": f"{nsteps} full steps of the same workload ({ndofs} DOF), {el:.1f} s"}
        if world == 1 and args.forms and args.workload == DEFAULT_WORKLOAD:
            out.update(forms_records())
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def forms_records():
    """The metric's other two forms, measured on their own workloads in the same run: the batched form against
    looping the plain path (512 uneven instances, 50 steps) and the adjoint gradient against the forward solve
    (128^2, N = 4, 200 steps, checkpoints every 20; 8 finite-difference directions)."""
    b = run_batched(argparse.Namespace(workload="batched512_vortex_lw", steps=50, warmup=3, no_cpu_baseline=True),
                    emit=False)
    a = run_adjoint(argparse.Namespace(workload="adjoint128_vortex_lw", steps=5, warmup=3, fd_directions=8),
                    emit=False)
    return {
        "batched": {"workload": "batched512_vortex_lw", "value": b["value"], "unit": UNIT, "steps": b["steps"],
                    "ms_per_step": b["ms_per_step"], "looped_plain": b["looped_plain"]["value"],
                    "speedup_vs_looped": b["speedup_vs_looped"],
                    "speedup_vs_looped_async": b["speedup_vs_looped_async"],
                    "per_instance_l2_error_max_rel_diff": b["per_instance_l2_error_max_rel_diff"],
                    "bitwise_equal_to_looped": b["bitwise_equal_to_looped"], "e2e": b["e2e"],
                    "instances": b["config"]["instances"], "ndofs_total": b["config"]["ndofs_total"]},
        "adjoint": {"workload": "adjoint128_vortex_lw", "value": a["value"], "unit": a["unit"],
                    "gradient_ms": a["gradient_ms"], "forward_solve_ms": a["forward_solve_ms"],
                    "gradient_cost_vs_forward": a["gradient_cost_vs_forward"],
                    "store_all_cost_vs_forward": a["store_all"]["gradient_cost_vs_forward"],
                    "fd_check": a["fd_check"], "nsteps": a["config"]["nsteps"],
                    "checkpoint_every": a["config"]["checkpoint_every"]},
    }


def run_decomposed(args):
    """Strong scaling of one TreeMesh over the ranks: each rank owns a contiguous range of the elements'
    space-filling-curve order and steps with the library's split step (tlw_dd_begin / _volume / _finish);
    the CFL maximum is all-reduced (MAX) and the cut-face traces exchanged with the neighbouring ranks over
    NCCL on the library's comm stream (the exchange overlaps the part's x interfaces). value = the whole mesh's DOF-updates over the max-over-ranks
    device time."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    import trixilw as tl
    from trixilw import _lib
    from trixilw.domain import DomainDecomposedLW, partition, torch_collectives

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if "RANK" not in os.environ:   # one rank without torchrun
        os.environ.update({"RANK": "0", "WORLD_SIZE": "1", "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": "29511"})
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local_rank))
    level, N, td, icname = WORKLOADS[args.workload]
    if td not in DECOMPOSED_TD or icname not in ("vortex",):
        raise SystemExit("--decompose: the periodic vortex workloads")
    mesh = make_mesh(tl, level, icname)
    part = partition(mesh, world)[rank]
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    semi = tl.SemidiscretizationHyperbolic(part.mesh, tdo, eq, tl.IsentropicVortex(5.0), solver, device=local_rank)
    cfl = cfl_for(N)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tdo, (0.0, 1e9)))
    u0 = semi.compute_coefficients(0.0)
    integ.set_state(u0, 0.0)
    allreduce_max, exchange = torch_collectives()
    dd = DomainDecomposedLW(semi, part, allreduce_max, exchange)
    dd.step(max(args.warmup, 3), cfl)
    torch.cuda.synchronize()
    gpu_index = int(os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local_rank]) \
        if os.environ.get("CUDA_VISIBLE_DEVICES") else local_rank
    sampler = ClockSampler(gpu_index)
    sampler.start()
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(dd.lib_stream)
    dd.step(args.steps, cfl)
    ev1.record(dd.lib_stream)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    t = torch.tensor([ev0.elapsed_time(ev1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    # end to end: this rank's part from pinned host memory, one split step, back to host
    n_e2e = max(1, min(args.steps, 10))
    uh = torch.empty(u0.size, dtype=torch.float64, pin_memory=True).numpy()
    uh[:] = u0
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(dd.lib_stream)
    for _ in range(n_e2e):
        integ.set_state(uh, 0.0)
        dd.step(1, cfl)
        uh[:] = integ.get_state()
    e1.record(dd.lib_stream)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_e2e = float(t.item())
    ndofs = mesh.ndofs(N)
    if rank == 0:
        part_bytes = 8 * 4 * part.mesh.ndofs(N)
        out = {
            "metric": METRIC, "value": ndofs * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "polydeg": N, "elements": mesh.n_elements, "ndofs": ndofs,
                       "time_discretization": td, "cfl": cfl, "parallelism": f"domain decomposition over {world} ranks (space-filling-curve "
                       "ranges; MAX all-reduce of the CFL maximum and cut-face trace exchange over NCCL)",
                       "halo_faces_rank0": int(len(part.halo_keys)),
                       "l2": "inputs larger than L2" if part_bytes > 126e6 else "state of a part may fit in L2"},
            "e2e": {"value": ndofs * n_e2e / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": part_bytes,
                    "d2h_bytes_per_step": part_bytes, "steps": n_e2e, "note": "per rank: its part"},
            "clocks": clocks,
            # speed, dt, volume, x / y interfaces, and per class of cut faces one pack and one halo launch
            "gpu_launches": args.steps * (2 + (3 + 2 * len({int(f) >> 1 for f in part.halo_faces}))
                                          * (2 if td == "mdrk" else 1)),
        }
        print(json.dumps(out), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def batch_instances(tl, count):
    """The uneven batch: instance k draws its parameters from numpy's default_rng(k)."""
    import numpy as np
    from trixilw.batch import compute_coefficients
    eq = tl.CompressibleEulerEquations2D(1.4)
    out = []
    for k in range(count):
        rng = np.random.default_rng(k)
        side = int(rng.choice([8, 16, 32, 64]))
        N = int(rng.choice([3, 4, 5]))
        beta = float(rng.uniform(1.0, 5.0))
        centre = tuple(float(c) for c in rng.uniform(-2.0, 2.0, 2))
        mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), side.bit_length() - 1)
        ic = tl.IsentropicVortex(beta, center=centre)
        out.append({"mesh": mesh, "polydeg": N, "ic": ic, "u0": compute_coefficients(mesh, N, ic, eq),
                    "cfl": cfl_for(N), "side": side})
    return eq, out


def run_batched(args, emit=True):
    """Batched form vs looping the plain (single-instance) path over the same instances. emit=False: return
    the record instead of printing it (rank 0)."""
    import numpy as np
    import torch

    import trixilw as tl
    from trixilw import _lib

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    count = BATCH_WORKLOADS[args.workload]
    eq, insts = batch_instances(tl, count)
    ndofs = [i["mesh"].ndofs(i["polydeg"]) for i in insts]
    total = sum(ndofs)
    K, W = args.steps, max(args.warmup, 3)
    L = _lib.lib()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- batched arm
    b = tl.LWBatch(eq, device=local_rank)
    for inst in insts:
        b.add(inst["mesh"], inst["polydeg"])
    b.finalize()
    for i, inst in enumerate(insts):
        b.set_state(i, inst["u0"], 0.0, inst["cfl"])
    t0 = time.perf_counter()
    choices = b.autotune(trials=3)
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.stream(), device=torch.device("cuda", local_rank))
    b.step(W)
    b.synchronize()
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[local_rank]) \
        if os.environ.get("CUDA_VISIBLE_DEVICES") else local_rank
    sampler = ClockSampler(gpu_index)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    ev0.record(stream)
    b.step(K)
    ev1.record(stream)
    torch.cuda.synchronize()
    wall_batch = time.perf_counter() - w0
    barrier()
    ms_batch = max_over_ranks(ev0.elapsed_time(ev1))
    b.synchronize()
    res_batch = [b.get_state(i) for i in range(count)]

    # e2e through the public API with host buffers: every step uploads all instances' states from pinned
    # host memory, runs one batch step and downloads all states
    n_e2e = 3
    hosts = []
    for i, inst in enumerate(insts):
        h = torch.empty(inst["u0"].size, dtype=torch.float64, pin_memory=True).numpy()
        h[:] = res_batch[i][0]
        hosts.append(h)
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for _ in range(n_e2e):
        for i, inst in enumerate(insts):
            _lib.check(b.ptr, L.tlw_batch_set_state(b.ptr, i, hosts[i].ctypes.data_as(ctypes.c_void_p),
                                                    _lib.TLW_WHERE_HOST, 0.0, inst["cfl"], 1e30), batch=True)
        b.step(1)
        for i in range(count):
            tt, ss = ctypes.c_double(), ctypes.c_int64()
            _lib.check(b.ptr, L.tlw_batch_get_state(b.ptr, i, hosts[i].ctypes.data_as(ctypes.c_void_p),
                                                    _lib.TLW_WHERE_HOST, ctypes.byref(tt), ctypes.byref(ss)),
                       batch=True)
    ms_e2e = max_over_ranks(1e3 * (time.perf_counter() - e0))
    b.close()

    # ---- looped plain arm: one single-instance handle per instance, K plain graph steps each, in a loop
    semis, integs = [], []
    for inst in insts:
        solver = tl.DGSEM(inst["polydeg"], tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
        semi = tl.SemidiscretizationHyperbolic(inst["mesh"], tl.LW(), eq, inst["ic"], solver, device=local_rank)
        integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e30)))
        integ.set_state(inst["u0"], 0.0)
        semis.append(semi)
        integs.append(integ)
    for inst, integ in zip(insts, integs):
        integ.step(W, inst["cfl"])
    torch.cuda.synchronize()
    # (a) a host loop of plain solves: each instance runs its K steps to completion (the plain API returns
    # the state to the caller) before the next one starts
    barrier()
    w0 = time.perf_counter()
    for inst, integ in zip(insts, integs):
        integ.step(K, inst["cfl"])
        _lib.check(integ.handle, L.tlw_synchronize(integ.handle))
    wall_loop = max_over_ranks(time.perf_counter() - w0)
    # (b) the same loop without waiting: every handle has its own stream, so the instances overlap on the
    # device and only the launch rate limits
    for inst, integ in zip(insts, integs):
        integ.set_state(inst["u0"], 0.0)
        integ.step(W, inst["cfl"])
    torch.cuda.synchronize()
    barrier()
    w0 = time.perf_counter()
    for inst, integ in zip(insts, integs):
        integ.step(K, inst["cfl"])
    torch.cuda.synchronize()
    wall_async = max_over_ranks(time.perf_counter() - w0)
    barrier()
    clocks = sampler.stop()
    # per-instance L2 errors against the exact (advected) vortex, both arms
    worst_err_diff, bitwise = 0.0, True
    for i, (semi, integ) in enumerate(zip(semis, integs)):
        u_loop = integ.get_state()
        integ.sync_time()
        u_b, t_b, s_b = res_batch[i]
        bitwise = bitwise and bool(np.array_equal(u_loop, u_b)) and integ.t == t_b
        l2_b, _ = tl.l2_linf_errors(semi, u_b, t_b)
        l2_l, _ = tl.l2_linf_errors(semi, u_loop, integ.t)
        worst_err_diff = max(worst_err_diff, float(np.max(np.abs(l2_b - l2_l) / np.maximum(np.abs(l2_l), 1e-300))))
    del integs, semis

    value = total * K * world / (ms_batch * 1e-3)
    loop_value = total * K * world / wall_loop
    if rank == 0:
        peak, peak_kind = measured_peaks()
        E_by_N = {}
        for inst in insts:
            E_by_N[inst["polydeg"]] = E_by_N.get(inst["polydeg"], 0) + inst["mesh"].n_elements
        step_alg = sum(alg_bytes_per_element_step(N, "lw") * E for N, E in E_by_N.items())
        achieved = step_alg * K / (ms_batch * 1e-3) / 1e9
        state_bytes = 8 * 4 * total
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_batch / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "instances": count, "ndofs_total": total,
                       "elements_by_degree": {str(k): v for k, v in sorted(E_by_N.items())},
                       "sides": sorted({i["side"] for i in insts}), "autotune": choices, "autotune_s": tune_s,
                       "l2": "inputs larger than L2 (state %.0f MB per array)" % (state_bytes / 1e6),
                       "parallelism": f"replicas{world}" if world > 1 else "single"},
            "looped_plain": {"value": loop_value, "unit": UNIT, "wall_s": wall_loop,
                             "how": f"host loop over {count} single-instance handles: {K} graph-replayed plain "
                                    "steps each, run to completion before the next instance; host wall clock"},
            "looped_plain_async": {"value": total * K * world / wall_async, "unit": UNIT, "wall_s": wall_async,
                                   "how": "the same loop without waiting per instance: each handle's stream "
                                          "overlaps the others on the device; host wall clock to device idle"},
            "batched_wall_s": wall_batch,
            "speedup_vs_looped": (total * K / wall_batch) / loop_value if wall_batch > 0 else None,
            "speedup_vs_looped_async": wall_async / wall_batch if wall_batch > 0 else None,
            "per_instance_l2_error_max_rel_diff": worst_err_diff,
            "bitwise_equal_to_looped": bitwise,
            "e2e": {"value": total * n_e2e * world / (ms_e2e * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes, "steps": n_e2e},
            "roofline": {"kernel": "batched LW step (all kernels of the graph)", "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                         "alg_bytes_per_step": step_alg},
            "clocks": clocks,
            "gpu_launches": K * (1 + 4 * len(E_by_N)),
        }
        if world == 1 and not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import pyoracle
            done, el, used = 0, 0.0, 0
            threads = os.cpu_count() or 1
            for inst in insts:
                o = pyoracle.Oracle(inst["mesh"], inst["polydeg"])
                u = inst["u0"].copy()
                t0 = time.perf_counter()
                o.steps(u, 5, inst["cfl"], 0.0, 1e9, kind=0, nthreads=threads)
                el += time.perf_counter() - t0
                done += 5 * inst["mesh"].ndofs(inst["polydeg"])
                used += 1
                if el > 15.0:
                    break
            out["cpu_baseline"] = {"value": done / el, "unit": UNIT, "cores": threads, "kind": "port",
                                   "sample": f"5 steps of each of the first {used} instances, {el:.1f} s"}
        if not emit:
            return out
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def run_adjoint(args, emit=True):
    """Gradient of J = 1/2 ||rho(T) - rho_target||^2 with respect to the discrete initial state by the
    checkpointed discrete adjoint, against the cost of the plain forward solve; central finite differences
    on 64 random unit directions check it."""
    import numpy as np
    import torch

    import trixilw as tl
    from trixilw import _lib
    from trixilw.batch import compute_coefficients

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    level, N, nsteps, ck = ADJOINT_WORKLOADS[args.workload]
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.IsentropicVortex(5.0), solver, device=local_rank)
    cfl = cfl_for(N)
    u0 = compute_coefficients(mesh, N, tl.IsentropicVortex(5.0), eq)
    u0 = u0 + 1e-3 * np.random.default_rng(0).standard_normal(u0.size)
    ut0 = compute_coefficients(mesh, N, tl.IsentropicVortex(4.5), eq)
    target = np.ascontiguousarray(tl.forward_record(semi, ut0, nsteps, cfl, ck)[0::4])
    ndofs = semi.ndofs()
    L = _lib.lib()
    sp = ctypes.c_void_p()
    L.tlw_get_stream(semi.handle, ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local_rank))
    # device-resident inputs for the timed calls
    d_u0 = torch.tensor(u0, dtype=torch.float64, device="cuda")
    d_target = torch.tensor(target, dtype=torch.float64, device="cuda")
    d_grad = torch.empty_like(d_u0)
    d_uT = torch.empty_like(d_u0)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    J = ctypes.c_double()
    ph = (ctypes.c_double * 3)()

    def gradient(timing=False, every=ck):
        _lib.check(semi.handle, L.tlw_adjoint_solve(semi.handle, vp(d_u0), nsteps, cfl, every, vp(d_target),
                                                    vp(d_grad), ctypes.byref(J), vp(d_uT), _lib.TLW_WHERE_DEVICE,
                                                    ph if timing else None))

    def forward():
        _lib.check(semi.handle, L.tlw_set_state(semi.handle, vp(d_u0), _lib.TLW_WHERE_DEVICE, 0.0))
        _lib.check(semi.handle, L.tlw_step(semi.handle, nsteps, cfl, 0.0, 1e30, 1))

    W = max(args.warmup, 3)
    for _ in range(W):
        forward()
        gradient()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    reps = max(1, min(args.steps, 5))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(reps):
        forward()
    ev[1].record(stream)
    torch.cuda.synchronize()
    ev[2].record(stream)
    for _ in range(reps):
        gradient()
    ev[3].record(stream)
    torch.cuda.synchronize()
    fwd_ms = ev[0].elapsed_time(ev[1]) / reps
    grad_ms = ev[2].elapsed_time(ev[3]) / reps
    gradient(timing=True)
    phases = tuple(ph)
    g_ck = d_grad.clone()
    # the same gradient with every step's data kept from the record pass (one segment: no recomputation)
    for _ in range(2):
        gradient(every=nsteps)
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(reps):
        gradient(every=nsteps)
    ev[1].record(stream)
    torch.cuda.synchronize()
    all_ms = ev[0].elapsed_time(ev[1]) / reps
    all_equal = bool(torch.equal(d_grad, g_ck))
    clocks = sampler.stop()
    # e2e through the public API with host arrays
    e0 = time.perf_counter()
    Jh, g_host, uT_host = tl.adjoint_solve(semi, u0, nsteps, cfl, ck, target)
    e2e_s = time.perf_counter() - e0
    # finite-difference check with the recorded dt sequence held fixed
    dts = tl.adjoint.dt_sequence(semi, nsteps)

    def Jf(x):
        return 0.5 * np.sum((tl.solve_dts(semi, x, dts)[0::4] - target) ** 2)

    rng = np.random.default_rng(0)
    worst = 0.0
    h = 1e-4
    for _ in range(args.fd_directions):
        d = rng.standard_normal(u0.size)
        d /= np.linalg.norm(d)
        d1 = (Jf(u0 + h * d) - Jf(u0 - h * d)) / (2 * h)
        d2 = (Jf(u0 + 2 * h * d) - Jf(u0 - 2 * h * d)) / (4 * h)
        ref = (4 * d1 - d2) / 3
        worst = max(worst, abs(float(g_host @ d) - ref) / max(abs(ref), 1e-300))
    value = ndofs * nsteps / (grad_ms * 1e-3)
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT + " (forward steps differentiated per second)",
            "n_gpus": world, "steps": nsteps, "warmup": W, "ms_per_step": grad_ms / nsteps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "polydeg": N, "elements": mesh.n_elements, "ndofs": ndofs,
                       "nsteps": nsteps, "checkpoint_every": ck, "cfl": cfl,
                       "objective": "J = 1/2 sum over nodes (rho(T) - rho_target)^2, rho_target from a strength-4.5 run",
                       "u0": "strength-5 vortex + N(0, 1e-3^2) noise (seed 0)", "repeats": reps},
            "forward_solve_ms": fwd_ms, "gradient_ms": grad_ms, "gradient_cost_vs_forward": grad_ms / fwd_ms,
            # phases timed one after another on one stream; the timed gradient overlaps the recomputation
            # with the adjoint steps
            "phase_ms": {"forward_record": phases[0], "recompute": phases[1], "adjoint_steps": phases[2],
                         "serial": True},
            "backward_cost_vs_forward": (grad_ms - phases[0]) / fwd_ms,
            "store_all": {"checkpoint_every": nsteps, "gradient_ms": all_ms, "gradient_cost_vs_forward": all_ms / fwd_ms,
                          # per step: the input state (4 values a node), U traces (16 / (N + 1) a node) and
                          # stage derivatives (4 * depth a node), plus u(T)
                          "device_bytes": int(8 * ndofs * (nsteps * (4 + 16 / (N + 1) + 4 * (4 if N >= 4 else 3)) + 4)),
                          "gradient_bit_equal": all_equal},
            "J": Jh, "fd_check": {"directions": args.fd_directions, "h": h, "max_rel_err": worst, "richardson": True},
            "e2e": {"value": ndofs * nsteps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * 5 * ndofs / nsteps,
                    "d2h_bytes_per_step": 8 * 8 * ndofs / nsteps, "seconds": e2e_s},
            "clocks": clocks,
            # per gradient: record 5 a step (speed, dt, volume, 2 interface sweeps), objective 2, recompute 3 a
            # step (the last segment comes from the record, each segment's last step is a volume launch only),
            # adjoint 2 a step
            "gpu_launches": reps * (5 * nsteps + 2 + 3 * (nsteps - ck) - 2 * ((nsteps - 1) // ck) + 2 * nsteps),
        }
        if not emit:
            return out
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS) + sorted(ADJOINT_WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", dest="forms", action="store_false",
                    help="default workload: leave out the batched and adjoint sub-records")
    ap.add_argument("--fd-directions", type=int, default=64,
                    help="adjoint workload: random directions of the finite-difference gradient check")
    ap.add_argument("--decompose", action="store_true",
                    help="split one mesh over the ranks (halo exchange over NCCL) also at one rank; under torchrun "
                         "with more than one rank this is the default for the periodic vortex workloads")
    ap.add_argument("--replicas", action="store_true",
                    help="under torchrun: N independent replicas of the workload instead of one mesh split over the ranks")
    args = ap.parse_args()
    world = dist_env()[2]
    decomposable = args.workload in WORKLOADS and WORKLOADS[args.workload][3] == "vortex" and \
        WORKLOADS[args.workload][2] in DECOMPOSED_TD
    if args.impl == "ours" and decomposable and (args.decompose or (world > 1 and not args.replicas)):
        run_decomposed(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload in BATCH_WORKLOADS:
        run_batched(args)
    elif args.workload in ADJOINT_WORKLOADS:
        run_adjoint(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
