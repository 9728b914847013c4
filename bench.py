#!/usr/bin/env python
"""PISO steps/s of the Taylor-Hood P2/P1 tetrahedral Navier-Stokes step on B200.

Workload (one "step" = one pisoStep): cylinder L=30, R=2 along x, ~1M tets (16 disk rings x 217
axial prism layers -> 999,936 tets, N2 = 1,378,515 P2 nodes, nv = 178,106 pressure DOFs),
rho = 1060, nu = 0.004, dt = 0.01, parabolic inlet u_x = 2*0.5*(1 - r^2/4), no-slip wall, p = 0
outlet, FP64, two-level CG pressure (single-reduction CG with Jacobi plus an aggregation coarse
correction) and batched Jacobi CG momentum (the momentum system is symmetric positive definite; the
reference solves it with BiCGSTAB, `--momentum-solver bicgstab`) to 1e-10 relative residual, from rest. The CPU baseline is the oracle port of the reference algorithm (BiCGSTAB pressure).
The mesh is synthetic (the reference meshes with TetGen, which is not available here).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cfsa|reference]

Multi-GPU (torchrun, one rank per GPU): the step does not shard in this build, every rank runs
an independent replica ("replicas only"); value = all ranks' steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "cell-fluid-structure-analysis_b200"
sys.path.insert(0, str(PKG))

METRIC = "PISO steps/s at 1M tets (FP64 GPU step)"
DATA = "synthetic: procedural cylinder mesh (TetGen unavailable), random-free"
UNIT = "steps/s"
GEOM = dict(length=30.0, radius=2.0, rings=16, layers=217)
FLUID = (1060.0, 0.004)
DT = 0.01
TOL = 1e-10
MAXIT = (5000, 50000)
INLET_PEAK = 2 * 0.5


ADJ_GEOM = dict(rings=8, layers=217)  # 249,984 tets: the 1M mesh coarsened 2x in the cross-section
ADJ_STEPS, ADJ_CHECKPOINT, ADJ_SEED, ADJ_NODES = 50, 10, 20261203, 20
ADJ_TOL = 1e-18  # Jacobi-scaled; see adjoint_section
ADJ_PATCH = dict(kind=0, axis=0, lo=14.0, hi=16.0)  # wall patch at mid-length of the x-axis tube


class MT19937_64:
    """64-bit Mersenne Twister (Nishimura, ACM TOMACS 10(4), 2000), the generator behind C++
    std::mt19937_64; used to pick the seeded inlet nodes."""

    def __init__(self, seed: int):
        self.mt = [0] * 312
        self.mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, 312):
            self.mt[i] = (6364136223846793005 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.idx = 312

    def __call__(self) -> int:
        if self.idx >= 312:
            for i in range(312):
                x = (self.mt[i] & 0xFFFFFFFF80000000) | (self.mt[(i + 1) % 312] & 0x7FFFFFFF)
                xa = x >> 1
                if x & 1:
                    xa ^= 0xB5026F5AA96619E9
                self.mt[i] = self.mt[(i + 156) % 312] ^ xa
            self.idx = 0
        y = self.mt[self.idx]
        self.idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y


def seeded_nodes(candidates, count, seed):
    """`count` distinct entries of `candidates`: raw mt19937_64(seed) draws modulo the candidate
    count, repeats skipped."""
    g = MT19937_64(seed)
    out = []
    while len(out) < min(count, len(candidates)):
        c = int(candidates[g() % len(candidates)])
        if c not in out:
            out.append(c)
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cfsa", choices=["cfsa", "reference"])
    ap.add_argument("--rings", type=int, default=GEOM["rings"])
    ap.add_argument("--layers", type=int, default=GEOM["layers"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--momentum-solver", default=MOMENTUM_SOLVER, choices=sorted(MOMENTUM),
                    help="momentum Krylov method of the FP64 headline step")
    ap.add_argument("--no-oracle", action="store_true",
                    help="skip every oracle run (parity at 1M tets, config-2 CPU comparison, CPU baseline)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision run")
    ap.add_argument("--mixed-marks", default="1,50,200", help="steps at which the mixed-precision comparison reads the fields")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint run")
    ap.add_argument("--no-y-bifurcation", action="store_true",
                    help="skip the ~4M-tet Y-bifurcation run (mixed precision + adjoint)")
    ap.add_argument("--y-steps", type=int, default=20, help="steps of each config-4 run")
    ap.add_argument("--y-checkpoint", type=int, default=5, help="checkpoint interval of the config-4 adjoint")
    ap.add_argument("--y-cell", type=float, default=0.081, help="lattice edge of the Y-bifurcation mesh")
    ap.add_argument("--adjoint-fd-nodes", type=int, default=ADJ_NODES,
                    help="seeded inlet nodes checked against central finite differences")
    ap.add_argument("--reference-budget-s", type=float, default=120.0,
                    help="cap on each timed CPU loop of --impl reference")
    ap.add_argument("--reference-single-core-steps", type=int, default=5,
                    help="steps of the 1-thread figure of --impl reference (0: skip)")
    return ap.parse_args()


def workload_desc(sizes, rings, layers, world):
    """The workload both arms run (mesh, boundary conditions, fluid, time step, stopping rule);
    each arm names its Krylov methods in its own "solver" key. sizes = (nv, nt, ne)."""
    nv, nt, ne = sizes
    return {
        "workload": f"cylinder L=30 R=2, {nt} tets ({rings} rings x {layers} layers), "
                    f"N2={nv + ne} P2 nodes, nv={nv}; FP64 PISO from rest, parabolic inlet peak 1.0, no-slip wall, "
                    f"p=0 outlet, rho 1060, nu 0.004, dt 0.01, Krylov solves to 1e-10 relative residual",
        "tets": nt, "p2_nodes": nv + ne, "pressure_dofs": nv,
        "velocity_dofs": 3 * (nv + ne),
        "l2": "no flush: momentum operator ~0.5 GB and M ~0.3 GB stream through the 126 MB L2 every step",
        "parallelism": f"replicas x{world}",
    }


def gpu_solver_label():
    mom = "Jacobi CG" if MOMENTUM_SOLVER == "cg" else "Jacobi BiCGSTAB"
    return ("two-level CG pressure (single-reduction CG, Jacobi + ~256-aggregate coarse correction) + "
            f"batched 3-component {mom} momentum, FP64, on the GPU")
REF_SOLVER = ("reference algorithm (src/FEM/NavierStokes.cpp:416-668): Jacobi BiCGSTAB pressure + per-component "
              "Jacobi BiCGSTAB momentum, FP64, oracle port on the host cores")


def make_mesh(cf, rings, layers):
    m = cf.Mesh.cylinder(GEOM["length"], GEOM["radius"], rings, layers)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    return m


MOMENTUM = {"bicgstab": 1, "cg": 0}  # --momentum-solver -> CFSA_KRYLOV_BICGSTAB / CFSA_KRYLOV_CG
MOMENTUM_SOLVER = "cg"


def bicgstab_headline(cf, m, steps, warm, world):
    """The headline workload with the momentum method the configuration names, the reference's
    batched Jacobi BiCGSTAB, instead of the headline's Jacobi CG: same mesh, inputs, pressure
    solver, criterion, warm-up and step count, timed with CUDA events on this rank. Any failure is
    reported in the returned record instead of ending the run."""
    global MOMENTUM_SOLVER
    saved = MOMENTUM_SOLVER
    try:
        MOMENTUM_SOLVER = "bicgstab"
        s, _ = make_solver(cf, m)
    except Exception as e:  # noqa: BLE001 - a side measurement must not end the bench line
        return {"ok": False, "error": str(e)}
    finally:
        MOMENTUM_SOLVER = saved
    try:
        ok, _ = s.pisoSteps(warm)
        ok2, done = s.pisoSteps(steps)
        st = s.stats()
        ms = st["last_step_ms"]
        return {"what": "the same FP64 headline with batched Jacobi BiCGSTAB momentum (the reference's method "
                        "and the configuration's); device time of this rank",
                "ok": bool(ok and ok2 and done == steps), "value": world * done / (ms / 1e3) if ms > 0 else 0.0,
                "unit": UNIT, "ms_per_step": ms / max(done, 1),
                "krylov_iters_per_step": [st["krylov_iters"][0] / max(done, 1), st["krylov_iters"][1] / max(done, 1)]}
    except Exception as e:  # noqa: BLE001
        return {"ok": False, "error": str(e)}
    finally:
        del s


def make_solver(cf, m, tol=TOL, norm=0):
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(tol, tol)
    s.setConvergenceNorm(norm)
    s.setMaxIterations(*MAXIT)
    s.setPressureSolver(cf.KRYLOV_CG2L)
    s.setMomentumSolver(MOMENTUM[MOMENTUM_SOLVER])
    s.setDt(DT)
    s.initialize(m, cf.Fluid(*FLUID))  # from rest; inlet set after initialize (CLI order)
    profile = cf.parabolic_inlet(m.nodePositions(), INLET_PEAK, GEOM["radius"])
    s.setInletVelocityProfile(profile)
    return s, profile


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self, indices):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                if int(f[0]) not in indices:
                    continue
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_table():
    p = ROOT / "profiles" / "dram_traffic.json"
    return json.loads(p.read_text()) if p.exists() else {}


def adjoint_section(cf, args, barrier):
    """Discrete adjoint on the 250k-tet cylinder: 50 FP64 PISO steps from rest, objective
    J = mean |WSS|^2 over the wall vertices with 14 <= x <= 16, checkpoint every 10 steps with
    recomputation; gradients with respect to every inlet nodal axial velocity and the viscosity,
    checked against central finite differences (h = 1e-6; relative h for the viscosity) on seeded
    inlet nodes. The 1e10 inlet penalty rows dominate ||b|| of the momentum solve even in the
    Jacobi-scaled norm, so the relative tolerance pins the interior only loosely; the FD
    quotients need the Krylov solves at 1e-18 (Jacobi-scaled) to get their solver noise below
    the 1e-5 bar, and the adjoint run uses the same setting."""
    m = make_mesh(cf, ADJ_GEOM["rings"], ADJ_GEOM["layers"])
    nv, nt, ne, _, _ = m.sizes
    prof = cf.parabolic_inlet(m.nodePositions(), INLET_PEAK, GEOM["radius"])
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(ADJ_TOL, ADJ_TOL)
    s.setConvergenceNorm(cf.NORM_JACOBI)
    s.setMaxIterations(50000, 200000)
    s.setPressureSolver(cf.KRYLOV_CG2L)
    s.setDt(DT)
    s.initialize(m, cf.Fluid(*FLUID))
    s.setInletVelocityProfile(prof)
    u0, p0 = s.getVelocity().copy(), s.getPressure().copy()
    barrier()
    ok = s.adjointForward(ADJ_STEPS, ADJ_CHECKPOINT)
    g = s.adjointBackward(**ADJ_PATCH) if ok else None
    barrier()
    if g is None:
        return {"ok": False, "error": "forward pass failed"}
    st = s.adjointStats()
    p1, p2 = m.fluidBC()
    inlet = np.nonzero(np.concatenate([p1, p2]) == 1)[0]
    res = {
        "workload": f"discrete adjoint: cylinder L=30 R=2, {nt} tets ({ADJ_GEOM['rings']} rings x "
                    f"{ADJ_GEOM['layers']} layers), N2={nv + ne}; {ADJ_STEPS} FP64 PISO steps from rest, "
                    f"parabolic inlet peak 1.0, J = mean |WSS|^2 over wall vertices with 14<=x<=16, "
                    f"checkpoint every {ADJ_CHECKPOINT} steps; Krylov tol {ADJ_TOL:g} (Jacobi-scaled)",
        "J": g["J"], "grad_viscosity": g["grad_viscosity"], "inlet_nodes": int(len(inlet)),
        "forward_ms": st["forward_ms"], "backward_ms": st["backward_ms"],
        "recomputed_steps": st["recomputed_steps"], "checkpoints": st["checkpoints"],
        "record_mb": st["record_bytes"] / 2**20,
        "adjoint_krylov_iters": [st["momentum_iters"], st["pressure_iters"]],
        "gpu_launches_backward": st["kernel_launches"],
        "steps_per_s_forward_plus_backward": ADJ_STEPS / ((st["forward_ms"] + st["backward_ms"]) / 1e3),
        "backward_over_forward": st["backward_ms"] / st["forward_ms"],
    }
    nodes = seeded_nodes(inlet, args.adjoint_fd_nodes, ADJ_SEED)
    if nodes:
        h = 1e-6

        def J_of(pr, nu=FLUID[1]):
            s.setViscosity(nu)
            s.setInletVelocityProfile(pr)
            s.setFields(u0, p0)
            ok_, done = s.pisoSteps(ADJ_STEPS)
            if not ok_:
                raise SystemExit(f"FD forward run failed after {done} steps")
            return s.objective(**ADJ_PATCH)

        t0 = time.perf_counter()
        adj, fd = [], []
        for i in nodes:
            pp, pm = prof.copy(), prof.copy()
            pp[i, 0] += h
            pm[i, 0] -= h
            fd.append((J_of(pp) - J_of(pm)) / (2 * h))
            adj.append(float(g["grad_inlet"][i, 0]))
        hn = h * FLUID[1]
        fdn = (J_of(prof, FLUID[1] + hn) - J_of(prof, FLUID[1] - hn)) / (2 * hn)
        adj_a, fd_a = np.array(adj), np.array(fd)
        big = np.abs(fd_a) >= 1e-3 * np.abs(fd_a).max()
        res["fd_check"] = {
            "nodes": nodes, "p1_nodes": int(sum(1 for i in nodes if i < nv)), "h": h,
            "seed": f"std::mt19937_64({ADJ_SEED}) draws modulo the inlet-node count",
            "rel_err_vector": float(np.linalg.norm(adj_a - fd_a) / np.linalg.norm(fd_a)),
            "rel_err_max_significant": float(np.max(np.abs(adj_a[big] - fd_a[big]) / np.abs(fd_a[big]))),
            "rel_err_viscosity": abs(g["grad_viscosity"] - fdn) / abs(fdn),
            "adjoint": adj, "fd": fd, "fd_viscosity": fdn, "fd_seconds": time.perf_counter() - t0,
        }
        res["ok"] = bool(res["fd_check"]["rel_err_vector"] <= 1e-5 and res["fd_check"]["rel_err_viscosity"] <= 1e-5)
    else:
        res["ok"] = True
    del s
    return res


Y_CELL = 0.081  # Kuhn lattice edge of the Y-bifurcation: ~4M tets (mean volume ~1e-4)


def ybif_section(cf, args, barrier, peak):
    """The ~4M-tet Y-bifurcation (parent R=2 L=15, daughters R=1.5 L=12 at +-35 deg, blend 0.5),
    ~4M tets, parabolic inlet peak 1.0, both outlets p=0, from rest; FP64 and mixed-precision
    forward runs (Jacobi-scaled criterion, tol 1e-10) over `--y-steps` steps (the configuration
    names 100; the default budget keeps the whole benchmark within minutes), the pressure solve's
    achieved bandwidth where its operator no longer fits in L2, then the mixed-precision
    forward/backward pair of the pressure-drop objective differentiated with respect to the inlet
    profile, checkpointing every `--y-checkpoint` steps."""
    t0 = time.perf_counter()
    m = cf.Mesh.yBifurcation(cell=args.y_cell)
    mesh_s = time.perf_counter() - t0
    nv, nt, ne, _, _ = m.sizes
    prof = cf.parabolic_inlet(m.nodePositions(), INLET_PEAK, 2.0)
    p1, p2 = m.fluidBC()
    n = args.y_steps

    def solver(precision):
        return make_solver_with(cf, m, prof, tol=TOL, norm=cf.NORM_JACOBI, precision=precision)

    out = {"workload": f"Y-bifurcation, mixed precision and adjoint: {nt} tets, N2={nv + ne}, nv={nv} (Kuhn lattice cell "
                       f"{args.y_cell}); {n} steps from rest (budget; the configuration names 100), parabolic "
                       f"inlet peak 1.0, both outlets p=0, Krylov tol {TOL:g} Jacobi-scaled, two-level CG pressure",
           "tets": nt, "p2_nodes": nv + ne, "pressure_dofs": nv, "inlet_vertices": int((p1 == 1).sum()),
           "outlet_vertices": int((p1 == 2).sum()), "mesh_seconds": mesh_s, "steps": n}
    res = {}
    for name, prec in (("fp64", cf.PRECISION_FP64), ("mixed", cf.PRECISION_MIXED)):
        s = solver(prec)
        barrier()
        ok, done = s.pisoSteps(n)
        st = s.stats()
        barrier()
        res[name] = dict(ok=bool(ok), steps=done, ms=st["last_step_ms"], u=s.getVelocity().copy(),
                         p=s.getPressure().copy(),
                         iters=[st["krylov_iters"][0] / max(done, 1), st["krylov_iters"][1] / max(done, 1)],
                         phase_ms=st["phase_ms"])
        if name == "fp64":
            ms, by = s.profileKernel(cf.KERNEL_PRESSURE_SOLVE, 3)
            gbs = by / (ms * 1e-3) / 1e9
            out["pressure_cg_solve"] = {
                "avg_ms": ms, "alg_bytes": by, "achieved_gbs": gbs, "frac_of_peak": gbs / peak,
                "iterations": s.stats()["pressure_iters"],
                "note": "whole two-level CG solve in one resident kernel; Poisson operator of "
                        f"{nv} rows does not fit in the 126 MB L2 together with its vectors"}
        del s
        import torch

        torch.cuda.empty_cache()
    for name in ("fp64", "mixed"):
        r = res[name]
        out[name] = {"ok": r["ok"], "steps_per_s": r["steps"] / (r["ms"] / 1e3), "ms_per_step": r["ms"] / max(r["steps"], 1),
                     "krylov_iters_per_step": r["iters"], "phase_ms_last_step": r["phase_ms"],
                     "dof_updates_per_s": (3 * (nv + ne) + nv) * r["steps"] / (r["ms"] / 1e3)}
    out["mixed_speedup_vs_fp64"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    out["rel_l2_mixed_vs_fp64"] = {"u": rel_l2(res["mixed"]["u"], res["fp64"]["u"]),
                                   "p": rel_l2(res["mixed"]["p"], res["fp64"]["p"])}
    # adjoint (mixed-precision forward and adjoint solves)
    s = solver(cf.PRECISION_MIXED)
    barrier()
    ok = s.adjointForward(n, args.y_checkpoint)
    g = s.adjointBackward(kind=cf.OBJECTIVE_PRESSURE_DROP) if ok else None
    barrier()
    if g is not None:
        ast_ = s.adjointStats()
        inl = np.concatenate([p1, p2]) == 1
        out["adjoint"] = {"ok": True, "J_pressure_drop": g["J"], "forward_ms": ast_["forward_ms"],
                          "backward_ms": ast_["backward_ms"], "recomputed_steps": ast_["recomputed_steps"],
                          "checkpoints": ast_["checkpoints"], "record_gb": ast_["record_bytes"] / 2**30,
                          "adjoint_krylov_iters": [ast_["momentum_iters"], ast_["pressure_iters"]],
                          "grad_inlet_axial_l2": float(np.linalg.norm(g["grad_inlet"][inl, 0])),
                          "grad_viscosity": g["grad_viscosity"],
                          "steps_per_s_forward_plus_backward": n / ((ast_["forward_ms"] + ast_["backward_ms"]) / 1e3)}
    else:
        out["adjoint"] = {"ok": False}
    del s
    return out


def oracle_cylinder(rings, layers, pressure_solver):
    """Oracle (test infrastructure) set up on the benchmark workload from its own mesher, so that
    a CPU-only run maps no product library: the 999,936-tet cylinder with the parabolic inlet."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po

    xyz, tets = po.cylinder(GEOM["length"], GEOM["radius"], rings, layers)
    o = po.Oracle(xyz, tets)
    o.set_fluid(*FLUID)
    o.set_params(dt=DT, tol_mom=TOL, tol_p=TOL, maxit_mom=MAXIT[0], maxit_p=MAXIT[1],
                 pressure_solver=pressure_solver)
    o.initialize()
    o.set_inlet(po.parabolic_inlet(o, INLET_PEAK, GEOM["radius"]))
    return po, o


def time_oracle_steps(po, o, threads, nsteps, budget_s):
    """Wall time of up to `nsteps` oracle PISO steps on `threads` host threads, stopping early
    once `budget_s` seconds of steps have run. Returns (steps done, seconds, threads used)."""
    cores = po.set_threads(threads)
    done, t0 = 0, time.perf_counter()
    while done < nsteps:
        if o.piso_step() != 0:
            break
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    return done, time.perf_counter() - t0, cores


def cpu_baseline(rings, layers, n_threads, steps=5, budget_s=30.0):
    """Oracle port of the reference algorithm (BiCGSTAB pressure and momentum) timed on the host
    cores: steps 2.. of the same workload from rest (set-up and the first step untimed), up to
    `steps` steps or `budget_s` seconds, all host threads."""
    po, o = oracle_cylinder(rings, layers, pressure_solver=0)
    po.set_threads(n_threads)
    if o.piso_step() != 0:
        return None
    done, el, cores = time_oracle_steps(po, o, n_threads, steps, budget_s)
    if done == 0:
        return None
    return {"value": done / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} PISO steps (steps 2-{done + 1} from rest) of the {o.nt}-tet workload, {el:.1f} s, "
                      f"FP64 oracle port of the reference algorithm (BiCGSTAB pressure and momentum) "
                      f"with OpenMP on {cores} threads"}


def max_over_ranks(value: float, dist, device: str = "cuda") -> float:
    """The largest value over all ranks (times are reported as the slowest rank's); `dist` is
    torch.distributed or None for a single process."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    """The reference arm: the reference algorithm (oracle port, BiCGSTAB pressure and momentum)
    on the host cores, on the same workload, metric and unit as the GPU arm. It builds its mesh
    with the oracle's own mesher and loads no product library. All host threads over the
    requested steps (after the same warm-up steps as the GPU arm), then the same solver on one
    thread over `--reference-single-core-steps` steps, as the reference itself runs (its build has
    no OpenMP and Eigen's sparse products are serial)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    warm = max(args.warmup, 3)
    po, o = oracle_cylinder(args.rings, args.layers, pressure_solver=0)
    cores = po.set_threads(os.cpu_count() or 1)
    for _ in range(warm):
        o.piso_step()
    done, el, cores = time_oracle_steps(po, o, os.cpu_count() or 1, args.steps, args.reference_budget_s)
    value = done / el if el > 0 else 0.0
    one = None
    if args.reference_single_core_steps > 0:
        d1, e1, c1 = time_oracle_steps(po, o, 1, args.reference_single_core_steps, args.reference_budget_s)
        one = {"value": d1 / e1 if e1 > 0 else 0.0, "unit": UNIT, "cores": c1, "steps": d1,
               "sample": f"{d1} PISO steps right after the all-thread ones, same solver on 1 thread"}
    sample = (f"{done} of {args.steps} requested PISO steps after {warm} warm-up steps from rest, FP64 "
              f"oracle port of the reference algorithm (BiCGSTAB pressure and momentum) with OpenMP on "
              f"{cores} threads, capped at {args.reference_budget_s:.0f} s of timed work")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": done, "warmup": warm,
            "ms_per_step": 1e3 * el / max(done, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": workload_desc((o.nv, o.nt, o.ne), args.rings, args.layers, world),
            "solver": REF_SOLVER,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                             "single_core": one},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def rel_l2(a, b) -> float:
    from numpy.linalg import norm

    nb = norm(b)
    return float(norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def trajectory(cf, m, profile, precision, tol, norm, marks, momentum=None):
    """A solver from rest: device ms over all steps and (u, p, per-step stats) at each mark."""
    s = make_solver_with(cf, m, profile, tol=tol, norm=norm, precision=precision, momentum=momentum)
    out, ms, done, ok = {}, 0.0, 0, True
    iters, upd = [0, 0], 0
    for k in marks:
        good, n = s.pisoSteps(k - done)
        st = s.stats()
        ok = ok and good and n == k - done
        ms += st["last_step_ms"]
        iters = [iters[0] + st["krylov_iters"][0], iters[1] + st["krylov_iters"][1]]
        done = k
        out[k] = (s.getVelocity().copy(), s.getPressure().copy(), st)
    del s
    return out, ms, ok, iters


def make_solver_with(cf, m, profile, tol=TOL, norm=0, precision=0, momentum=None):
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(tol, tol)
    s.setConvergenceNorm(norm)
    s.setMaxIterations(*MAXIT)
    s.setPressureSolver(cf.KRYLOV_CG2L)
    s.setPrecision(precision)
    s.setMomentumSolver(MOMENTUM[momentum or MOMENTUM_SOLVER])
    s.setDt(DT)
    s.initialize(m, cf.Fluid(*FLUID))
    s.setInletVelocityProfile(profile)
    return s


def mixed_section(cf, m, profile, marks):
    """Mixed precision on the headline mesh and inputs: FP64 and mixed precision (the headline's momentum
    Krylov method in FP32 with FP64 reliable updates) from rest over marks[-1] steps, both under the Jacobi-scaled criterion at
    1e-10 (the reference's criterion is dominated by the 1e10 penalty rows and pins the interior
    only loosely), and an FP64 run at 1e-14 in the same norm as the converged solution; fields at
    every mark. Both paths run the two-level CG pressure solve in FP64."""
    J = cf.NORM_JACOBI
    f64, f_ms, f_ok, f_it = trajectory(cf, m, profile, cf.PRECISION_FP64, TOL, J, marks)
    mix, m_ms, m_ok, m_it = trajectory(cf, m, profile, cf.PRECISION_MIXED, TOL, J, marks)
    full, x_ms, x_ok, x_it = trajectory(cf, m, profile, cf.PRECISION_MIXED_FULL, TOL, J, marks)
    conv, _, c_ok, _ = trajectory(cf, m, profile, cf.PRECISION_FP64, 1e-14, J, marks)
    n = marks[-1]
    mom = "Jacobi CG" if MOMENTUM_SOLVER == "cg" else "BiCGSTAB"
    res = {"workload": f"mixed precision on the headline mesh and inputs, {n} steps from rest; momentum {mom} with FP32 "
                       f"operator and Krylov vectors and FP64 reliable updates (true residual, solution, dots) vs "
                       f"FP64 {mom}; two-level CG pressure in FP64 in both (CFSA_PRECISION_MIXED); "
                       f"Jacobi-scaled criterion 1e-10",
           "ok": bool(f_ok and m_ok and c_ok), "steps": n,
           "value": n / (m_ms / 1e3), "unit": UNIT, "fp64_value": n / (f_ms / 1e3),
           "speedup_vs_fp64": f_ms / m_ms, "ms_per_step": m_ms / n, "fp64_ms_per_step": f_ms / n,
           "krylov_iters_per_step": {"mixed": [m_it[0] / n, m_it[1] / n], "fp64": [f_it[0] / n, f_it[1] / n]},
           "mixed_full": {
               "what": "also the pressure in float storage: two-level CG inside FP64 defect correction "
                       "(CFSA_PRECISION_MIXED_FULL); each sweep restarts the CG",
               "ok": bool(x_ok), "value": n / (x_ms / 1e3), "speedup_vs_fp64": f_ms / x_ms,
               "krylov_iters_per_step": [x_it[0] / n, x_it[1] / n],
               "vs_fp64_at_last_step": {"u": rel_l2(full[n][0], f64[n][0]), "p": rel_l2(full[n][1], f64[n][1])},
               "vs_converged_at_last_step": {"u": rel_l2(full[n][0], conv[n][0]), "p": rel_l2(full[n][1], conv[n][1])}},
           "at_step": {}}
    for k in marks:
        res["at_step"][str(k)] = {
            "mixed_vs_fp64": {"u": rel_l2(mix[k][0], f64[k][0]), "p": rel_l2(mix[k][1], f64[k][1])},
            "mixed_vs_converged": {"u": rel_l2(mix[k][0], conv[k][0]), "p": rel_l2(mix[k][1], conv[k][1])},
            "fp64_vs_converged": {"u": rel_l2(f64[k][0], conv[k][0]), "p": rel_l2(f64[k][1], conv[k][1])},
            "momentum_iters": {"mixed": mix[k][2]["momentum_iters"], "fp64": f64[k][2]["momentum_iters"]},
            "reliable_updates": mix[k][2]["momentum_outer"],
            "pressure_iters": mix[k][2]["pressure_iters"],
        }
    if MOMENTUM_SOLVER == "cg":
        # the same comparison with the reference's momentum method (BiCGSTAB in both precisions)
        bf, bf_ms, bf_ok, bf_it = trajectory(cf, m, profile, cf.PRECISION_FP64, TOL, J, marks, "bicgstab")
        bm, bm_ms, bm_ok, bm_it = trajectory(cf, m, profile, cf.PRECISION_MIXED, TOL, J, marks, "bicgstab")
        res["bicgstab"] = {
            "what": "momentum BiCGSTAB (the reference's method) in both precisions, same pressure and criterion",
            "ok": bool(bf_ok and bm_ok), "value": n / (bm_ms / 1e3), "fp64_value": n / (bf_ms / 1e3),
            "speedup_vs_fp64": bf_ms / bm_ms, "ms_per_step": bm_ms / n, "fp64_ms_per_step": bf_ms / n,
            "krylov_iters_per_step": {"mixed": [bm_it[0] / n, bm_it[1] / n], "fp64": [bf_it[0] / n, bf_it[1] / n]},
            "mixed_vs_fp64": {str(k): {"u": rel_l2(bm[k][0], bf[k][0]), "p": rel_l2(bm[k][1], bf[k][1])} for k in marks},
            "mixed_vs_converged": {str(k): {"u": rel_l2(bm[k][0], conv[k][0]), "p": rel_l2(bm[k][1], conv[k][1])}
                                   for k in marks}}
    first = marks[0]
    return res, {"mixed": mix[first][:2], "fp64": f64[first][:2]}


def cpu_section(args, gpu_headline, gpu_step1_jacobi):
    """Everything the oracle (test infrastructure) does in the GPU arm, on one oracle instance of
    the headline workload, after the GPU sections: (1) parity of the headline FP64 path, the same
    solver (two-level CG pressure, same coarse target, reference criterion 1e-10) from rest, at
    steps 1 and 3; (2) the mixed-precision section's CPU comparison, FP64 in the Jacobi-scaled
    criterion, step 1;
    (3) the timed CPU baseline, the reference algorithm (BiCGSTAB pressure) on all host threads."""
    po, o = oracle_cylinder(args.rings, args.layers, pressure_solver=3)
    o.set_momentum_solver(1 if MOMENTUM_SOLVER == "cg" else 0)
    threads = po.set_threads(os.cpu_count() or 1)
    zero_u, zero_p = np.zeros((o.N2, 3)), np.zeros(o.nv)
    mom = "Jacobi CG" if MOMENTUM_SOLVER == "cg" else "BiCGSTAB"
    parity = {"workload": f"headline FP64 step (two-level CG pressure, {mom} momentum, reference criterion 1e-10) "
                          "from rest, GPU vs the oracle on the same mesh and inputs", "at_step": {}}
    t0 = time.perf_counter()
    for k in (1, 2, 3):
        if o.piso_step() != 0:
            parity["ok"] = False
            break
        if k in gpu_headline:
            st = o.state()
            gu, gp = gpu_headline[k]
            parity["at_step"][str(k)] = {"u": rel_l2(gu, st["u"]), "p": rel_l2(gp, st["p"]),
                                         "bit_exact": bool(np.array_equal(gu, st["u"]) and np.array_equal(gp, st["p"]))}
    parity.setdefault("ok", all(v["u"] <= 1e-8 and v["p"] <= 1e-8 for v in parity["at_step"].values()))
    parity["oracle_seconds"] = time.perf_counter() - t0
    parity["oracle_threads"] = threads
    mixed_cpu = None
    if gpu_step1_jacobi is not None:
        o.set_state(zero_u, zero_p)
        o.set_params(dt=DT, tol_mom=TOL, tol_p=TOL, maxit_mom=MAXIT[0], maxit_p=MAXIT[1], pressure_solver=3,
                     conv_norm=1)
        o.set_momentum_solver(1 if MOMENTUM_SOLVER == "cg" else 0)  # the mixed-precision section's FP64 path
        if o.piso_step() == 0:
            st = o.state()
            mixed_cpu = {"reference": "FP64 oracle (CPU), Jacobi-scaled criterion 1e-10, step 1 from rest"}
            for name, (gu, gp) in gpu_step1_jacobi.items():
                mixed_cpu[name] = {"u": rel_l2(gu, st["u"]), "p": rel_l2(gp, st["p"])}
    cpu = None
    if not args.no_cpu_baseline:
        o.set_state(zero_u, zero_p)
        o.set_params(dt=DT, tol_mom=TOL, tol_p=TOL, maxit_mom=MAXIT[0], maxit_p=MAXIT[1], pressure_solver=0)
        o.set_momentum_solver(0)  # the reference algorithm
        if o.piso_step() == 0:
            done, el, cores = time_oracle_steps(po, o, os.cpu_count() or 1, 5, 30.0)
            if done:
                cpu = {"value": done / el, "unit": UNIT, "cores": cores, "kind": "port",
                       "sample": f"{done} PISO steps (steps 2-{done + 1} from rest) of the {o.nt}-tet workload, "
                                 f"{el:.1f} s, FP64 oracle port of the reference algorithm (BiCGSTAB pressure and "
                                 f"momentum) with OpenMP on {cores} threads"}
    return parity, mixed_cpu, cpu


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import cfsa_b200 as cf

    global MOMENTUM_SOLVER
    MOMENTUM_SOLVER = args.momentum_solver
    m = make_mesh(cf, args.rings, args.layers)
    s, profile = make_solver(cf, m)
    nv, nt, ne, _, _ = m.sizes
    N2 = nv + ne
    warm = max(args.warmup, 3)

    # warm-up from rest; its steps 1 and 3 are kept for the parity check against the oracle
    headline_states = {}
    done = 0
    for k in (1, 3, warm):
        if k == done:
            continue
        ok, n = s.pisoSteps(k - done)
        if not ok:
            raise SystemExit(f"warm-up failed at step {done + n}: {s.stats()}")
        done = k
        headline_states.setdefault(k, (s.getVelocity().copy(), s.getPressure().copy()))
    headline_states = {k: v for k, v in headline_states.items() if k in (1, 3)}
    # the end-to-end loop and the accuracy check below replay the timed steps from this state
    import tempfile
    snap = os.path.join(tempfile.gettempdir(), f"cfsa_bench_state_{os.getpid()}.bin")
    s.saveState(snap)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    clocks = ClockSampler()
    barrier()
    if rank == 0:
        clocks.start()
    ok, done = s.pisoSteps(args.steps)  # device-timed with CUDA events on the solver's stream
    st = s.stats()
    barrier()
    clk = clocks.stop(set(range(world))) if rank == 0 else None
    if not ok:
        raise SystemExit(f"timed steps failed after {done} steps: {st}")
    ms_total = st["last_step_ms"]
    ms_max = max_over_ranks(ms_total, dist)
    value = world * args.steps / (ms_max / 1e3)
    timed_u, timed_p = s.getVelocity().copy(), s.getPressure().copy()

    # end to end through the public API with host buffers: per step upload the inlet profile
    # (H2D), pisoStep, read back u and p (D2H); the host buffers are pinned, as an application
    # streaming fields every step would hold them. Same steps as the timed loop (restored state).
    s.loadState(snap)
    prof_host = torch.empty(profile.shape, dtype=torch.float64, pin_memory=True).numpy()
    prof_host[:] = profile
    u_host = torch.empty((s.N2, 3), dtype=torch.float64, pin_memory=True).numpy()
    p_host = torch.empty((s.nv,), dtype=torch.float64, pin_memory=True).numpy()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.setInletVelocityProfile(prof_host)
        if not s.pisoStep():
            raise SystemExit("e2e step failed")
        # stream-ordered read-back: each step's u and p are copied to the pinned host arrays while
        # the next step computes; the last copies are waited for inside the timed region
        s.getVelocityAsync(u_host)
        s.getPressureAsync(p_host)
    s.waitOutputs()
    barrier()
    e2e_s = time.perf_counter() - t0
    # the e2e loop replays the device-timed steps from the same state: same fields, bit for bit
    e2e_match = bool(np.array_equal(u_host, timed_u) and np.array_equal(p_host, timed_p))
    e2e_value = world * args.steps / max_over_ranks(e2e_s, dist)

    # roofline of the step's kernels on live data (CUDA events on the solver's stream)
    peak, peak_kind = measured_peak()
    traffic = traffic_table()
    kernels = {}
    products = 1 if MOMENTUM_SOLVER == "cg" else 2  # momentum products per Krylov iteration
    for name, which, per_step in (("momentum_spmv_3rhs", cf.KERNEL_MOMENTUM_SPMV, products * st["krylov_iters"][0]),
                                  ("pressure_cg_solve", cf.KERNEL_PRESSURE_SOLVE, args.steps),
                                  ("momentum_spmv_3rhs_f32", cf.KERNEL_MOMENTUM_SPMV_F32, 0)):
        ms, by = s.profileKernel(which, 3 if which == cf.KERNEL_PRESSURE_SOLVE else 20)
        gbs = by / (ms * 1e-3) / 1e9
        kernels[name] = {"avg_ms": ms, "alg_bytes": by, "achieved_gbs": gbs, "frac_of_peak": gbs / peak,
                         "launches_timed_region": int(per_step),
                         "time_share_est": None, "traffic": traffic.get(name)}
    kernels["momentum_spmv_3rhs_f32"]["note"] = (
        "the FP32 product of the mixed-precision momentum solve, all three components active; "
        "not part of the FP64 headline step")
    kernels["pressure_cg_solve"]["note"] = (
        "one launch = one whole two-level CG solve (fused product, coarse correction and vector updates "
        "in one resident kernel); alg_bytes = iterations x per-iteration bytes; the 1M-tet Poisson operator "
        "and vectors (~50 MB) stay in the 126 MB L2, so this rate is L2-served, not HBM")
    total_ms = ms_max
    for k in kernels.values():
        k["time_share_est"] = k["avg_ms"] * k["launches_timed_region"] / total_ms
    dom_name = max(kernels, key=lambda k: kernels[k]["time_share_est"])
    dom = kernels[dom_name]
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": dom["achieved_gbs"], "peak": peak,
                "unit": "GB/s", "frac": dom["achieved_gbs"] / peak, "peak_kind": peak_kind,
                "traffic": dom["traffic"],
                "traffic_note": "scaled, not measured on this workload: ncu dram__bytes_read.sum + write.sum of "
                                "the momentum product captured at 414,720 tets (k_mcg_q<3>), times the ratio of "
                                "algorithmic bytes per launch (profiles/dram_traffic.json)"}

    # accuracy of the headline itself: the timed steps again from the same state with the Krylov
    # solves converged (1e-14 in the Jacobi-scaled criterion, which sees the interior rows)
    s.loadState(snap)
    os.remove(snap)
    s.setConvergenceNorm(cf.NORM_JACOBI)
    s.setKrylovTolerances(1e-14, 1e-14)
    ok_c, _ = s.pisoSteps(args.steps)
    headline_accuracy = {
        "reference": "same steps from the same state, FP64, Krylov tol 1e-14 in the Jacobi-scaled criterion",
        "ok": bool(ok_c), "u": rel_l2(timed_u, s.getVelocity()), "p": rel_l2(timed_p, s.getPressure()),
        "note": "the reference's criterion ||r|| <= 1e-10 ||b|| is dominated by the 1e10 penalty rows, so the "
                "interior is solved loosely at the headline tolerance; this is the headline's own error"}
    del s
    torch.cuda.empty_cache()
    momentum_bicgstab = None
    if MOMENTUM_SOLVER == "cg":
        momentum_bicgstab = bicgstab_headline(cf, m, args.steps, warm, world)
        torch.cuda.empty_cache()

    mixed, step1 = None, None
    if not args.no_mixed:
        marks = [int(x) for x in args.mixed_marks.split(",")]
        mixed, step1 = mixed_section(cf, m, profile, marks)
        torch.cuda.empty_cache()

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_section(cf, args, barrier)
        torch.cuda.empty_cache()

    ybif = None
    if not args.no_y_bifurcation:
        ybif = ybif_section(cf, args, barrier, peak)
        torch.cuda.empty_cache()

    parity, cpu = None, None
    if rank == 0 and world == 1 and not args.no_oracle:
        parity, mixed_cpu, cpu = cpu_section(args, headline_states, step1)
        if mixed is not None:
            mixed["vs_cpu_oracle_step1"] = mixed_cpu

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA,
            "config": workload_desc((nv, nt, ne), args.rings, args.layers, world),
            "solver": gpu_solver_label(),
            "dof_updates_per_s": value * (3 * N2 + nv),
            "krylov_iters_per_step": [st["krylov_iters"][0] / args.steps, st["krylov_iters"][1] / args.steps],
            "gpu_launches": int(st["kernel_launches"]),
            "phase_ms_last_step": {"momentum": st["phase_ms"][0], "pressure_solve": st["phase_ms"][1],
                                   "other": st["phase_ms"][2]},
            "roofline": roofline, "kernels": kernels,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(profile.nbytes),
                    "d2h_bytes_per_step": int(u_host.nbytes + p_host.nbytes),
                    "readback": "stream-ordered (cfsa_ns_get_velocity_async / _pressure_async): each step's "
                                "fields copy to pinned host arrays while the next step computes",
                    "fields_match_device_timed": e2e_match},
            "cpu_baseline": cpu, "clocks": clk, "parity": parity, "headline_accuracy": headline_accuracy,
            "momentum_bicgstab": momentum_bicgstab,
            "mixed": mixed, "adjoint": adjoint, "y_bifurcation": ybif,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
