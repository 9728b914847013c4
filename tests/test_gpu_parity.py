"""GPU solver (libcfsa.so, sm_100a) against the CPU oracle on identical meshes and inputs.

Bars: assembly, element operators and forces are bit-exact (same arithmetic order, no FMA).
PISO states must agree to relative L2 <= 1e-8 in FP64 (the stated tolerance); because the oracle
reduces its Krylov dot products in the device's fixed tree, FP64 trajectories are in fact
bit-identical, which test_trajectory_bit_exact and the config-0 run check explicitly.
"""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"

RHO, NU = 1060.0, 0.004  # config-0 fluid


def make_mesh(cf, rings=3, layers=12, length=30.0, radius=2.0):
    m = cf.Mesh.cylinder(length, radius, rings, layers)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    return m


def make_pair(cf, po, m, *, tol=1e-12, krylov=0, dt=0.01, inlet=0.5, profile=None, ncorr=1,
              relax=(1.0, 1.0), outlet=0, outlet_p=0.0, maxit=(5000, 20000), norm=0, mom_cg=False):
    """GPU solver and oracle configured identically (the reference's CLI order: initialize with
    a zero inlet, then set the inlet)."""
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(tol, tol)
    s.setMaxIterations(*maxit)
    s.setPressureSolver(krylov)
    s.setDt(dt)
    s.setNumberOfCorrections(ncorr)
    s.setRelaxU(relax[0])
    s.setRelaxP(relax[1])
    s.setOutletType(outlet)
    s.setConvergenceNorm(norm)
    if mom_cg:
        s.setMomentumSolver(cf.KRYLOV_CG)
    s.initialize(m, cf.Fluid(RHO, NU))
    s.setOutletPressure(outlet_p)
    o = po.Oracle(m.vertices(), m.tets())
    o.set_fluid(RHO, NU)
    o.set_params(dt=dt, tol_mom=tol, tol_p=tol, maxit_mom=maxit[0], maxit_p=maxit[1],
                 n_corr=ncorr, relax_u=relax[0], relax_p=relax[1], outlet_type=outlet,
                 outlet_pressure=outlet_p, reference_node=s.reference_node,
                 pressure_solver={0: 1, 1: 0, 2: 2, 3: 3}[krylov], conv_norm=norm)
    if mom_cg:
        o.set_momentum_solver(1)
    o.initialize()
    if profile is not None:
        s.setInletVelocityProfile(profile)
        o.set_inlet(profile)
    else:
        s.setMeanInletVelocity([inlet, 0.0, 0.0])
        v = np.zeros((o.N2, 3))
        v[:, 0] = inlet
        o.set_inlet(v)
    return s, o


def csr_equal(a, b):
    return (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]))


@pytest.fixture(scope="module")
def small(cf, po):
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m)
    return m, s, o


@pytest.mark.parametrize("which,name", [(0, "M"), (1, "K"), (2, "Gx"), (3, "Gy"), (4, "Gz"), (5, "L")])
def test_assembly_bit_exact(small, which, name):
    m, s, o = small
    g = s.matrix(which)
    r = o.matrix(name)
    assert csr_equal(g, r), name


def test_assembly_bit_exact_structured_prism(cf, po):
    m = cf.Mesh.structuredRectangularPrism(3.0, 1.0, 1.0, 6, 2, 2)
    m.setupBoundaryConditions()
    s, o = make_pair(cf, po, m)
    for which, name in [(0, "M"), (1, "K"), (2, "Gx"), (5, "L")]:
        assert csr_equal(s.matrix(which), o.matrix(name)), name
    assert np.array_equal(s.invLumpedMass(), o.inv_lumped_mass())


def test_lumped_mass_bit_exact(small):
    m, s, o = small
    assert np.array_equal(s.invLumpedMass(), o.inv_lumped_mass())


def test_operators_bit_exact(small, cf):
    m, s, o = small
    rng = np.random.default_rng(1)
    u = rng.standard_normal((s.N2, 3))
    p = rng.standard_normal(s.nv)
    s.setFields(u, p)
    o.set_state(u, p)
    assert np.array_equal(s.computeAdvectionRHS(), o.advection())
    assert np.array_equal(s.computeDivergence(u), o.divergence(u))


def test_forces_bit_exact(small):
    m, s, o = small
    rng = np.random.default_rng(2)
    u = rng.standard_normal((s.N2, 3))
    p = rng.standard_normal(s.nv)
    s.setFields(u, p)
    o.set_state(u, p)
    assert np.array_equal(s.computePressureForces(), o.pressure_forces())
    assert np.array_equal(s.computeShearStress(), o.shear_stress())
    tot = s.computeTotalFluidForces()
    np.testing.assert_allclose(tot, o.pressure_forces() + o.shear_stress(), rtol=0, atol=0)


def run_both(s, o, steps):
    states = []
    for _ in range(steps):
        assert s.pisoStep()
        assert o.piso_step() == 0
        states.append((s.getVelocity(), s.getPressure(), o.state()))
    return states


@pytest.mark.parametrize("krylov", [0, 1, 2, 3], ids=["cg", "bicgstab", "cg1", "cg2l"])
def test_piso_parity_tight(cf, po, krylov):
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-13, krylov=krylov)
    for u, p, st in run_both(s, o, 5):
        assert rel_l2(u, st["u"]) < 1e-8
        assert rel_l2(p, st["p"]) < 1e-8
    assert abs(s.getTime() - st["time"]) == 0.0


def test_piso_matches_golden_fixture(cf):
    g = np.load(GOLD / "cyl_piso.npz")
    m = cf.Mesh.cylinder(30.0, 2.0, 2, 4)
    m.setupBoundaryConditions()
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(1e-14, 1e-14)
    s.setMaxIterations(5000, 5000)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(RHO, NU))
    s.setMeanInletVelocity([0.5, 0.0, 0.0])
    for k in range(3):
        assert s.pisoStep()
        assert rel_l2(s.getVelocity(), g["u"][k]) < 1e-8
        assert rel_l2(s.getPressure(), g["p"][k]) < 1e-8
        assert rel_l2(s.getPressureCorrection(), g["pcorr"][k]) < 1e-8


def test_cylinder_30k_parity_100_steps(cf, po):
    """The reference-runnable case: cylinder L=30 R=2 (~30k tets), rho 1060, nu 0.004, plug inlet 0.5, p=0 outlet,
    dt 0.01, 100 steps from rest, Krylov tolerance 1e-10 (CG pressure on both sides)."""
    m = make_mesh(cf, 5, 68)
    assert 29000 < m.nTets() < 32000
    s, o = make_pair(cf, po, m, tol=1e-10, krylov=cf.KRYLOV_CG)
    for k in range(100):
        assert s.pisoStep(), k
        assert o.piso_step() == 0, k
    st = o.state()
    eu, ep = rel_l2(s.getVelocity(), st["u"]), rel_l2(s.getPressure(), st["p"])
    print(f"30k-tet cylinder, 100 steps: rel L2 u {eu:.3e} p {ep:.3e}")
    assert eu < 1e-8 and ep < 1e-8
    assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"])


def test_reference_default_tolerances(cf, po):
    """The reference's own solver settings: BiCGSTAB pressure, tolerances 1e-6 / 1e-8, 1000
    iterations. Same iteration counts as the oracle and states within 1e-8."""
    m = make_mesh(cf, 3, 12)
    s = cf.NavierStokesSolver()
    s.setPressureSolver(cf.KRYLOV_BICGSTAB)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(RHO, NU))
    s.setMeanInletVelocity([0.5, 0.0, 0.0])
    o = po.Oracle(m.vertices(), m.tets())
    o.set_fluid(RHO, NU)
    o.set_params(dt=0.01)
    o.initialize()
    v = np.zeros((o.N2, 3))
    v[:, 0] = 0.5
    o.set_inlet(v)
    for _ in range(4):
        assert s.pisoStep() and o.piso_step() == 0
        gs, os_ = s.stats(), o.stats()
        assert gs["momentum_iters"] == os_["momentum_iters"]
        assert gs["pressure_iters"] == os_["pressure_iters"]
    assert rel_l2(s.getVelocity(), o.state()["u"]) < 1e-8
    assert rel_l2(s.getPressure(), o.state()["p"]) < 1e-8


@pytest.mark.parametrize("case", ["neumann", "two_correctors", "relaxed", "parabolic", "outlet_p",
                                  "neumann_cg2l", "neumann_momentum_cg", "two_correctors_relaxed_momentum_cg"])
def test_variants_parity(cf, po, case):
    m = make_mesh(cf, 3, 12)
    kw = dict(tol=1e-13)
    if case == "neumann_cg2l":
        kw.update(outlet=1, krylov=cf.KRYLOV_CG2L)
    elif case == "neumann_momentum_cg":
        kw.update(outlet=1, krylov=cf.KRYLOV_CG2L, mom_cg=True)
    elif case == "two_correctors_relaxed_momentum_cg":
        kw.update(ncorr=2, relax=(0.7, 0.6), krylov=cf.KRYLOV_CG2L, mom_cg=True)
    if case == "neumann":
        kw.update(outlet=1)
    elif case == "two_correctors":
        kw.update(ncorr=2)
    elif case == "relaxed":
        kw.update(relax=(0.5, 0.5))
    elif case == "parabolic":
        kw.update(profile=cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0))
    elif case == "outlet_p":
        kw.update(outlet_p=10.0)
    s, o = make_pair(cf, po, m, **kw)
    if case.startswith("neumann"):
        assert s.reference_node >= 0 and o.reference_node() == s.reference_node
    for u, p, st in run_both(s, o, 3):
        assert rel_l2(u, st["u"]) < 1e-8, case
        assert rel_l2(p, st["p"]) < 1e-8, case


def test_simple_step_parity(cf, po):
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-13)
    for _ in range(3):
        assert s.simpleStep()
        assert o.simple_step() == 0
    st = o.state()
    assert rel_l2(s.getVelocity(), st["u"]) < 1e-8
    assert rel_l2(s.getPressure(), st["p"]) < 1e-8


def test_phase_api_equals_step(cf, po):
    """solveMomentumPredictor + solvePressurePoisson + correctVelocity == pisoStep (bit-exact)."""
    m = make_mesh(cf, 3, 12)
    a, _ = make_pair(cf, po, m, tol=1e-12)
    b, _ = make_pair(cf, po, m, tol=1e-12)
    for _ in range(2):
        assert a.pisoStep()
        assert b.solveMomentumPredictor() and b.solvePressurePoisson() and b.correctVelocity()
    assert np.array_equal(a.getVelocity(), b.getVelocity())
    assert np.array_equal(a.getPressure(), b.getPressure())


def test_graph_and_eager_identical_and_deterministic(cf, po):
    m = make_mesh(cf, 3, 12)
    runs = []
    for no_graph in ("0", "1", "0"):
        os.environ["CFSA_NO_GRAPH"] = no_graph
        try:
            s, _ = make_pair(cf, po, m, tol=1e-12)
        finally:
            os.environ.pop("CFSA_NO_GRAPH", None)
        ok, done = s.pisoSteps(4)
        assert ok and done == 4
        runs.append((s.getVelocity(), s.getPressure()))
    for u, p in runs[1:]:
        assert np.array_equal(u, runs[0][0]) and np.array_equal(p, runs[0][1])


def test_batched_steps_equal_single_steps(cf, po):
    m = make_mesh(cf, 3, 12)
    a, _ = make_pair(cf, po, m, tol=1e-12)
    b, _ = make_pair(cf, po, m, tol=1e-12)
    ok, done = a.pisoSteps(5)
    assert ok and done == 5
    for _ in range(5):
        assert b.pisoStep()
    assert np.array_equal(a.getVelocity(), b.getVelocity())
    assert a.getTime() == b.getTime()


@pytest.mark.parametrize("krylov", [0, 3], ids=["cg", "cg2l"])
def test_not_converged_is_reported(cf, po, krylov):
    """maxit = 1 with a tight tolerance: pisoStep returns false, time does not advance (the
    reference returns before time_ += dt, NavierStokes.cpp:387-390)."""
    m = make_mesh(cf, 3, 12)
    s, _ = make_pair(cf, po, m, tol=1e-14, maxit=(1, 1), krylov=krylov)
    assert not s.pisoStep()
    assert s.getTime() == 0.0
    ok, done = s.pisoSteps(3)
    assert not ok and done == 0


@pytest.mark.parametrize("krylov", [0, 3], ids=["cg", "cg2l"])
def test_nan_is_reported(cf, po, krylov):
    """A NaN relaxation factor poisons u in the corrector: the step completes (time advances, as
    in the reference) and pisoStep returns false through the hasNans() check."""
    m = make_mesh(cf, 3, 12)
    s, _ = make_pair(cf, po, m, tol=1e-12, relax=(float("nan"), 1.0), krylov=krylov)
    assert not s.pisoStep()
    assert s.getTime() == pytest.approx(0.01)
    assert np.isnan(s.getVelocity()).any()


@pytest.mark.parametrize("krylov", [0, 3], ids=["cg", "cg2l"])
def test_nan_input_fails_fast(cf, po, krylov):
    m = make_mesh(cf, 3, 12)
    s, _ = make_pair(cf, po, m, tol=1e-12, krylov=krylov)
    p = np.zeros(s.nv)
    p[5] = np.nan
    s.setFields(None, p)
    assert not s.pisoStep()
    st = s.stats()
    assert max(st["momentum_iters"]) <= 1


@pytest.mark.parametrize("krylov", [0, 2, 3], ids=["cg", "cg1", "cg2l"])
def test_grid_barrier_wait_runs_out(cf, po, krylov):
    """The resident pressure solvers wait at grid barriers with a bounded number of polls. With
    the bound at 0 the first CTA to wait gives up: every CTA leaves the kernel, the step reports
    CFSA_CUDA_ERROR through the C ABI (the facade's pisoStep() is false), time does not advance,
    and after the default bound is restored the same handle steps on from the unchanged state
    bit for bit with the oracle's first step. No GPU fault is involved: the wait ends on its own
    and the host reads the status word."""
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-12, krylov=krylov)
    lib = cf.load_library()
    u0, p0 = s.getVelocity().copy(), s.getPressure().copy()
    s.setBarrierSpinLimit(0)
    code = lib.cfsa_ns_piso_step(s._h)
    assert code == cf.CUDA_ERROR
    assert "grid barrier" in lib.cfsa_ns_last_error(s._h).decode()
    assert s.getTime() == 0.0
    assert np.array_equal(s.getVelocity(), u0) and np.array_equal(s.getPressure(), p0)
    s.setBarrierSpinLimit(-1)
    assert s.pisoStep()
    assert o.piso_step() == 0
    st = o.state()
    assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"])
    assert s.getTime() == st["time"]


def test_solve_pressure_bicgstab_matches_oracle(cf, po):
    """solvePressureBiCGSTAB (NavierStokes.cpp:773-802): raw Poisson matrix, no boundary penalty,
    tol 1e-8, maxit 1000, zero guess. A consistent right-hand side (L y) converges; the GPU iterate
    equals the oracle's bit for bit (same reduction tree). An inconsistent one with a small cap
    fails on both sides with the same last iterate. The solver's fields are left unchanged."""
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-12, krylov=1)
    rng = np.random.default_rng(11)
    rp, ci, vals = s.matrix(5)
    L = np.zeros((s.nv, s.nv))
    for i in range(s.nv):
        L[i, ci[rp[i]:rp[i + 1]]] = vals[rp[i]:rp[i + 1]]
    rhs = L @ rng.standard_normal(s.nv)
    u0, p0 = s.getVelocity().copy(), s.getPressure().copy()
    ok, x = s.solvePressureBiCGSTAB(rhs)
    ok_o, x_o, it_o = o.solve_poisson_raw(rhs)
    assert ok and ok_o and it_o > 1
    assert np.array_equal(x, x_o)
    assert np.linalg.norm(L @ x - rhs) <= 1e-8 * np.linalg.norm(rhs) * (1 + 1e-6)
    assert np.array_equal(s.getVelocity(), u0) and np.array_equal(s.getPressure(), p0)
    bad = rng.standard_normal(s.nv)  # not in the range of the singular L: stays unconverged
    ok, x = s.solvePressureBiCGSTAB(bad, maxit=5)
    ok_o, x_o, it_o = o.solve_poisson_raw(bad, maxit=5)
    assert not ok and not ok_o and it_o == 5
    assert np.array_equal(x, x_o)
    ok, x = s.solvePressureBiCGSTAB(np.zeros(s.nv))
    assert ok and not x.any()


def test_reassembly_after_vertex_motion(cf, po):
    """build_sparse_matrices after the mesh moved (coupled path): device re-assembly equals the
    oracle built on the moved mesh."""
    m = make_mesh(cf, 3, 12)
    s, _ = make_pair(cf, po, m)
    xyz = m.vertices().copy()
    xyz[:, 1] *= 1.0 + 0.05 * np.sin(xyz[:, 0] / 5.0)
    s.updateVertices(xyz)
    o2 = po.Oracle(xyz, m.tets())
    o2.set_fluid(RHO, NU)
    o2.initialize()
    for which, name in [(0, "M"), (1, "K"), (2, "Gx"), (5, "L")]:
        assert csr_equal(s.matrix(which), o2.matrix(name)), name


@pytest.mark.parametrize("krylov", [0, 1, 2, 3], ids=["cg", "bicgstab", "cg1", "cg2l"])
def test_trajectory_bit_exact(cf, po, krylov):
    """The oracle reduces its Krylov dot products in the device's fixed tree and applies the
    same column-scaled operator, so FP64 trajectories agree bit for bit, iteration counts too."""
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-10, krylov=krylov)
    for k in range(6):
        assert s.pisoStep() and o.piso_step() == 0
        gs, os_ = s.stats(), o.stats()
        assert gs["momentum_iters"] == os_["momentum_iters"], k
        assert gs["pressure_iters"] == os_["pressure_iters"], k
        st = o.state()
        assert np.array_equal(s.getVelocityStar(), st["ustar"]), k
        assert np.array_equal(s.getPressureCorrection(), st["pcorr"]), k
        assert np.array_equal(s.getVelocity(), st["u"]), k
        assert np.array_equal(s.getPressure(), st["p"]), k


@pytest.mark.parametrize("krylov,norm", [(3, 0), (3, 1), (1, 0)], ids=["cg2l", "cg2l_jacobi_norm", "bicgstab"])
def test_momentum_cg_trajectory_bit_exact(cf, po, krylov, norm):
    """Momentum CG (CFSA_KRYLOV_CG) against the oracle's Jacobi CG on the same system: the batched
    kernels reduce in the oracle's orders (products over the SELL runs, vector updates over natural
    blocks), so the FP64 trajectories and iteration counts agree bit for bit."""
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-10, krylov=krylov, norm=norm, mom_cg=True)
    for k in range(6):
        assert s.pisoStep() and o.piso_step() == 0
        assert s.stats()["momentum_iters"] == o.stats()["momentum_iters"], k
        assert s.stats()["pressure_iters"] == o.stats()["pressure_iters"], k
        st = o.state()
        assert np.array_equal(s.getVelocityStar(), st["ustar"]), k
        assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"]), k


def test_momentum_cg_matches_bicgstab(cf, po):
    """CG and BiCGSTAB solve the same momentum system: at a tight tolerance in the Jacobi-scaled norm
    their trajectories agree to the FP64 bar, and CG needs fewer sparse products (one per
    iteration against two)."""
    m = make_mesh(cf, 4, 20)
    out = []
    for mom_cg in (False, True):
        s, _ = make_pair(cf, po, m, tol=1e-13, krylov=3, norm=cf.NORM_JACOBI, mom_cg=mom_cg)
        ok, done = s.pisoSteps(3)
        assert ok and done == 3
        out.append((s.getVelocity(), s.getPressure(), s.stats()["momentum_iters"]))
    assert rel_l2(out[1][0], out[0][0]) <= 1e-8
    assert rel_l2(out[1][1], out[0][1]) <= 1e-8
    assert max(out[1][2]) < 2 * max(out[0][2])


def test_momentum_cg_graph_equals_eager_and_failures(cf, po):
    """Graph and eager stepping give the same bits with momentum CG, and an iteration cap of one is
    reported as a failed step (as the oracle's CG reports it)."""
    m = make_mesh(cf, 3, 12)
    out = []
    for eager in ("0", "1"):
        os.environ["CFSA_NO_GRAPH"] = eager
        try:
            s, _ = make_pair(cf, po, m, tol=1e-10, krylov=3, mom_cg=True)
            ok, done = s.pisoSteps(3)
        finally:
            os.environ.pop("CFSA_NO_GRAPH", None)
        assert ok and done == 3
        out.append((s.getVelocity(), s.getPressure()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    s, o = make_pair(cf, po, m, tol=1e-10, krylov=3, maxit=(1, 20000), mom_cg=True)
    assert not s.pisoStep()
    assert o.piso_step() != 0


def test_persistent_cg_equals_loop_cg(cf, po):
    """The single-launch cooperative CG equals the three-kernel loop body bit for bit."""
    m = make_mesh(cf, 4, 20)
    out = []
    for loop in ("1", "0"):
        os.environ["CFSA_CG_LOOP"] = loop
        try:
            s, _ = make_pair(cf, po, m, tol=1e-10)
        finally:
            os.environ.pop("CFSA_CG_LOOP", None)
        ok, done = s.pisoSteps(3)
        assert ok and done == 3
        out.append((s.getVelocity(), s.getPressure(), s.stats()["pressure_iters"]))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


@pytest.mark.parametrize("layers", [20, 300], ids=["small", "many_blocks"])
def test_resident_cg_equals_persistent_cg(cf, po, layers):
    """The shared-memory-resident CG (one 1024-thread CTA per SM) equals the 256-thread persistent
    kernel and the three-kernel loop bit for bit; the larger mesh gives each CTA several blocks."""
    m = make_mesh(cf, 6, layers)
    out = []
    for env in ({"CFSA_CG_LOOP": "1"}, {"CFSA_CG_KERNEL": "persistent"}, {}):
        os.environ.update(env)
        try:
            s, _ = make_pair(cf, po, m, tol=1e-10)
        finally:
            for k in env:
                os.environ.pop(k, None)
        ok, done = s.pisoSteps(2)
        assert ok and done == 2
        out.append((s.getVelocity(), s.getPressure(), s.stats()["pressure_iters"]))
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])
        assert out[0][2] == o[2]


@pytest.mark.parametrize("krylov", [0, 1, 2, 3], ids=["cg", "bicgstab", "cg1", "cg2l"])
def test_jacobi_norm_trajectory_bit_exact(cf, po, krylov):
    """The Jacobi-scaled convergence norm, oracle and device in the same reduction tree."""
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-10, krylov=krylov, norm=cf.NORM_JACOBI, outlet_p=5.0)
    for k in range(4):
        assert s.pisoStep() and o.piso_step() == 0
        assert s.stats()["momentum_iters"] == o.stats()["momentum_iters"], k
        assert s.stats()["pressure_iters"] == o.stats()["pressure_iters"], k
        st = o.state()
        assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"]), k


def test_single_reduction_cg_matches_cg(cf, po):
    """CG with one reduction per iteration (CFSA_KRYLOV_CG1) converges to CG's solution (u, p
    within 1e-9 at a tight Jacobi-scaled tolerance) with the same iteration counts (within 2) at
    the benchmark tolerance 1e-10, on a mesh large enough that each CTA of the resident grid owns
    several blocks. Near the attainable accuracy (1e-13) the recurrence for s = A p makes the
    single-reduction variant need more iterations than CG, so counts are compared at 1e-10."""
    m = make_mesh(cf, 6, 300)
    for tol, check_iters in ((1e-13, False), (1e-10, True)):
        out = []
        for krylov in (cf.KRYLOV_CG, cf.KRYLOV_CG1):
            s, _ = make_pair(cf, po, m, tol=tol, krylov=krylov, norm=cf.NORM_JACOBI)
            ok, done = s.pisoSteps(3)
            assert ok and done == 3
            out.append((s.getVelocity(), s.getPressure(), s.stats()["pressure_iters"]))
        if check_iters:
            assert abs(out[1][2] - out[0][2]) <= 2, (out[0][2], out[1][2])
        else:
            assert rel_l2(out[1][0], out[0][0]) <= 1e-9
            assert rel_l2(out[1][1], out[0][1]) <= 1e-9


@pytest.mark.parametrize("target", [16, 256])
def test_two_level_cg_bit_exact_many_blocks(cf, po, target):
    """CFSA_KRYLOV_CG2L on a mesh where every CTA of the resident grid owns several blocks and
    aggregates span several CTAs: same coarse space (aggregate count), same iteration counts and
    the same bits as the oracle's cg2l, for a coarse and a fine aggregation."""
    m = make_mesh(cf, 6, 300)
    s, o = make_pair(cf, po, m, tol=1e-10, krylov=cf.KRYLOV_CG2L, norm=cf.NORM_JACOBI)
    s.setCoarseTarget(target)
    o.set_coarse_target(target)
    for k in range(2):
        assert s.pisoStep() and o.piso_step() == 0
        assert s.stats()["pressure_iters"] == o.stats()["pressure_iters"], k
        st = o.state()
        assert np.array_equal(s.getPressureCorrection(), st["pcorr"]), k
        assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"]), k
    assert s.coarseSize() == o.coarse_size() >= target


def test_two_level_cg_matches_cg(cf, po):
    """The two-level preconditioner changes the iterates, not the solution: u and p within 1e-8 of
    Jacobi CG (the FP64 parity bar) at a tight tolerance, in several times fewer pressure
    iterations."""
    m = make_mesh(cf, 6, 300)
    out = []
    for krylov in (cf.KRYLOV_CG, cf.KRYLOV_CG2L):
        s, _ = make_pair(cf, po, m, tol=1e-13, krylov=krylov, norm=cf.NORM_JACOBI)
        ok, done = s.pisoSteps(3)
        assert ok and done == 3
        out.append((s.getVelocity(), s.getPressure(), s.stats()["pressure_iters"]))
    assert rel_l2(out[1][0], out[0][0]) <= 1e-8
    assert rel_l2(out[1][1], out[0][1]) <= 1e-8
    assert out[1][2] * 2 < out[0][2], (out[0][2], out[1][2])


def test_two_level_cg_graph_equals_eager(cf, po):
    m = make_mesh(cf, 4, 40)
    res = []
    for env in ({"CFSA_NO_GRAPH": "1"}, {}):
        os.environ.update(env)
        try:
            s, _ = make_pair(cf, po, m, tol=1e-10, krylov=cf.KRYLOV_CG2L)
        finally:
            for k in env:
                os.environ.pop(k, None)
        ok, done = s.pisoSteps(3)
        assert ok and done == 3
        res.append((s.getVelocity(), s.getPressure()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_two_level_cg_bit_exact_y_bifurcation(cf, po):
    """The two-level CG on the Y-bifurcation (lattice vertex numbering, two outlets, boxes that cut
    across the branches): same coarse space, iteration counts and bits as the oracle."""
    m = cf.Mesh.yBifurcation(cell=0.4)
    prof = cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0)
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(1e-10, 1e-10)
    s.setMaxIterations(5000, 20000)
    s.setPressureSolver(cf.KRYLOV_CG2L)
    s.setConvergenceNorm(cf.NORM_JACOBI)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(RHO, NU))
    s.setInletVelocityProfile(prof)
    o = po.Oracle(m.vertices(), m.tets(), apply_bc=False)
    o.set_bc(*m.fluidBC())  # the generator's tags (inlet cap, both daughter caps outlet)
    o.set_fluid(RHO, NU)
    o.set_params(dt=0.01, tol_mom=1e-10, tol_p=1e-10, maxit_mom=5000, maxit_p=20000, pressure_solver=3,
                 conv_norm=1)
    o.initialize()
    o.set_inlet(prof)
    for k in range(2):
        assert s.pisoStep() and o.piso_step() == 0
        assert s.stats()["pressure_iters"] == o.stats()["pressure_iters"], k
        st = o.state()
        assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"]), k
    assert s.coarseSize() == o.coarse_size() > 0


@pytest.mark.parametrize("case", ["one_aggregate", "two_correctors_relaxed", "retarget_between_steps"])
def test_two_level_cg_edge_cases(cf, po, case):
    """Two-level CG against the oracle bit for bit: a single aggregate (a one-dimensional coarse
    space), two correctors with under-relaxation, and a coarse target changed between steps
    (coarse space and step graph rebuilt on both sides)."""
    m = make_mesh(cf, 4, 40)
    kw = dict(tol=1e-10, krylov=cf.KRYLOV_CG2L, norm=cf.NORM_JACOBI)
    if case == "two_correctors_relaxed":
        kw.update(ncorr=2, relax=(0.7, 0.6))
    s, o = make_pair(cf, po, m, **kw)
    if case == "one_aggregate":
        s.setCoarseTarget(1)
        o.set_coarse_target(1)
    for k in range(3):
        if case == "retarget_between_steps" and k == 1:
            s.setCoarseTarget(64)
            o.set_coarse_target(64)
        assert s.pisoStep() and o.piso_step() == 0
        assert s.stats()["pressure_iters"] == o.stats()["pressure_iters"], k
        st = o.state()
        assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"]), k
    assert s.coarseSize() == o.coarse_size()


def test_state_file_restart(cf, po, tmp_path):
    """saveState / loadState: a run restarted from the file after two steps continues bit for bit
    like the uninterrupted run (same u, p, time, step count); a file of another mesh is refused."""
    m = make_mesh(cf, 3, 12)
    a, _ = make_pair(cf, po, m, tol=1e-10, krylov=cf.KRYLOV_CG2L)
    ok, _ = a.pisoSteps(2)
    assert ok
    path = str(tmp_path / "state.bin")
    a.saveState(path)
    ok, _ = a.pisoSteps(2)
    assert ok
    b, _ = make_pair(cf, po, m, tol=1e-10, krylov=cf.KRYLOV_CG2L)
    b.loadState(path)
    assert b.getTime() == pytest.approx(0.02)
    ok, _ = b.pisoSteps(2)
    assert ok
    assert np.array_equal(a.getVelocity(), b.getVelocity()) and np.array_equal(a.getPressure(), b.getPressure())
    assert a.getTime() == b.getTime() and a.stats()["steps"] == b.stats()["steps"]
    other, _ = make_pair(cf, po, make_mesh(cf, 3, 13), tol=1e-10)
    with pytest.raises(cf.CfsaError) as ei:
        other.loadState(path)
    assert ei.value.code == cf.BAD_ARG


@pytest.mark.parametrize("mom_cg", [True, False], ids=["momentum_cg", "momentum_bicgstab"])
def test_headline_config_parity_1m_tets(cf, po, mom_cg):
    """The benchmark's own configuration: 999,936-tet cylinder, parabolic inlet (peak 1.0), FP64,
    two-level CG pressure (256-aggregate target) and batched Jacobi CG momentum (the bench's
    headline; BiCGSTAB, the reference's method, too) to 1e-10 in the reference's criterion, from
    rest. The oracle runs the same solver on the same mesh (its own mesher, identical arrays) and
    inputs; the first two steps agree bit for bit."""
    m = make_mesh(cf, 16, 217)
    assert m.nTets() == 999936
    prof = cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0)
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(1e-10, 1e-10)
    s.setMaxIterations(5000, 50000)
    s.setPressureSolver(cf.KRYLOV_CG2L)
    if mom_cg:
        s.setMomentumSolver(cf.KRYLOV_CG)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(RHO, NU))
    s.setInletVelocityProfile(prof)
    xyz, tets = po.cylinder(30.0, 2.0, 16, 217)
    assert np.array_equal(xyz, m.vertices()) and np.array_equal(tets, m.tets())
    o = po.Oracle(xyz, tets)
    o.set_fluid(RHO, NU)
    o.set_params(dt=0.01, tol_mom=1e-10, tol_p=1e-10, maxit_mom=5000, maxit_p=50000, pressure_solver=3)
    o.set_momentum_solver(1 if mom_cg else 0)
    o.initialize()
    o.set_inlet(prof)
    for k in range(2):
        assert s.pisoStep() and o.piso_step() == 0
        st = o.state()
        eu, ep = rel_l2(s.getVelocity(), st["u"]), rel_l2(s.getPressure(), st["p"])
        print(f"1M tets step {k + 1}: rel L2 u {eu:.2e} p {ep:.2e}")
        assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"])


def test_profile_kernel_leaves_the_solver_state(cf, po):
    """cfsa_ns_profile_kernel (momentum product, pressure product, whole pressure solve) runs on
    scratch buffers: the fields are unchanged and the next step is still bit-exact with the oracle."""
    m = make_mesh(cf, 3, 12)
    s, o = make_pair(cf, po, m, tol=1e-12, krylov=cf.KRYLOV_CG2L)
    assert s.pisoStep() and o.piso_step() == 0
    u, p = s.getVelocity().copy(), s.getPressure().copy()
    for which in (cf.KERNEL_MOMENTUM_SPMV, cf.KERNEL_PRESSURE_SPMV, cf.KERNEL_PRESSURE_SOLVE,
                  cf.KERNEL_MOMENTUM_SPMV_F32):
        ms, by = s.profileKernel(which, 3)
        assert ms > 0.0 and by > 0.0, which
    assert np.array_equal(s.getVelocity(), u) and np.array_equal(s.getPressure(), p)
    assert s.pisoStep() and o.piso_step() == 0
    st = o.state()
    assert np.array_equal(s.getVelocity(), st["u"]) and np.array_equal(s.getPressure(), st["p"])
