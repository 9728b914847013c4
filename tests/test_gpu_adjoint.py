"""Discrete adjoint on the GPU (ns_adjoint.cuh behind cfsa_ns_adjoint_*):
  * against the oracle's adjoint restatement on the same mesh and inputs (bit-exact in FP64:
    both sides use the same summation orders and Krylov reduction trees);
  * against central finite differences of the GPU's own forward steps (the 1e-5 bar);
  * checkpointing with recomputation gives the same bits as a fully stored history;
  * graph-captured and eager reverse steps agree; seeds; invalidation; state restoration.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

RHO, NU, DT = 1060.0, 0.004, 0.01
WSS = dict(kind=0, axis=0, lo=14.0, hi=16.0)
PDROP = dict(kind=1)


def make_mesh(cf, rings, layers):
    m = cf.Mesh.cylinder(30.0, 2.0, rings, layers)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    return m


def gpu_solver(cf, m, prof, *, tol=1e-13, nu=NU, precision=0, krylov=0, mom_cg=False):
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(tol, tol)
    s.setMaxIterations(20000, 50000)
    s.setPressureSolver(krylov)
    s.setPrecision(precision)
    if mom_cg:
        s.setMomentumSolver(cf.KRYLOV_CG)
    s.setConvergenceNorm(cf.NORM_JACOBI)
    s.setDt(DT)
    s.initialize(m, cf.Fluid(RHO, nu))
    s.setInletVelocityProfile(prof)
    return s


def oracle(po, m, prof, *, tol=1e-13, nu=NU, krylov=0, mom_cg=False):
    o = po.Oracle(m.vertices(), m.tets())
    o.set_fluid(RHO, nu)
    o.set_params(dt=DT, tol_mom=tol, tol_p=tol, maxit_mom=20000, maxit_p=50000,
                 pressure_solver={0: 1, 1: 0, 2: 2, 3: 3}[krylov], conv_norm=1)
    if mom_cg:
        o.set_momentum_solver(1)
    o.initialize()
    o.set_inlet(prof)
    return o


@pytest.fixture(scope="module")
def small(cf):
    m = make_mesh(cf, 3, 12)
    prof = cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0)
    return m, prof


@pytest.mark.parametrize("obj", [WSS, PDROP], ids=["wall_shear_patch", "pressure_drop"])
@pytest.mark.parametrize("krylov", [0, 1, 2, 3], ids=["cg", "bicgstab", "cg1", "cg2l"])
def test_adjoint_bit_exact_vs_oracle(cf, po, small, obj, krylov):
    m, prof = small
    n = 4
    s = gpu_solver(cf, m, prof, krylov=krylov)
    assert s.adjointForward(n)
    g = s.adjointBackward(**obj)
    o = oracle(po, m, prof, krylov=krylov)
    assert o.adjoint_forward(n) == 0
    J, su, sp, dnu = o.objective(**obj)
    r = o.adjoint_backward(su, sp, dnu)
    assert r["rc"] == 0
    errs = {k: rel_l2(g[k], r[k]) for k in ("grad_inlet", "grad_u0", "grad_p0")}
    errs["grad_viscosity"] = abs(g["grad_viscosity"] - r["grad_viscosity"]) / abs(r["grad_viscosity"])
    errs["J"] = abs(g["J"] - J) / abs(J)
    assert all(e <= 1e-10 for e in errs.values()), errs
    assert g["J"] == J
    assert np.array_equal(g["grad_inlet"], r["grad_inlet"]), errs
    assert np.array_equal(g["grad_u0"], r["grad_u0"]), errs
    assert np.array_equal(g["grad_p0"], r["grad_p0"]), errs
    assert g["grad_viscosity"] == r["grad_viscosity"], errs


@pytest.mark.parametrize("obj", [WSS, PDROP], ids=["wall_shear_patch", "pressure_drop"])
def test_adjoint_momentum_cg_bit_exact_vs_oracle(cf, po, small, obj):
    """With the momentum CG the forward steps and the reverse pass's momentum solves (A is
    symmetric, so the adjoint solve is CG on A too) match the oracle bit for bit."""
    m, prof = small
    s = gpu_solver(cf, m, prof, krylov=3, mom_cg=True)
    assert s.adjointForward(4)
    g = s.adjointBackward(**obj)
    o = oracle(po, m, prof, krylov=3, mom_cg=True)
    assert o.adjoint_forward(4) == 0
    J, su, sp, dnu = o.objective(**obj)
    r = o.adjoint_backward(su, sp, dnu)
    assert r["rc"] == 0
    assert g["J"] == J
    for k in ("grad_inlet", "grad_u0", "grad_p0"):
        assert np.array_equal(g[k], r[k]), (k, rel_l2(g[k], r[k]))
    assert g["grad_viscosity"] == r["grad_viscosity"]


def test_adjoint_matches_gpu_central_fd(cf):
    """dJ/dg on 8 seeded inlet nodes (4 P1, 4 P2) and dJ/dnu against central FD, h = 1e-6.

    The momentum right-hand side carries 1e10 * g on inlet rows, so the penalty rows dominate
    ||b|| even in the Jacobi-scaled norm and a relative tolerance constrains the interior far
    less than the number suggests: at 1e-14 the FD quotients still carry ~1e-12 of solver noise
    (relative 1e-3 on this mesh), at 1e-16 ~1e-14, at 1e-18 ~1e-16. The adjoint itself does not
    move with the tolerance. Both runs therefore solve to 1e-18 (Jacobi-scaled)."""
    m = make_mesh(cf, 4, 40)
    prof = cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0)
    p1, p2 = m.fluidBC()
    nv = len(p1)
    inl = np.nonzero(np.concatenate([p1, p2]) == 1)[0]
    n = 10
    s = gpu_solver(cf, m, prof, tol=1e-18)
    u0, p0 = s.getVelocity().copy(), s.getPressure().copy()
    assert s.adjointForward(n)
    g = s.adjointBackward(**WSS)
    h = 1e-6

    def J_of(pr, nu=NU):
        s.setViscosity(nu)
        s.setInletVelocityProfile(pr)
        s.setFields(u0, p0)
        ok, done = s.pisoSteps(n)
        assert ok and done == n
        return s.objective(**WSS)

    rng = np.random.default_rng(20261203)
    sel = np.concatenate([rng.choice(inl[inl < nv], size=4, replace=False),
                          rng.choice(inl[inl >= nv], size=4, replace=False)])
    adj, fd = [], []
    for i in sel:
        pp, pm = prof.copy(), prof.copy()
        pp[i, 0] += h
        pm[i, 0] -= h
        fd.append((J_of(pp) - J_of(pm)) / (2 * h))
        adj.append(g["grad_inlet"][i, 0])
    adj, fd = np.array(adj), np.array(fd)
    assert np.linalg.norm(adj - fd) <= 1e-5 * np.linalg.norm(fd), (adj, fd)
    assert np.all(np.abs(adj[:4] - fd[:4]) <= 1e-5 * np.abs(fd[:4])), (adj, fd)
    hn = h * NU
    fdn = (J_of(prof, NU + hn) - J_of(prof, NU - hn)) / (2 * hn)
    assert abs(g["grad_viscosity"] - fdn) <= 1e-5 * abs(fdn), (g["grad_viscosity"], fdn)


def test_checkpoint_recompute_bit_exact(cf, small):
    m, prof = small
    n = 7
    a = gpu_solver(cf, m, prof)
    assert a.adjointForward(n, 0)
    ga = a.adjointBackward(**WSS)
    sa = a.adjointStats()
    assert sa["checkpoints"] == 1 and sa["recomputed_steps"] == 0
    b = gpu_solver(cf, m, prof)
    assert b.adjointForward(n, 3)
    gb = b.adjointBackward(**WSS)
    sb = b.adjointStats()
    assert sb["checkpoint_every"] == 3 and sb["checkpoints"] == 3 and sb["recomputed_steps"] == 6
    for k in ("grad_inlet", "grad_u0", "grad_p0"):
        assert np.array_equal(ga[k], gb[k]), k
    assert ga["grad_viscosity"] == gb["grad_viscosity"]
    # a second backward pass re-runs every segment (the record buffers hold segment 0 now)
    gb2 = b.adjointBackward(**WSS)
    assert b.adjointStats()["recomputed_steps"] == 7
    assert np.array_equal(gb2["grad_inlet"], gb["grad_inlet"])
    assert gb2["grad_viscosity"] == gb["grad_viscosity"]
    # the fields are left at the recorded final state
    assert np.array_equal(a.getVelocity(), b.getVelocity())
    assert a.getTime() == pytest.approx(n * DT)


def test_adjoint_graph_equals_eager(cf, small):
    m, prof = small
    os.environ["CFSA_NO_GRAPH"] = "1"
    try:
        e = gpu_solver(cf, m, prof)
    finally:
        del os.environ["CFSA_NO_GRAPH"]
    g = gpu_solver(cf, m, prof)
    for s in (e, g):
        assert s.adjointForward(5, 2)
    ge = e.adjointBackward(**PDROP)
    gg = g.adjointBackward(**PDROP)
    assert np.array_equal(ge["grad_inlet"], gg["grad_inlet"])
    assert ge["grad_viscosity"] == gg["grad_viscosity"]


def test_seed_api_equals_objective(cf, po, small):
    m, prof = small
    s = gpu_solver(cf, m, prof)
    assert s.adjointForward(3)
    g = s.adjointBackward(**WSS)
    o = oracle(po, m, prof)
    assert o.adjoint_forward(3) == 0
    J, su, sp, dnu = o.objective(**WSS)
    gs = s.adjointBackwardSeed(su, sp, dnu)
    assert np.array_equal(gs["grad_inlet"], g["grad_inlet"])
    assert gs["grad_viscosity"] == g["grad_viscosity"]


def test_recording_invalidated_by_changes(cf, small):
    m, prof = small
    s = gpu_solver(cf, m, prof)
    assert s.adjointForward(2)
    s.setInletVelocityProfile(prof * 1.01)
    with pytest.raises(cf.CfsaError) as ei:
        s.adjointBackward(**WSS)
    assert ei.value.code == cf.BAD_ARG
    fresh = gpu_solver(cf, m, prof)
    with pytest.raises(cf.CfsaError) as ei:
        fresh.adjointBackward(**WSS)
    assert ei.value.code == cf.NOT_INITIALIZED
    with pytest.raises(cf.CfsaError):
        fresh.objective(kind=0, axis=0, lo=100.0, hi=101.0)  # empty patch


def test_mixed_precision_adjoint(cf, small):
    """FP32 BiCGSTAB with FP64 reliable updates in forward and adjoint: gradients within 1e-6 of
    the FP64 adjoint (both to 1e-13 in the Jacobi-scaled norm)."""
    m, prof = small
    out = []
    for prec in (0, 1):
        s = gpu_solver(cf, m, prof, precision=prec)
        assert s.adjointForward(4)
        out.append(s.adjointBackward(**WSS))
    assert rel_l2(out[1]["grad_inlet"], out[0]["grad_inlet"]) <= 1e-6
    assert abs(out[1]["grad_viscosity"] - out[0]["grad_viscosity"]) <= 1e-6 * abs(out[0]["grad_viscosity"])
