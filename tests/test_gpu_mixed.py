"""Mixed precision (FP32 BiCGSTAB with FP64 reliable updates) against the FP64 GPU path.

The momentum right-hand side is dominated by the 1e10 penalty rows, so the reference's criterion
||r|| <= tol ||b|| leaves the interior loosely determined at tol = 1e-10: FP64 solves at 1e-10
and at 1e-14 differ by ~1e-3 after one step on the 30k-tet cylinder. Mixed precision is therefore
checked against a converged FP64 reference (tol 1e-14): the mixed-precision bar, relative L2 <= 1e-6
on u and p, holds with the outer tolerance at 1e-12 (tested on the true FP64 residual).
"""
import os

import numpy as np
import pytest

from conftest import rel_l2
from test_gpu_parity import make_mesh, make_pair

pytestmark = pytest.mark.gpu


def run(cf, po, m, precision, steps, tol, **kw):
    kw.setdefault("maxit", (20000, 50000))
    s, _ = make_pair(cf, po, m, tol=tol, **kw)
    s.setPrecision(precision)
    out = []
    for _ in range(steps):
        assert s.pisoStep()
        out.append((s.getVelocity(), s.getPressure(), s.stats()))
    return out


@pytest.mark.parametrize("rings,layers", [(3, 12), (5, 68)])
def test_mixed_matches_converged_fp64(cf, po, rings, layers):
    """Mixed at outer tolerance 1e-12 against FP64 at 1e-14, both under the Jacobi-scaled
    criterion (under the reference criterion 1e-12 itself leaves ~1e-6 of interior slack, for FP64
    as much as for mixed; that norm is covered by the next test)."""
    m = make_mesh(cf, rings, layers)
    ref = run(cf, po, m, cf.PRECISION_FP64, 10, 1e-14, norm=cf.NORM_JACOBI)
    mix = run(cf, po, m, cf.PRECISION_MIXED, 10, 1e-12, norm=cf.NORM_JACOBI)
    for k in (0, 4, 9):
        eu, ep = rel_l2(mix[k][0], ref[k][0]), rel_l2(mix[k][1], ref[k][1])
        print(f"step {k + 1}: mixed(1e-12) vs fp64(1e-14) rel L2 u {eu:.2e} p {ep:.2e}; "
              f"iters {mix[k][2]['momentum_iters']} updates {mix[k][2]['momentum_outer']}")
        assert eu <= 1e-6 and ep <= 1e-6, (k, eu, ep)
    for _, _, st in mix:
        assert max(st["momentum_residual"]) <= 1e-12  # true FP64 residual
        assert max(st["momentum_outer"]) >= 1


def test_mixed_at_config_tolerance_is_no_worse_than_fp64(cf, po):
    """At the configs' 1e-10 both paths are loose in the interior; the mixed path (true-residual
    test) stays at least as close to the converged solution as the FP64 path."""
    m = make_mesh(cf, 3, 12)
    ref = run(cf, po, m, cf.PRECISION_FP64, 5, 1e-14)
    f64 = run(cf, po, m, cf.PRECISION_FP64, 5, 1e-10)
    mix = run(cf, po, m, cf.PRECISION_MIXED, 5, 1e-10)
    e64 = rel_l2(f64[-1][0], ref[-1][0])
    emx = rel_l2(mix[-1][0], ref[-1][0])
    print(f"5 steps at tol 1e-10: fp64 {e64:.2e}, mixed {emx:.2e} from the converged solution")
    assert emx <= 1.5 * e64


def test_mixed_graph_and_eager_identical(cf, po):
    m = make_mesh(cf, 3, 12)
    res = []
    for ng in ("0", "1"):
        os.environ["CFSA_NO_GRAPH"] = ng
        try:
            out = run(cf, po, m, cf.PRECISION_MIXED, 3, 1e-12)
        finally:
            os.environ.pop("CFSA_NO_GRAPH", None)
        res.append(out[-1])
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_mixed_reports_non_convergence(cf, po):
    """A tolerance below the FP64 residual floor cannot be met: the iteration cap ends the solve
    (the last reliable update finds the true residual above the tolerance) and pisoStep returns
    false without advancing time."""
    m = make_mesh(cf, 2, 6)
    s, _ = make_pair(cf, po, m, tol=1e-20)
    s.setPrecision(cf.PRECISION_MIXED)
    assert not s.pisoStep()
    assert s.getTime() == 0.0


def test_jacobi_norm_makes_1e10_meaningful(cf, po):
    """Under the Jacobi-scaled norm the configs' 1e-10 constrains the interior to a few 1e-6 of the
    converged solution, for FP64 as for mixed precision: mixed at 1e-10 is no farther from the
    converged solution than FP64 at 1e-10 (reliable updates stop where the FP64 solve stops), and at
    1e-12 both meet the 1e-6 bar."""
    m = make_mesh(cf, 5, 68)
    J = cf.NORM_JACOBI
    ref = run(cf, po, m, cf.PRECISION_FP64, 10, 1e-14, norm=J)
    f64 = run(cf, po, m, cf.PRECISION_FP64, 10, 1e-10, norm=J)
    mix = run(cf, po, m, cf.PRECISION_MIXED, 10, 1e-10, norm=J)
    mix12 = run(cf, po, m, cf.PRECISION_MIXED, 10, 1e-12, norm=J)
    for k in (0, 4, 9):
        e64 = (rel_l2(f64[k][0], ref[k][0]), rel_l2(f64[k][1], ref[k][1]))
        emx = (rel_l2(mix[k][0], ref[k][0]), rel_l2(mix[k][1], ref[k][1]))
        e12 = (rel_l2(mix12[k][0], ref[k][0]), rel_l2(mix12[k][1], ref[k][1]))
        print(f"jacobi norm step {k + 1}: fp64(1e-10) u {e64[0]:.2e} p {e64[1]:.2e}; "
              f"mixed(1e-10) u {emx[0]:.2e} p {emx[1]:.2e}; mixed(1e-12) u {e12[0]:.2e} p {e12[1]:.2e}; "
              f"iters fp64 {f64[k][2]['momentum_iters']} mixed {mix[k][2]['momentum_iters']} "
              f"updates {mix[k][2]['momentum_outer']}")
        assert emx[0] <= 1.5 * e64[0] + 1e-7 and emx[1] <= 1.5 * e64[1] + 1e-7, (k, emx, e64)
        assert max(e12) <= 1e-6, (k, e12)


def test_mixed_pressure_two_level_cg(cf, po):
    """CFSA_PRECISION_MIXED_FULL with the two-level CG pressure: the pressure solve runs in float storage
    inside FP64 defect correction (sweeps > 0, true FP64 residual at the tolerance). Against the
    converged FP64 solution: at 1e-10 no farther than FP64 at 1e-10, at 1e-12 within 1e-6."""
    m = make_mesh(cf, 5, 68)
    J, K = cf.NORM_JACOBI, cf.KRYLOV_CG2L
    ref = run(cf, po, m, cf.PRECISION_FP64, 10, 1e-14, norm=J, krylov=K)
    f64 = run(cf, po, m, cf.PRECISION_FP64, 10, 1e-10, norm=J, krylov=K)
    mix = run(cf, po, m, cf.PRECISION_MIXED_FULL, 10, 1e-10, norm=J, krylov=K)
    mix12 = run(cf, po, m, cf.PRECISION_MIXED_FULL, 10, 1e-12, norm=J, krylov=K)
    for k in (0, 4, 9):
        e64 = (rel_l2(f64[k][0], ref[k][0]), rel_l2(f64[k][1], ref[k][1]))
        emx = (rel_l2(mix[k][0], ref[k][0]), rel_l2(mix[k][1], ref[k][1]))
        e12 = (rel_l2(mix12[k][0], ref[k][0]), rel_l2(mix12[k][1], ref[k][1]))
        st = mix[k][2]
        print(f"step {k + 1}: fp64(1e-10) u {e64[0]:.2e} p {e64[1]:.2e}; mixed(1e-10) u {emx[0]:.2e} "
              f"p {emx[1]:.2e}; mixed(1e-12) u {e12[0]:.2e} p {e12[1]:.2e}; pressure iters "
              f"{st['pressure_iters']} sweeps {st['pressure_outer']}")
        assert emx[0] <= 1.5 * e64[0] + 1e-7 and emx[1] <= 1.5 * e64[1] + 1e-7, (k, emx, e64)
        assert max(e12) <= 1e-6, (k, e12)
    for _, _, st in mix:
        assert st["pressure_outer"] >= 1
        assert st["pressure_residual"] <= 1e-10


def test_mixed_pressure_graph_and_eager_identical(cf, po):
    m = make_mesh(cf, 3, 12)
    res = []
    for ng in ("0", "1"):
        os.environ["CFSA_NO_GRAPH"] = ng
        try:
            out = run(cf, po, m, cf.PRECISION_MIXED_FULL, 3, 1e-12, krylov=cf.KRYLOV_CG2L)
        finally:
            os.environ.pop("CFSA_NO_GRAPH", None)
        res.append(out[-1])
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    assert res[0][2]["pressure_outer"] == res[1][2]["pressure_outer"] >= 1


def test_mixed_keeps_fp64_pressure(cf, po):
    """CFSA_PRECISION_MIXED runs only the momentum solve in FP32: its pressure solve is the FP64
    two-level CG (no defect-correction sweeps)."""
    m = make_mesh(cf, 3, 12)
    out = run(cf, po, m, cf.PRECISION_MIXED, 2, 1e-12, krylov=cf.KRYLOV_CG2L)
    for _, _, st in out:
        assert st["pressure_outer"] == 0 and max(st["momentum_outer"]) >= 1


@pytest.mark.parametrize("rings,layers", [(3, 12), (5, 68)])
def test_mixed_momentum_cg_matches_converged_fp64(cf, po, rings, layers):
    """The momentum CG in FP32 with FP64 reliable updates (CFSA_KRYLOV_CG with a mixed precision)
    against a converged FP64 solution, Jacobi-scaled criterion: the same <= 1e-6 bar as the mixed
    BiCGSTAB, with the true FP64 residual at the tolerance."""
    m = make_mesh(cf, rings, layers)
    ref = run(cf, po, m, cf.PRECISION_FP64, 10, 1e-14, norm=cf.NORM_JACOBI)
    mix = run(cf, po, m, cf.PRECISION_MIXED, 10, 1e-12, norm=cf.NORM_JACOBI, mom_cg=True)
    for k in (0, 4, 9):
        eu, ep = rel_l2(mix[k][0], ref[k][0]), rel_l2(mix[k][1], ref[k][1])
        print(f"step {k + 1}: mixed CG(1e-12) vs fp64(1e-14) rel L2 u {eu:.2e} p {ep:.2e}; "
              f"iters {mix[k][2]['momentum_iters']} updates {mix[k][2]['momentum_outer']}")
        assert eu <= 1e-6 and ep <= 1e-6, (k, eu, ep)
    for _, _, st in mix:
        assert max(st["momentum_residual"]) <= 1e-12
        assert max(st["momentum_outer"]) >= 1


def test_mixed_momentum_cg_graph_eager_and_failure(cf, po):
    """Graph and eager stepping of the mixed momentum CG give the same bits; it stays as close to
    the converged solution as FP64 CG at the configs' tolerance; an unreachable tolerance ends in a
    failed step that does not advance time."""
    m = make_mesh(cf, 3, 12)
    res = []
    for ng in ("0", "1"):
        os.environ["CFSA_NO_GRAPH"] = ng
        try:
            out = run(cf, po, m, cf.PRECISION_MIXED, 3, 1e-12, mom_cg=True)
        finally:
            os.environ.pop("CFSA_NO_GRAPH", None)
        res.append(out[-1])
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    ref = run(cf, po, m, cf.PRECISION_FP64, 5, 1e-14)
    f64 = run(cf, po, m, cf.PRECISION_FP64, 5, 1e-10, mom_cg=True)
    mix = run(cf, po, m, cf.PRECISION_MIXED, 5, 1e-10, mom_cg=True)
    e64, emx = rel_l2(f64[-1][0], ref[-1][0]), rel_l2(mix[-1][0], ref[-1][0])
    print(f"5 steps at tol 1e-10: fp64 CG {e64:.2e}, mixed CG {emx:.2e} from the converged solution")
    assert emx <= 1.5 * e64
    s, _ = make_pair(cf, po, make_mesh(cf, 2, 6), tol=1e-20, mom_cg=True)
    s.setPrecision(cf.PRECISION_MIXED)
    assert not s.pisoStep()
    assert s.getTime() == 0.0
