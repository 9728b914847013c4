"""The CPU oracle against the golden fixtures of the independent numpy restatement and against
analytic identities of the reference's element matrices (src/FEM/NavierStokes.cpp:70-356)."""
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
import numpy_restatement as nr  # noqa: E402


def dense(csr, n):
    rp, ci, va = csr
    A = np.zeros((n, n))
    for i in range(n):
        A[i, ci[rp[i]:rp[i + 1]]] = va[rp[i]:rp[i + 1]]
    return A


@pytest.fixture(scope="module")
def prism(po):
    g = np.load(GOLD / "prism6.npz")
    o = po.Oracle(g["xyz"], g["tets"], apply_bc=False)
    o.set_fluid(1000.0, 0.001)
    o.initialize()
    return g, o


@pytest.mark.parametrize("name", ["M", "K", "Gx", "Gy", "Gz", "L"])
def test_prism_matrices_match_golden(prism, name):
    g, o = prism
    n = o.N2 if name in ("M", "K") else o.nv
    A = dense(o.matrix(name), n)
    np.testing.assert_allclose(A, g[name], rtol=1e-13, atol=1e-12 * np.abs(g[name]).max())


def test_prism_edge_numbering_and_lumped_mass(prism):
    g, o = prism
    assert np.array_equal(o.mesh()["tet_edges"], g["te"])
    np.testing.assert_allclose(o.inv_lumped_mass(), g["invm"], rtol=1e-14)


def test_prism_element_identities(prism):
    """Row sums: L, G and K rows sum to zero (sum_j grad phi_j = 0); mass rows are 0.45 rho V
    (vertex) and 0.28333 rho V (edge) per element (NavierStokes.cpp:256-284)."""
    g, o = prism
    nv = o.nv
    for name in ("L", "Gx", "Gy", "Gz"):
        A = dense(o.matrix(name), nv)
        assert np.abs(A.sum(axis=1)).max() < 1e-12 * np.abs(A).max()
    K = dense(o.matrix("K"), o.N2)
    assert np.abs(K.sum(axis=1)).max() < 1e-10 * np.abs(K).max()
    M = dense(o.matrix("M"), o.N2)
    mt = nr.mass_table()
    assert abs(mt[0].sum() - 0.45) < 1e-15 and abs(mt[4].sum() - (4 / 30 + 1 / 15 + 5 / 60)) < 1e-15
    # total mass-table weight per tet: 3.5 rho V; unit cube volume 1, rho = 1000
    assert abs(M.sum() - 3.5 * 1000.0) < 1e-9
    assert np.all(np.linalg.eigvalsh(mt) > 0.02)


def test_gradients_exact_on_unit_tet(po):
    xyz = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    o = po.Oracle(xyz, np.array([[0, 1, 2, 3]]), apply_bc=False)
    m = o.mesh()
    np.testing.assert_array_equal(m["grads"][0], [[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    assert m["vol"][0] == 1.0 / 6.0


@pytest.fixture(scope="module")
def cyl(po):
    g = np.load(GOLD / "cyl_piso.npz")
    return g


def run_oracle_cyl(po, g, solver, steps=3, momentum_solver=0):
    o = po.Oracle(g["xyz"], g["tets"])
    o.set_fluid(1060.0, 0.004)
    o.set_params(dt=0.01, tol_mom=1e-14, tol_p=1e-14, maxit_mom=5000, maxit_p=5000,
                 pressure_solver=solver)
    o.set_momentum_solver(momentum_solver)
    o.initialize()
    inl = np.zeros((o.N2, 3))
    inl[:, 0] = 0.5
    o.set_inlet(inl)
    out = []
    for _ in range(steps):
        assert o.piso_step() == 0
        out.append(o.state())
    return o, out


def test_cylinder_tags_match_golden(po, cyl):
    o = po.Oracle(cyl["xyz"], cyl["tets"])
    m = o.mesh()
    assert np.array_equal(m["p1"], cyl["p1"])
    assert np.array_equal(m["p2"], cyl["p2"])
    assert np.array_equal(m["tet_edges"], cyl["te"])


@pytest.mark.parametrize("solver,momentum_solver", [(0, 0), (1, 0), (1, 1)],
                         ids=["bicgstab", "cg", "cg_momentum_cg"])
def test_cylinder_piso_matches_golden(po, cyl, solver, momentum_solver):
    """Three pisoSteps of the oracle (tight Krylov tolerance) against the direct-solve numpy
    restatement: relative L2 <= 1e-8 on u, u*, p and p'. The momentum system is symmetric positive
    definite, so its CG solve (momentum_solver 1) meets the same bar."""
    _, states = run_oracle_cyl(po, cyl, solver, momentum_solver=momentum_solver)
    for k, s in enumerate(states):
        assert rel_l2(s["u"], cyl["u"][k]) < 1e-8
        assert rel_l2(s["ustar"], cyl["ustar"][k]) < 1e-8
        assert rel_l2(s["p"], cyl["p"][k]) < 1e-8
        assert rel_l2(s["pcorr"], cyl["pcorr"][k]) < 1e-8


def test_cylinder_operators_match_golden(po, cyl):
    o, states = run_oracle_cyl(po, cyl, 1, steps=1)
    o.set_state(cyl["u"][0], cyl["p"][0])  # same input as the golden operators
    np.testing.assert_allclose(o.advection(), cyl["conv0"], rtol=1e-12, atol=1e-12 * np.abs(cyl["conv0"]).max())
    d = o.divergence(cyl["ustar"][0])
    np.testing.assert_allclose(d, cyl["div0"], rtol=1e-12, atol=1e-12 * np.abs(cyl["div0"]).max())


def test_boundary_conditions_hold_after_step(po, cyl):
    _, states = run_oracle_cyl(po, cyl, 1, steps=2)
    u = states[-1]["u"]
    bc = np.concatenate([cyl["p1"], cyl["p2"]])
    assert np.all(u[bc == 0] == 0.0)
    assert np.all(u[bc == 1] == [0.5, 0.0, 0.0])
    assert np.all(states[-1]["p"][cyl["p1"] == 2] == 0.0)


def test_solver_failure_reports_not_converged(po, cyl):
    o = po.Oracle(cyl["xyz"], cyl["tets"])
    o.set_fluid(1060.0, 0.004)
    o.set_params(dt=0.01, tol_mom=1e-14, tol_p=1e-14, maxit_mom=1, maxit_p=1)
    o.initialize()
    inl = np.zeros((o.N2, 3))
    inl[:, 0] = 0.5
    o.set_inlet(inl)
    assert o.piso_step() == 1
    assert o.state()["time"] == 0.0
