"""CPU checks of the two-level pressure solver restated in the oracle (oracle/ns_oracle.cpp,
build_coarse / cg2l; pressure_solver 3, the device's CFSA_KRYLOV_CG2L): it solves the same system
as Jacobi CG (the reference's Poisson problem), needs far fewer iterations, and its coarse space
follows the requested aggregate count. The device is checked against it bit for bit in
test_gpu_parity.py."""
import numpy as np
import pytest

from conftest import rel_l2

RHO, NU, DT = 1060.0, 0.004, 0.01


def run(cf, po, m, solver, *, tol, steps=3, target=None, outlet=0, tags=None):
    o = po.Oracle(m.vertices(), m.tets(), apply_bc=tags is None)
    if tags is not None:
        o.set_bc(*tags)
    o.set_fluid(RHO, NU)
    o.set_params(dt=DT, tol_mom=tol, tol_p=tol, maxit_mom=20000, maxit_p=50000, outlet_type=outlet,
                 pressure_solver=solver, conv_norm=1)
    if target is not None:
        o.set_coarse_target(target)
    o.initialize()
    o.set_inlet(cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0))
    its = []
    for _ in range(steps):
        assert o.piso_step() == 0
        its.append(o.stats()["pressure_iters"])
    return o, its


@pytest.fixture(scope="module")
def mesh(cf):
    m = cf.Mesh.cylinder(30.0, 2.0, 4, 60)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    return m


@pytest.mark.parametrize("outlet", [0, 1], ids=["dirichlet", "neumann"])
def test_two_level_solves_the_same_system(cf, po, mesh, outlet):
    ref, it_cg = run(cf, po, mesh, 1, tol=1e-13, outlet=outlet)
    two, it_2l = run(cf, po, mesh, 3, tol=1e-13, outlet=outlet)
    a, b = ref.state(), two.state()
    assert rel_l2(b["u"], a["u"]) <= 1e-9
    assert rel_l2(b["p"], a["p"]) <= 1e-9
    assert all(2 * x < y for x, y in zip(it_2l, it_cg)), (it_cg, it_2l)
    assert two.coarse_size() >= 256


def test_coarse_target_controls_aggregates(cf, po, mesh):
    sizes, iters = [], []
    for target in (8, 64, 512):
        o, its = run(cf, po, mesh, 3, tol=1e-10, steps=1, target=target)
        sizes.append(o.coarse_size())
        iters.append(its[0])
    assert sizes[0] >= 8 and sizes[1] >= 64 and sizes[2] >= 512
    assert sizes[0] < sizes[1] < sizes[2]
    assert iters[2] <= iters[0], iters


def test_two_level_deterministic(cf, po, mesh):
    a, _ = run(cf, po, mesh, 3, tol=1e-10, steps=2)
    b, _ = run(cf, po, mesh, 3, tol=1e-10, steps=2)
    assert np.array_equal(a.state()["p"], b.state()["p"])
    assert np.array_equal(a.state()["u"], b.state()["u"])


def test_two_level_on_y_bifurcation(cf, po):
    """Lattice-numbered Y mesh: geometric aggregates still cut the pressure iterations and the
    solution matches Jacobi CG."""
    m = cf.Mesh.yBifurcation(cell=0.4)
    ref, it_cg = run(cf, po, m, 1, tol=1e-13, steps=2, tags=m.fluidBC())
    two, it_2l = run(cf, po, m, 3, tol=1e-13, steps=2, tags=m.fluidBC())
    assert rel_l2(two.state()["p"], ref.state()["p"]) <= 1e-8
    assert rel_l2(two.state()["u"], ref.state()["u"]) <= 1e-8
    assert all(2 * x < y for x, y in zip(it_2l, it_cg)), (it_cg, it_2l)
