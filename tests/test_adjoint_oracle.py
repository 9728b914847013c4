"""CPU checks of the discrete adjoint restated in the oracle (oracle/ns_oracle.cpp, adjoint_*):
gradients of both objectives with respect to inlet nodal values and viscosity against central
finite differences of the oracle's own forward PISO steps.

The adjoint differentiates the map (inlet values, viscosity) -> J(u^N, p^N) with the state at the
start of recording held fixed; the FD runs therefore restart from the same initial state (here:
rest, inlet set after initialize as in the reference's CLI order). Krylov solves run to 1e-15 in
the Jacobi-scaled norm so that solver noise stays far below the FD step's signal.
"""
import numpy as np
import pytest

RHO, NU, DT = 1060.0, 0.004, 0.01
H = 1e-6  # central-difference step (relative for viscosity)


def setup(cf, po, rings=2, layers=10):
    m = cf.Mesh.cylinder(30.0, 2.0, rings, layers)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    prof = cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0)
    p1, p2 = m.fluidBC()
    inlet_nodes = np.nonzero(np.concatenate([p1, p2]) == 1)[0]
    return m, prof, inlet_nodes


def oracle(po, m, prof, nu=NU):
    o = po.Oracle(m.vertices(), m.tets())
    o.set_fluid(RHO, nu)
    o.set_params(dt=DT, tol_mom=1e-15, tol_p=1e-15, maxit_mom=20000, maxit_p=50000,
                 pressure_solver=1, conv_norm=1)
    o.initialize()
    o.set_inlet(prof)
    return o


def objective_after(po, m, prof, nsteps, obj, nu=NU):
    o = oracle(po, m, prof, nu)
    for _ in range(nsteps):
        assert o.piso_step() == 0
    return o.objective(**obj)[0]


@pytest.mark.parametrize("obj", [dict(kind=0, axis=0, lo=14.0, hi=16.0), dict(kind=1)],
                         ids=["wall_shear_patch", "pressure_drop"])
def test_oracle_adjoint_matches_central_fd(cf, po, obj):
    nsteps = 3
    m, prof, inl = setup(cf, po)
    o = oracle(po, m, prof)
    assert o.adjoint_forward(nsteps) == 0
    J, su, sp, dnu = o.objective(**obj)
    r = o.adjoint_backward(su, sp, dnu)
    assert r["rc"] == 0
    assert r["iters"][0] > 0 and r["iters"][1] > 0
    gin = r["grad_inlet"]
    # the gradient lives on inlet nodes only
    mask = np.zeros(o.N2, bool)
    mask[inl] = True
    assert np.all(gin[~mask] == 0.0)
    rng = np.random.default_rng(20261203)
    sel = rng.choice(inl, size=6, replace=False)
    adj, fd = [], []
    for i in sel:
        pp = prof.copy()
        pm = prof.copy()
        pp[i, 0] += H
        pm[i, 0] -= H
        fd.append((objective_after(po, m, pp, nsteps, obj) - objective_after(po, m, pm, nsteps, obj)) / (2 * H))
        adj.append(gin[i, 0])
    adj, fd = np.array(adj), np.array(fd)
    assert np.linalg.norm(adj - fd) <= 1e-5 * np.linalg.norm(fd)
    hn = H * NU
    fdn = (objective_after(po, m, prof, nsteps, obj, NU + hn) -
           objective_after(po, m, prof, nsteps, obj, NU - hn)) / (2 * hn)
    assert abs(r["grad_viscosity"] - fdn) <= 1e-5 * abs(fdn)


def test_oracle_adjoint_initial_state_gradient(cf, po):
    """dJ/du0 and dJ/dp0 from the backward pass against FD on the initial state (same map).
    J here is O(1e3) while single components of the gradient are O(1e-4..1e-2), so the steps are
    large enough for the FD quotient to stay above the solver noise of J: over two steps J is a
    polynomial of degree 4 in u0 (h = 1e-3 leaves an O(h^2) truncation far below the bound) and of
    degree 2 in p0 (central differences are exact for any step)."""
    nsteps = 2
    h0, hp = 1e-3, 1.0
    obj = dict(kind=1)
    m, prof, _ = setup(cf, po)
    o = oracle(po, m, prof)
    st0 = o.state()
    assert o.adjoint_forward(nsteps) == 0
    J, su, sp, dnu = o.objective(**obj)
    r = o.adjoint_backward(su, sp, dnu)

    def J_from(u0, p0):
        o2 = oracle(po, m, prof)
        o2.set_state(u0, p0)
        for _ in range(nsteps):
            assert o2.piso_step() == 0
        return o2.objective(**obj)[0]

    p1, _ = m.fluidBC()
    free = np.nonzero(p1 == 3)[0][:3]
    for i in free:
        for c in range(3):
            up = st0["u"].copy()
            um = st0["u"].copy()
            up[i, c] += h0
            um[i, c] -= h0
            fd = (J_from(up, st0["p"]) - J_from(um, st0["p"])) / (2 * h0)
            assert abs(r["grad_u0"][i, c] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(r["grad_u0"]).max())
        pp = st0["p"].copy()
        pm = st0["p"].copy()
        pp[i] += hp
        pm[i] -= hp
        fd = (J_from(st0["u"], pp) - J_from(st0["u"], pm)) / (2 * hp)
        assert abs(r["grad_p0"][i] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(r["grad_p0"]).max())
