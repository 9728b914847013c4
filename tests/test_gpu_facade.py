"""The C++ drop-in facade (host/NavierStokes.hpp + FEMIntegrator.hpp) driven by the example
program that mirrors the reference's examples/NavierStokes.cpp call sequence, against the oracle
configured the same way (inlet set before initialize, relaxation 0.5/0.5, Krylov tolerance 1e-10).
"""
import subprocess

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu


def read_output(path):
    raw = open(path, "rb").read()
    n2, nv = np.frombuffer(raw[:16], np.int64)
    u = np.frombuffer(raw[16:16 + 24 * n2], np.float64).reshape(n2, 3)
    p = np.frombuffer(raw[16 + 24 * n2:], np.float64)
    assert len(p) == nv
    return u, p


def test_cpp_example_matches_oracle(cf, po, tmp_path):
    exe = PKG / "examples" / "ns_cylinder"
    assert exe.exists(), "build the package (make) first"
    out = tmp_path / "state.bin"
    r = subprocess.run([str(exe), "3", "12", "10", str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "[Complete] steps 10" in r.stdout
    u, p = read_output(out)

    m = cf.Mesh.cylinder(30.0, 2.0, 3, 12)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    o = po.Oracle(m.vertices(), m.tets())
    o.set_fluid(1060.0, 0.004)
    o.set_params(dt=0.01, tol_mom=1e-10, tol_p=1e-10, maxit_mom=5000, maxit_p=50000,
                 relax_u=0.5, relax_p=0.5, pressure_solver=0)  # the default: BiCGSTAB, as the reference
    inl = np.zeros((o.N2, 3))
    inl[:, 0] = 0.5
    o.set_inlet(inl)  # before initialize, as in the example
    o.initialize()
    for _ in range(10):
        assert o.piso_step() == 0
    st = o.state()
    assert np.array_equal(u, st["u"])
    assert np.array_equal(p, st["p"])


def test_cpp_adjoint_pair_matches_python_api(cf, tmp_path):
    """examples/ns_adjoint.cpp (NavierStokesAdjoint forward/backward through the C++ facade)
    against the same run through the Python binding: identical bits."""
    exe = PKG / "examples" / "ns_adjoint"
    assert exe.exists(), "build the package (make) first"
    out = tmp_path / "grad.bin"
    r = subprocess.run([str(exe), "3", "12", "5", "2", str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "recomputed steps 4" in r.stdout, r.stdout
    raw = open(out, "rb").read()
    n2 = int(np.frombuffer(raw[:8], np.int64)[0])
    J, gnu = np.frombuffer(raw[8:24], np.float64)
    gin = np.frombuffer(raw[24:], np.float64).reshape(n2, 3)

    m = cf.Mesh.cylinder(30.0, 2.0, 3, 12)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(1e-13, 1e-13)
    s.setMaxIterations(20000, 50000)
    s.setConvergenceNorm(cf.NORM_JACOBI)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(1060.0, 0.004))
    s.setInletVelocityProfile(cf.parabolic_inlet(m.nodePositions(), 1.0, 2.0))
    assert s.adjointForward(5, 2)
    g = s.adjointBackward(kind=cf.OBJECTIVE_WALL_SHEAR, axis=0, lo=14.0, hi=16.0)
    assert J == g["J"]
    assert gnu == g["grad_viscosity"]
    assert np.array_equal(gin, g["grad_inlet"])
