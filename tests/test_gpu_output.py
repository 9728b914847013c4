"""VTK export from device buffers (cfsa_ns_write_vtk behind io::exportToVtk): the file must be
the text the reference's writer (src/IO/VtkExport.cpp:49-84, 238-268) produces from the same
mesh and fields, i.e. C++ default stream formatting (6 significant digits, %g style)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def g(x):
    return format(float(x), "g")


def expected_text(m, u, p, scale):
    xyz = m.vertices()
    tets = m.tets()
    p1, _ = m.fluidBC()
    out = ["# vtk DataFile Version 3.0", "Shape export", "ASCII", "DATASET UNSTRUCTURED_GRID",
           f"POINTS {len(xyz)} double"]
    out += [f"{g(a * scale)} {g(b * scale)} {g(c * scale)}" for a, b, c in xyz]
    out.append(f"CELLS {len(tets)} {len(tets) * 5}")
    out += [f"4 {a} {b} {c} {d}" for a, b, c, d in tets]
    out.append(f"CELL_TYPES {len(tets)}")
    out += ["10"] * len(tets)
    out += ["", f"POINT_DATA {len(xyz)}", "SCALARS FluidBoundaryType int 1", "LOOKUP_TABLE default"]
    out += [str(int(b)) for b in p1]
    out += ["", "SCALARS pressure double 1", "LOOKUP_TABLE default"]
    out += [g(v) for v in p]
    out += ["", "VECTORS velocity double"]
    nv = len(xyz)
    out += [f"{g(a * scale)} {g(b * scale)} {g(c * scale)}" for a, b, c in u[:nv]]
    return "\n".join(out) + "\n"


def test_vtk_export_matches_reference_format(cf, tmp_path):
    m = cf.Mesh.cylinder(30.0, 2.0, 3, 12)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    s = cf.NavierStokesSolver()
    s.setTolerance(1e-10)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(1060.0, 0.004))
    s.setMeanInletVelocity([0.5, 0.0, 0.0])
    ok, _ = s.pisoSteps(3)
    assert ok
    path = tmp_path / "ns.vtk"
    s.exportToVtk(path, 2.0)
    assert path.read_text() == expected_text(m, s.getVelocity(), s.getPressure(), 2.0)
    # the optional boundary-force vectors equal computeShearStress / computePressureForces
    path2 = tmp_path / "ns_forces.vtk"
    s.exportToVtk(path2, 1.0, cf.VTK_SHEAR_STRESS | cf.VTK_PRESSURE_FORCES)
    text = path2.read_text()
    assert text.startswith(expected_text(m, s.getVelocity(), s.getPressure(), 1.0))
    tail = text[len(expected_text(m, s.getVelocity(), s.getPressure(), 1.0)):].split("\n")
    nv = m.sizes[0]
    assert tail[0] == "" and tail[1] == "VECTORS shear_stress double"
    sh = np.array([[float(x) for x in l.split()] for l in tail[2:2 + nv]])
    assert np.allclose(sh, s.computeShearStress(), rtol=1e-5, atol=1e-300)
    assert tail[2 + nv] == "" and tail[3 + nv] == "VECTORS pressure_forces double"
    pf = np.array([[float(x) for x in l.split()] for l in tail[4 + nv:4 + 2 * nv]])
    assert np.allclose(pf, s.computePressureForces(), rtol=1e-5, atol=1e-300)


@pytest.mark.parametrize("momentum", ["bicgstab", "cg"])
def test_yaml_cli_run_matches_api(cf, tmp_path, momentum):
    """`simulation config.yaml` (the reference CLI's fluid-only loop) writes the VTK files of the
    same run through the API: identical text at the last output step, with the reference's
    momentum BiCGSTAB and with `momentum_solver: cg`."""
    import subprocess

    from conftest import PKG

    exe = PKG / "examples" / "simulation"
    cfg = tmp_path / "cfg.yaml"
    cfg.write_text(
        "mesh:\n  type: cylinder\n  length: 30.0\n  radius: 2.0\n  rings: 3\n  layers: 12\n"
        "  flow_direction: [1.0, 0.0, 0.0]\n"
        "navier_stokes:\n  enabled: true\n  density: 1060.0\n  viscosity: 0.004\n"
        "  inlet_velocity: [0.5, 0.0, 0.0]\n  outlet_pressure: 0.0\n  dt: 0.01\n  relax_p: 0.5\n"
        "  relax_u: 0.5\n  tolerance: 1e-10\n  max_iterations: [5000, 50000]\n  pressure_solver: cg\n"
        f"  momentum_solver: {momentum}\n"
        f"output:\n  prefix: {tmp_path / 'run'}\n  total_steps: 5\n  output_frequency: 2\n  vtk_scale: 1.0\n")
    r = subprocess.run([str(exe), str(cfg)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    files = sorted(p.name for p in tmp_path.glob("run_*.vtk"))
    assert files == ["run_0.vtk", "run_1.vtk", "run_2.vtk"]
    m = cf.Mesh.cylinder(30.0, 2.0, 3, 12)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    s = cf.NavierStokesSolver()
    s.setTolerance(1e-10)
    s.setMaxIterations(5000, 50000)
    s.setPressureSolver(cf.KRYLOV_CG)
    s.setMomentumSolver(cf.KRYLOV_CG if momentum == "cg" else cf.KRYLOV_BICGSTAB)
    s.initialize(m, cf.Fluid(1060.0, 0.004))
    s.setMeanInletVelocity([0.5, 0.0, 0.0])
    s.setOutletType(cf.OutletType.DirichletPressure)
    s.setOutletPressure(0.0)
    s.setRelaxP(0.5)
    s.setRelaxU(0.5)
    s.setDt(0.01)
    for _ in range(5):
        assert s.pisoStep()
    api = tmp_path / "api.vtk"
    s.exportToVtk(api, 1.0)
    assert (tmp_path / "run_2.vtk").read_text() == api.read_text()


def test_async_readback_equals_synchronous_getters(cf):
    """cfsa_ns_get_velocity_async / _pressure_async: each step's fields, read back into alternating
    pinned host buffers while the next step runs, equal the synchronous getters of that step bit
    for bit once cfsa_ns_wait_outputs returns; pageable buffers work too (the copy then completes
    before the call returns)."""
    import torch

    m = cf.Mesh.cylinder(30.0, 2.0, 3, 12)
    m.setupBoundaryConditions((1.0, 0.0, 0.0), 1.0)
    s = cf.NavierStokesSolver()
    s.setKrylovTolerances(1e-10, 1e-10)
    s.setPressureSolver(cf.KRYLOV_CG2L)
    s.setMomentumSolver(cf.KRYLOV_CG)
    s.setDt(0.01)
    s.initialize(m, cf.Fluid(1060.0, 0.004))
    s.setMeanInletVelocity([0.5, 0.0, 0.0])
    ub = [torch.empty((s.N2, 3), dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    pb = [torch.empty((s.nv,), dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    ref = []
    for k in range(5):
        assert s.pisoStep()
        s.getVelocityAsync(ub[k % 2])
        s.getPressureAsync(pb[k % 2])
        ref.append((s.getVelocity().copy(), s.getPressure().copy()))
    s.waitOutputs()
    for k in (3, 4):
        assert np.array_equal(ub[k % 2], ref[k][0]) and np.array_equal(pb[k % 2], ref[k][1]), k
    u_pageable, p_pageable = np.empty((s.N2, 3)), np.empty(s.nv)
    assert s.pisoStep()
    s.getVelocityAsync(u_pageable)
    s.getPressureAsync(p_pageable)
    s.waitOutputs()
    assert np.array_equal(u_pageable, s.getVelocity()) and np.array_equal(p_pageable, s.getPressure())
    with pytest.raises(ValueError):
        s.getVelocityAsync(None)
