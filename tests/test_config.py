"""YAML front-end (host/YamlConfig.cpp) through `examples/simulation --dry-run` (no GPU): the
fluid sections of the reference's config schema (src/IO/YamlConfig.cpp) plus the new keys."""
import subprocess

import pytest

from conftest import PKG

EXE = PKG / "examples" / "simulation"

CONFIG = """# fluid-only run
mesh:
  type: cylinder
  length: 12.0
  radius: 1.5          # tube radius
  divisions: 20
  max_element_size: 0.05
  flow_direction: [1.0, 0.0, 0.0]
  inlet_outlet_coverage: 1.0

navier_stokes:
  enabled: true
  density: 1000.0
  viscosity: 0.0035
  is_newtonian: true
  inlet_velocity: [0.25, 0.0, 0.0]
  outlet_pressure: 2.5
  use_dirichlet_pressure: true
  dt: 0.005
  relax_p: 0.7
  relax_u: 0.6
  tolerance: 1e-10
  max_iterations: [4000, 20000]
  precision: mixed
  pressure_solver: cg2l
  coarse_aggregates: 128
  convergence_norm: jacobi
  inlet_profile: parabolic

solid_mechanics:
  enabled: false

output:
  prefix: "run #1"
  total_steps: 7
  output_frequency: 3
  vtk_scale: 2.0

adjoint:
  enabled: true
  objective: pressure_drop
  checkpoint_every: 2
"""


def dry_run(tmp_path, text):
    p = tmp_path / "cfg.yaml"
    p.write_text(text)
    return subprocess.run([str(EXE), str(p), "--dry-run"], capture_output=True, text=True, timeout=60)


def parse(out):
    return dict(line.split(" = ", 1) for line in out.strip().splitlines())


def test_config_keys_resolved(tmp_path):
    assert EXE.exists()
    r = dry_run(tmp_path, CONFIG)
    assert r.returncode == 0, r.stderr
    d = parse(r.stdout)
    assert d["mesh.type"] == "cylinder" and float(d["mesh.length"]) == 12.0 and float(d["mesh.radius"]) == 1.5
    assert float(d["mesh.max_element_size"]) == 0.05 and d["mesh.flow_direction"] == "1 0 0"
    assert d["navier_stokes.enabled"] == "1" and float(d["navier_stokes.viscosity"]) == 0.0035
    assert d["navier_stokes.inlet_velocity"] == "0.25 0 0" and float(d["navier_stokes.outlet_pressure"]) == 2.5
    assert float(d["navier_stokes.dt"]) == 0.005 and float(d["navier_stokes.relax_p"]) == 0.7
    assert float(d["navier_stokes.tolerance"]) == 1e-10 and d["navier_stokes.max_iterations"] == "4000 20000"
    assert d["navier_stokes.precision"] == "mixed" and d["navier_stokes.pressure_solver"] == "cg2l"
    assert d["navier_stokes.coarse_aggregates"] == "128" and d["navier_stokes.momentum_solver"] == "bicgstab"
    assert d["navier_stokes.convergence_norm"] == "jacobi" and d["navier_stokes.inlet_profile"] == "parabolic"
    assert d["output.prefix"] == "run #1" and d["output.total_steps"] == "7" and d["output.output_frequency"] == "3"
    assert d["adjoint.enabled"] == "1" and d["adjoint.objective"] == "pressure_drop"
    assert d["adjoint.checkpoint_every"] == "2" and d["solid_mechanics.enabled"] == "0"


def test_config_defaults_are_the_references(tmp_path):
    r = dry_run(tmp_path, "mesh:\n  type: cylinder\nnavier_stokes:\n  enabled: true\n")
    assert r.returncode == 0, r.stderr
    d = parse(r.stdout)
    # src/IO/YamlConfig.cpp:45-96, 183-190
    assert float(d["mesh.length"]) == 30.0 and float(d["mesh.radius"]) == 2.0
    assert float(d["mesh.max_element_size"]) == 0.03
    assert float(d["navier_stokes.density"]) == 1060.0 and float(d["navier_stokes.viscosity"]) == 0.004
    assert d["navier_stokes.inlet_velocity"] == "0.10000000000000001 0 0"
    assert float(d["navier_stokes.dt"]) == 1e-3 and float(d["navier_stokes.relax_p"]) == 0.5
    assert d["navier_stokes.pressure_solver"] == "bicgstab" and d["navier_stokes.precision"] == "fp64"
    assert d["navier_stokes.momentum_solver"] == "bicgstab"
    assert d["output.prefix"] == "output" and d["output.total_steps"] == "1000" and d["output.output_frequency"] == "20"


@pytest.mark.parametrize("text,msg", [
    ("navier_stokes:\n  enabled: true\n", "Mesh configuration is required"),
    ("mesh:\n  length: 3\n", "Mesh type not specified"),
    ("mesh:\n  type: obj\n", "unknown value 'obj'"),
    ("mesh:\n  type: cylinder\n  flow_direction: [1, 0]\n", "expected [x, y, z]"),
    ("mesh:\n  type: cylinder\n  length: abc\n", "'length' must be a number"),
    ("mesh:\n  type: cylinder\n  type: msh\n", "duplicate key"),
    ("mesh:\n  type: cylinder\n    radius: 2\n", "unexpected indentation"),
    ("mesh:\n  type: msh\n", "msh_file required"),
    ("mesh:\n  type: cylinder\nnavier_stokes:\n  enabled: true\n  precision: fp16\n", "unknown value 'fp16'"),
    ("mesh:\n  type: cylinder\nnavier_stokes:\n  enabled: true\n  coarse_aggregates: 0\n", "coarse_aggregates must be in"),
    ("mesh:\n  type: cylinder\nnavier_stokes:\n  enabled: true\n  momentum_solver: gmres\n", "unknown value 'gmres'"),
])
def test_config_errors(tmp_path, text, msg):
    r = dry_run(tmp_path, text)
    assert r.returncode == 1
    assert msg in r.stderr, r.stderr
