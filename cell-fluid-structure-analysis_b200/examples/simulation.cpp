// `simulation <config.yaml> [--dry-run]`: the reference's YAML-driven CLI (src/main.cpp:313-370,
// 527-580, runNavierStokesOnly) for the fluid solver on the GPU. Same call order as the reference
// (mesh, boundary tags, initialize, inlet set after initialize, outlet, relaxation, dt,
// NavierStokesIntegrator loop, VTK every output_frequency steps and at the last step, max |u| and
// |p| per step). New keys (YamlConfig.hpp) select tolerances, precision, the pressure Krylov
// method, a parabolic inlet, and an adjoint gradient run. --dry-run prints the resolved settings
// and exits without touching the GPU.
#include "FEMIntegrator.hpp"
#include "Mesh.hpp"
#include "NavierStokes.hpp"
#include "NavierStokesAdjoint.hpp"
#include "VtkExport.hpp"
#include "YamlConfig.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>

namespace {

std::shared_ptr<Mesh> create_mesh(const config::MeshConfig &mc) {
  std::shared_ptr<Mesh> m;
  if (mc.type == "cylinder") {
    // procedural cylinder at the edge length of a regular tet of volume max_element_size
    const double h = std::cbrt(6.0 * std::sqrt(2.0) * mc.max_element_size);
    const int rings = mc.rings > 0 ? mc.rings : std::max(1, (int)std::lround(mc.cylinder_radius / h));
    const int layers = mc.layers > 0 ? mc.layers : std::max(1, (int)std::lround(mc.cylinder_length / h));
    m = std::make_shared<Mesh>(Mesh::cylinder(mc.cylinder_length, mc.cylinder_radius, rings, layers));
    Mesh::setupBoundaryConditions(mc.flow_direction, mc.inlet_outlet_coverage, *m);
  } else if (mc.type == "msh") {
    m = std::make_shared<Mesh>(Mesh::fromMshFile(mc.msh_file));
    Mesh::setupBoundaryConditions(mc.flow_direction, mc.inlet_outlet_coverage, *m);
  } else {
    YBifurcation y;
    y.cell = mc.cell;
    m = std::make_shared<Mesh>(Mesh::yBifurcation(y));
  }
  std::cout << "[Setup] Mesh created with " << m->nVertices() << " vertices, " << m->nTets() << " tetrahedra"
            << std::endl;
  return m;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::cerr << "Usage: " << argv[0] << " <config.yaml> [--dry-run]" << std::endl;
    return 1;
  }
  config::SimulationConfig cfg;
  try {
    cfg = config::loadConfig(argv[1]);
  } catch (const std::exception &e) {
    std::cerr << "ERROR: " << e.what() << std::endl;
    return 1;
  }
  if (argc > 2 && std::strcmp(argv[2], "--dry-run") == 0) {
    std::cout << config::describe(cfg);
    return 0;
  }
  if (cfg.solid_mechanics_enabled || cfg.dpm_enabled || cfg.fsi_enabled) {
    std::cerr << "ERROR: only the Navier-Stokes solver is part of this build" << std::endl;
    return 2;
  }
  if (!cfg.navier_stokes.enabled) {
    std::cerr << "ERROR: No solver enabled in configuration!" << std::endl;
    return 1;
  }
  const auto &N = cfg.navier_stokes;
  auto mesh = create_mesh(cfg.mesh);
  auto ns = std::make_shared<NavierStokesSolver>();
  Fluid fluid;
  fluid.density = N.density;
  fluid.viscosity = N.viscosity;
  if (N.tolerance > 0.0) ns->setTolerance(N.tolerance);
  ns->setMaxIterations(N.max_iterations[0], N.max_iterations[1]);
  ns->setNumberOfCorrections(N.n_corrections);
  ns->setPressureSolver(N.pressure_solver == "bicgstab" ? CFSA_KRYLOV_BICGSTAB
                        : N.pressure_solver == "cg"     ? CFSA_KRYLOV_CG
                        : N.pressure_solver == "cg1"    ? CFSA_KRYLOV_CG1
                                                        : CFSA_KRYLOV_CG2L);
  ns->setCoarseTarget(N.coarse_aggregates);
  ns->setPrecision(N.precision == "mixed"        ? CFSA_PRECISION_MIXED
                   : N.precision == "mixed_full" ? CFSA_PRECISION_MIXED_FULL
                                                 : CFSA_PRECISION_FP64);
  ns->setMomentumSolver(N.momentum_solver == "cg" ? CFSA_KRYLOV_CG : CFSA_KRYLOV_BICGSTAB);
  ns->setConvergenceNorm(N.convergence_norm == "jacobi" ? CFSA_NORM_JACOBI : CFSA_NORM_REFERENCE);
  ns->initialize(mesh, fluid);
  if (N.inlet_profile == "parabolic") {
    std::vector<Vec3> nodes = mesh->getVertPositions();
    const auto &edges = mesh->getEdgeNodePositions();
    nodes.insert(nodes.end(), edges.begin(), edges.end());
    const Vec3 d = cfg.mesh.flow_direction.normalized();
    const double peak = N.inlet_velocity.norm(), R = cfg.mesh.cylinder_radius;
    std::vector<Vec3> prof(nodes.size(), Vec3::Zero());
    for (size_t i = 0; i < nodes.size(); ++i) {
      const Vec3 radial = nodes[i] - d * nodes[i].dot(d);
      const double r2 = radial.dot(radial);
      prof[i] = d * (peak * (1.0 - r2 / (R * R)));
    }
    ns->setInletVelocityProfile(prof);
  } else {
    ns->setMeanInletVelocity(N.inlet_velocity);
  }
  if (N.use_dirichlet_pressure) ns->setOutletType(OutletType::DirichletPressure);
  ns->setOutletPressure(N.outlet_pressure);
  ns->setRelaxP(N.relax_p);
  ns->setRelaxU(N.relax_u);
  ns->setDt(N.dt);

  const auto &O = cfg.output;
  if (cfg.adjoint.enabled) {
    NavierStokesAdjoint adj(ns, cfg.adjoint.checkpoint_every);
    if (!adj.forward(O.total_steps)) return 1;
    if (O.output_fluid) io::exportToVtk(O.output_prefix + "_final.vtk", *ns, O.vtk_scale);
    AdjointGradients g;
    const AdjointObjective obj = cfg.adjoint.objective == "pressure_drop"
                                     ? AdjointObjective::pressureDrop()
                                     : AdjointObjective::wallShear(cfg.adjoint.axis, cfg.adjoint.lo, cfg.adjoint.hi);
    if (!adj.backward(obj, g)) return 1;
    FILE *f = std::fopen(cfg.adjoint.output.c_str(), "w");
    if (!f) return 1;
    std::fprintf(f, "J %.17g\ndJ_dviscosity %.17g\n# node dJ/dinlet_x dJ/dinlet_y dJ/dinlet_z (inlet nodes)\n", g.J,
                 g.viscosity);
    for (size_t i = 0; i < g.inlet.size(); ++i)
      if (g.inlet[i].x() != 0.0 || g.inlet[i].y() != 0.0 || g.inlet[i].z() != 0.0)
        std::fprintf(f, "%zu %.17g %.17g %.17g\n", i, g.inlet[i].x(), g.inlet[i].y(), g.inlet[i].z());
    std::fclose(f);
    std::cout << "[Adjoint] J = " << g.J << ", dJ/dviscosity = " << g.viscosity << ", gradients in "
              << cfg.adjoint.output << std::endl;
    return 0;
  }
  NavierStokesIntegrator integrator(ns);
  for (int step = 0; step < O.total_steps; ++step) {
    std::cout << "\n========== Time Step " << (step + 1) << " / " << O.total_steps << " ==========" << std::endl;
    std::cout << "Time: " << integrator.getTime() << " s" << std::endl;
    if (!integrator.step()) {
      std::cerr << "[Error] Simulation failed at step " << step << std::endl;
      return 1;
    }
    if (O.output_fluid && (step % O.output_frequency == 0 || step == O.total_steps - 1)) {
      const std::string filename = O.output_prefix + "_" + std::to_string(step / O.output_frequency) + ".vtk";
      io::exportToVtk(filename, *ns, O.vtk_scale);
      std::cout << "  Output written: " << filename << std::endl;
    }
    double max_vel = 0.0, max_p = 0.0;
    for (const auto &v : ns->getVelocity()) max_vel = std::max(max_vel, v.norm());
    for (double p : ns->getPressure()) max_p = std::max(max_p, std::abs(p));
    std::cout << "  Max velocity: " << max_vel << " m/s" << std::endl;
    std::cout << "  Max pressure: " << max_p << " Pa" << std::endl;
  }
  std::cout << "\nSimulation completed successfully!" << std::endl;
  return 0;
}
