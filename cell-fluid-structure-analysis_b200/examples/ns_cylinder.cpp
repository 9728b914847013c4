// Transient flow in a cylinder through the drop-in C++ API: the same call sequence as the
// reference's examples/NavierStokes.cpp:43-131 (mesh, boundary tags, solver set-up with the
// inlet set before initialize, NavierStokesIntegrator loop, periodic statistics), on the GPU.
// The mesh comes from the procedural cylinder generator instead of TetGen.
//
//   ns_cylinder <rings> <layers> <steps> [out.bin]
// out.bin (optional): int64 N2, int64 nv, double u[N2][3], double p[nv] after the last step.
#include "FEMIntegrator.hpp"
#include "Mesh.hpp"
#include "NavierStokes.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>

int main(int argc, char **argv) {
  const int rings = argc > 1 ? std::atoi(argv[1]) : 5;
  const int layers = argc > 2 ? std::atoi(argv[2]) : 68;
  const int steps = argc > 3 ? std::atoi(argv[3]) : 20;
  const char *out_path = argc > 4 ? argv[4] : nullptr;
  const double length = 30.0, radius = 2.0, density = 1060.0, viscosity = 0.004;
  const double inlet_velocity = 0.5, outlet_pressure = 0.0, dt = 0.01;
  const int output_interval = std::max(1, steps / 4);

  auto mesh = std::make_shared<Mesh>(Mesh::cylinder(length, radius, rings, layers));
  std::cout << "[Setup] Mesh created with " << mesh->nVertices() << " vertices, " << mesh->nTets()
            << " tetrahedra" << std::endl;
  Mesh::setupBoundaryConditions(Vec3(1, 0, 0), 1, *mesh);

  auto ns_solver = std::make_shared<NavierStokesSolver>();
  ns_solver->setMeanInletVelocity(Vec3(inlet_velocity, 0.0, 0.0));
  ns_solver->setTolerance(1e-10);
  ns_solver->setMaxIterations(5000, 50000);
  Fluid blood;
  blood.density = density;
  blood.viscosity = viscosity;
  ns_solver->initialize(mesh, blood);
  ns_solver->setDt(dt);
  ns_solver->setOutletType(OutletType::DirichletPressure);
  ns_solver->setOutletPressure(outlet_pressure);
  ns_solver->setInletType(InletType::Uniform);
  ns_solver->setRelaxU(0.5);
  ns_solver->setRelaxP(0.5);

  NavierStokesIntegrator integrator(ns_solver);
  for (int step = 0; step < steps; ++step) {
    if (!integrator.step()) {
      std::cerr << "[Error] Simulation failed at step " << step << ", time = " << integrator.getTime()
                << std::endl;
      return 1;
    }
    if (step % output_interval == 0 || step == steps - 1) {
      double max_vel = 0.0, pmin = 1e300, pmax = -1e300;
      for (const auto &v : ns_solver->getVelocity()) max_vel = std::max(max_vel, v.norm());
      for (double p : ns_solver->getPressure()) {
        pmin = std::min(pmin, p);
        pmax = std::max(pmax, p);
      }
      const cfsa_ns_stats st = ns_solver->getStats();
      std::cout << "  Step " << step << ": t = " << integrator.getTime() << " s, max velocity = " << max_vel
                << " m/s, pressure range [" << pmin << ", " << pmax << "] Pa, iterations (momentum "
                << st.momentum_iters[0] << "/" << st.momentum_iters[1] << "/" << st.momentum_iters[2]
                << ", pressure " << st.pressure_iters << ")" << std::endl;
    }
  }
  std::cout << "[Complete] steps " << integrator.getStepCount() << ", time " << integrator.getTime()
            << std::endl;
  if (out_path) {
    FILE *f = std::fopen(out_path, "wb");
    if (!f) return 2;
    const auto &u = ns_solver->getVelocity();
    const auto &p = ns_solver->getPressure();
    const int64_t n2 = (int64_t)u.size(), nv = (int64_t)p.size();
    std::fwrite(&n2, sizeof(n2), 1, f);
    std::fwrite(&nv, sizeof(nv), 1, f);
    for (const auto &v : u) std::fwrite(v.data(), sizeof(double), 3, f);
    std::fwrite(p.data(), sizeof(double), p.size(), f);
    std::fclose(f);
  }
  return 0;
}
