// Gradient of a wall-shear objective through the C++ adjoint operator pair: a cylinder run of
// `steps` PISO steps from rest with a parabolic inlet (set after initialize, as in the
// reference's CLI path), then J = mean |WSS|^2 over the wall vertices with 14 <= x <= 16 and its
// gradients with respect to the inlet nodal values and the viscosity.
//
//   ns_adjoint <rings> <layers> <steps> <checkpoint_every> [out.bin]
// out.bin (optional): int64 N2, double J, double dJ/dviscosity, double dJ/dinlet[N2][3].
#include "Mesh.hpp"
#include "NavierStokes.hpp"
#include "NavierStokesAdjoint.hpp"

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>

int main(int argc, char **argv) {
  const int rings = argc > 1 ? std::atoi(argv[1]) : 3;
  const int layers = argc > 2 ? std::atoi(argv[2]) : 12;
  const int steps = argc > 3 ? std::atoi(argv[3]) : 5;
  const int every = argc > 4 ? std::atoi(argv[4]) : 0;
  const char *out_path = argc > 5 ? argv[5] : nullptr;
  const double radius = 2.0;

  auto mesh = std::make_shared<Mesh>(Mesh::cylinder(30.0, radius, rings, layers));
  Mesh::setupBoundaryConditions(Vec3(1, 0, 0), 1, *mesh);
  auto ns = std::make_shared<NavierStokesSolver>();
  ns->setKrylovTolerances(1e-13, 1e-13);
  ns->setMaxIterations(20000, 50000);
  ns->setConvergenceNorm(CFSA_NORM_JACOBI);
  ns->setDt(0.01);
  Fluid blood;
  blood.density = 1060.0;
  blood.viscosity = 0.004;
  ns->initialize(mesh, blood);
  std::vector<Vec3> nodes = mesh->getVertPositions();
  const auto &edges = mesh->getEdgeNodePositions();
  nodes.insert(nodes.end(), edges.begin(), edges.end());
  std::vector<Vec3> profile(nodes.size(), Vec3::Zero());
  for (size_t i = 0; i < profile.size(); ++i) {
    const double r2 = nodes[i].y() * nodes[i].y() + nodes[i].z() * nodes[i].z();
    profile[i] = Vec3(1.0 * (1.0 - r2 / (radius * radius)), 0.0, 0.0);
  }
  ns->setInletVelocityProfile(profile);

  NavierStokesAdjoint adjoint(ns, every);
  if (!adjoint.forward(steps)) return 1;
  AdjointGradients g;
  if (!adjoint.backward(AdjointObjective::wallShear(0, 14.0, 16.0), g)) return 1;
  const cfsa_adjoint_stats st = adjoint.stats();
  std::cout << "[Adjoint] J = " << g.J << ", dJ/dviscosity = " << g.viscosity << ", checkpoints "
            << st.checkpoints << ", recomputed steps " << st.recomputed_steps << ", adjoint iterations "
            << st.momentum_iters << "/" << st.pressure_iters << std::endl;
  if (out_path) {
    FILE *f = std::fopen(out_path, "wb");
    if (!f) return 2;
    const int64_t n2 = (int64_t)g.inlet.size();
    std::fwrite(&n2, sizeof(n2), 1, f);
    std::fwrite(&g.J, sizeof(double), 1, f);
    std::fwrite(&g.viscosity, sizeof(double), 1, f);
    for (const auto &v : g.inlet) std::fwrite(v.data(), sizeof(double), 3, f);
    std::fclose(f);
  }
  return 0;
}
