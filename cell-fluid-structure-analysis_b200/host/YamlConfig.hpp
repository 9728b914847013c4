// YAML configuration of a fluid simulation: the reference's config::loadConfig
// (include/IO/YamlConfig.hpp, src/IO/YamlConfig.cpp:30-96, 180-220) for the sections this build
// runs (mesh, navier_stokes, output), read by a self-contained parser of the YAML subset the
// reference's config files use (yaml-cpp is not required): nested block mappings by indentation,
// `key: value` scalars, `[a, b, c]` flow sequences, `#` comments, quoted or bare strings.
// The solid_mechanics, dpm and fsi_coupling sections are parsed for `enabled` only.
//
// New keys (all optional; defaults reproduce the reference's behaviour):
//   mesh.type: cylinder | msh | y_bifurcation
//   mesh.rings / mesh.layers        cylinder resolution (default: derived from max_element_size)
//   mesh.msh_file                   Gmsh MSH 4.1 file (type msh)
//   mesh.cell                       lattice edge of the Y-bifurcation (type y_bifurcation)
//   navier_stokes.tolerance          Krylov tolerance of both solves (reference: 1e-6 / 1e-8)
//   navier_stokes.max_iterations     [momentum, pressure] iteration caps (reference: 1000, 1000)
//   navier_stokes.n_corrections      PISO correctors (reference: 1)
//   navier_stokes.precision          fp64 | mixed | mixed_full
//   navier_stokes.pressure_solver    bicgstab | cg | cg1 | cg2l (reference: bicgstab)
//   navier_stokes.coarse_aggregates  aggregates of the cg2l coarse space (default 256)
//   navier_stokes.momentum_solver    bicgstab | cg (reference: bicgstab; cg needs precision fp64)
//   navier_stokes.convergence_norm   reference | jacobi
//   navier_stokes.inlet_profile      uniform | parabolic (peak = |inlet_velocity|, radius = mesh radius)
//   adjoint.enabled / objective (wall_shear | pressure_drop) / axis / lo / hi / checkpoint_every /
//   output (text file of J, dJ/dviscosity and dJ/dinlet per node)
#pragma once

#include "Vec3.hpp"

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace config {

struct MeshConfig {
  std::string type = "cylinder";
  double cylinder_length = 30.0, cylinder_radius = 2.0;
  int cylinder_divisions = 35;
  double max_element_size = 0.03;
  int rings = 0, layers = 0;  // 0: derived from max_element_size
  std::string msh_file;
  double cell = 0.081;
  Vec3 flow_direction = Vec3(1.0, 0.0, 0.0);
  double inlet_outlet_coverage = 1.0;
};

struct NavierStokesConfig {
  bool enabled = false;
  double density = 1060.0, viscosity = 0.004;
  bool is_newtonian = true, is_laminar = true;
  Vec3 inlet_velocity = Vec3(0.1, 0.0, 0.0);
  double outlet_pressure = 0.0;
  bool use_dirichlet_pressure = true;
  double dt = 1e-3, relax_p = 0.5, relax_u = 0.5;
  // new
  double tolerance = 0.0;  // 0: the reference's 1e-6 / 1e-8
  int max_iterations[2] = {1000, 1000};
  int n_corrections = 1;
  std::string precision = "fp64", pressure_solver = "bicgstab", convergence_norm = "reference";
  std::string momentum_solver = "bicgstab";
  std::string inlet_profile = "uniform";
  int coarse_aggregates = 256;
};

struct OutputConfig {
  std::string output_prefix = "output";
  int total_steps = 1000, output_frequency = 20;
  double vtk_scale = 1.0;
  bool output_fluid = true;
};

struct AdjointConfig {
  bool enabled = false;
  std::string objective = "wall_shear";
  int axis = 0;
  double lo = 0.0, hi = 0.0;
  int checkpoint_every = 0;
  std::string output = "adjoint_gradients.txt";
};

struct SimulationConfig {
  MeshConfig mesh;
  NavierStokesConfig navier_stokes;
  OutputConfig output;
  AdjointConfig adjoint;
  bool solid_mechanics_enabled = false, dpm_enabled = false, fsi_enabled = false;
};

// Parsed YAML node: a scalar, a sequence of scalars, or a mapping.
struct Node {
  enum Kind { Scalar, Sequence, Map } kind = Map;
  std::string scalar;
  std::vector<std::string> items;
  std::map<std::string, std::shared_ptr<Node>> children;
  const Node *get(const std::string &key) const;
};

// Parses YAML-subset text; throws std::runtime_error with a line number on malformed input.
std::shared_ptr<Node> parseYaml(const std::string &text);
SimulationConfig parseConfig(const std::string &text);
SimulationConfig loadConfig(const std::string &yaml_file);
// key = value lines of every resolved setting (used by `simulation --dry-run`)
std::string describe(const SimulationConfig &c);

}  // namespace config
