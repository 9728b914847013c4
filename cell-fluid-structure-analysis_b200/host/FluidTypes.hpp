// Fluid parameter and boundary-condition types of the Navier-Stokes solver API.
//
// Same enumerators, order and defaults as the reference
// (include/FEM/NavierStokes.hpp:13-51 and include/FEM/SolidMechanics.hpp SolidBCType),
// because callers store and compare these values and the C ABI passes them as integers.
#pragma once

#include <vector>

enum class FluidBCType {
  Wall,  // no-slip
  Inlet,
  Outlet,
  Internal,
  Undefined,
};

enum class OutletType {
  DirichletPressure,
  Neumann,
  Undefined,
};

enum class InletType {
  Uniform,
  Pulsitile,
  Undefined,
};

enum class ViscosityModel {
  Newtonian,
  Carreau,
};

enum class TurbulenceModel {
  Laminar,
  RANS,
  LES,
};

// Solid boundary tags written by Mesh::setupBoundaryConditions (only Free/Fixed are used by
// the fluid path).
enum class SolidBCType {
  Free,
  Fixed,
  Displacement,
  Fluid,
  Undefined,
};

struct Fluid {
  double density = 1000;     // water-like
  double viscosity = 0.001;  // water-like
  TurbulenceModel turbuelence_model = TurbulenceModel::Laminar;
  ViscosityModel viscosity_model = ViscosityModel::Newtonian;
  std::vector<double> effective_viscosity;
};
