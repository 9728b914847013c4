// Drop-in NavierStokesSolver: the reference class API (include/FEM/NavierStokes.hpp:53-251)
// with the numerics on the GPU behind the C ABI of cfsa_ns.h.
//
// Same members, signatures and semantics as the reference, with Vec3 in place of
// Eigen::Vector3d. Fields live on the device; getVelocity()/getPressure() return references to
// host mirrors that are refreshed after a step, so caller code that reads them every step works
// unchanged. Additions (marked "new") expose the settings the reference hard-codes.
#pragma once

#include "FluidTypes.hpp"
#include "Mesh.hpp"
#include "Vec3.hpp"
#include "cfsa_ns.h"

#include <cassert>
#include <memory>
#include <string>
#include <vector>

class NavierStokesSolver {
  cfsa_ns *h_ = nullptr;
  bool is_initialized_ = false;
  int reference_node_ = -1;

  double tolerance_ = 1e-12;  // NavierStokes.hpp:57 (the reference stores but never uses it)
  double momentum_tol_ = 1e-6;  // NavierStokes.cpp:500
  double pressure_tol_ = 1e-8;  // NavierStokes.cpp:635
  int momentum_maxit_ = 1000, pressure_maxit_ = 1000;
  int n_corrections_ = 1;
  double relax_u_ = 1.0;
  double relax_p_ = 1.0;
  double dt_ = 1e-4;
  int krylov_ = CFSA_KRYLOV_BICGSTAB;  // NavierStokes.cpp:633; the CG variants are opt-in
  int mom_krylov_ = CFSA_KRYLOV_BICGSTAB;  // NavierStokes.cpp:498; Jacobi CG is opt-in
  int coarse_target_ = 256;
  int precision_ = CFSA_PRECISION_FP64;
  int conv_norm_ = CFSA_NORM_REFERENCE;

  Fluid fluid_properties_;

  mutable std::vector<Vec3> velocity_;
  mutable std::vector<Vec3> velocity_star_;
  mutable std::vector<double> pressure_;
  mutable std::vector<double> pressure_correction_;
  mutable bool mirrors_stale_ = true;

  Vec3 mean_inlet_velocity_ = Vec3::Zero();
  std::vector<Vec3> inlet_profile_;  // per P2 node; empty = uniform mean_inlet_velocity_
  InletType inlet_type_ = InletType::Uniform;
  double outlet_pressure_ = 0.0;
  OutletType outlet_type_ = OutletType::DirichletPressure;

  std::shared_ptr<Mesh> mesh_ptr_ = nullptr;

  void syncMirrors() const;
  void pushInlet();
  void pushParameters();
  bool status(int code, const char *what) const;

 public:
  NavierStokesSolver() = default;
  ~NavierStokesSolver();
  NavierStokesSolver(const NavierStokesSolver &) = delete;
  NavierStokesSolver &operator=(const NavierStokesSolver &) = delete;

  void initialize(const std::shared_ptr<Mesh> mesh_ptr, const Fluid &fluid_properties);
  // The device assembles all four operators together; each build* call re-assembles them from
  // the mesh's current vertices and boundary tags (NavierStokes.cpp:70-356).
  void buildGradientMatrices() { build_sparse_matrices(); }
  void buildMassMatrix() { build_sparse_matrices(); }
  void buildStiffnessMatrix() { build_sparse_matrices(); }
  void buildPoissonMatrix() { build_sparse_matrices(); }
  void build_sparse_matrices();

  bool pisoStep();
  bool solveMomentumPredictor();
  void computeDivergence(const std::vector<Vec3> &u, std::vector<double> &div_out);
  std::vector<Vec3> computeAdvectionRHS();
  bool correctVelocity();
  bool solvePressurePoisson();
  // Declared but never defined by the reference (NavierStokes.hpp:111): returns false.
  bool solvePressureCG(const std::vector<double> &rhs, std::vector<double> &x);
  // NavierStokes.cpp:773-802: Jacobi BiCGSTAB (tol 1e-8, maxit 1000) on the raw Poisson matrix
  // (no boundary penalty) from a zero guess, on the device.
  bool solvePressureBiCGSTAB(const std::vector<double> &rhs, std::vector<double> &x);
  bool normalizePressire();

  bool hasNans();
  std::vector<Vec3> computePressureForces() const;
  std::vector<Vec3> computeShearStress() const;
  std::vector<Vec3> computeTotalFluidForces() const;
  Vec3 computeTotalMomentum() const;      // declared only, as in the reference
  double computeNetBoundaryFlux() const;  // declared only, as in the reference

  // getters
  double getViscosity() const { return fluid_properties_.viscosity; }
  double getDensity() const { return fluid_properties_.density; }
  double getTolerance() const { return tolerance_; }
  const std::vector<double> &getEffectiveViscosity() const {
    return fluid_properties_.effective_viscosity;
  }
  double getPressureAtNode(size_t ni) const {
    syncMirrors();
    assert(ni < pressure_.size());
    return pressure_[ni];
  }
  const Vec3 &getVelocityAtNode(size_t ni) const {
    syncMirrors();
    assert(ni < velocity_.size());
    return velocity_[ni];
  }
  const Mesh &getMesh() const { return *mesh_ptr_; }
  double getMeanFacePressure(size_t fi) const;
  Vec3 getPressureForceAtFace(size_t fi) const;

  // setters (NavierStokes.hpp:167-186)
  void setMeanInletVelocity(const Vec3 &vel);
  void setOutletType(OutletType type);
  void setOutletPressure(double p);
  void setInletType(InletType type) { inlet_type_ = type; }
  void setNumberOfCorrections(int n);
  void setRelaxU(double relax);
  void setRelaxP(double relax);
  void setReferencePressureNode(int node);
  void setDt(double dt);
  double getDt() const { return dt_; }
  // Routed to both Krylov solves (the reference keeps fixed 1e-6 / 1e-8).
  void setTolerance(double tol);
  double getTime() const;
  const std::vector<Vec3> &getVelocity() const {
    syncMirrors();
    return velocity_;
  }
  const std::vector<double> &getPressure() const {
    syncMirrors();
    return pressure_;
  }

  bool simpleStep();

  // new
  void setKrylovTolerances(double momentum, double pressure);
  void setMaxIterations(int momentum, int pressure);
  void setPressureSolver(int krylov);  // CFSA_KRYLOV_CG, _BICGSTAB, _CG1 or _CG2L
  void setMomentumSolver(int krylov);  // CFSA_KRYLOV_BICGSTAB or _CG (FP64 only)
  void setCoarseTarget(int target);    // aggregates of the CFSA_KRYLOV_CG2L coarse space (default 256)
  // new: binary restart file of u, p, time and step count (cfsa_ns_save_state / _load_state)
  bool saveState(const std::string &path);
  bool loadState(const std::string &path);
  void setPrecision(int precision);    // CFSA_PRECISION_FP64, _MIXED or _MIXED_FULL
  void setConvergenceNorm(int norm);   // CFSA_NORM_REFERENCE or CFSA_NORM_JACOBI
  void setInletVelocityProfile(const std::vector<Vec3> &per_node);
  bool pisoSteps(int n, int *n_done = nullptr);  // n steps, one host synchronisation
  cfsa_ns_stats getStats() const;
  cfsa_ns *handle() const { return h_; }
  // Host mirrors are re-read on the next getter call (for callers that change the device
  // fields through the C ABI directly, such as the adjoint forward/backward pair).
  void invalidateMirrors() const { mirrors_stale_ = true; }
};

// include/FEM/NavierStokes.hpp:201-251
class NavierStokesSimpleSolver {
 public:
  explicit NavierStokesSimpleSolver(std::shared_ptr<NavierStokesSolver> ns_solver)
      : solver_(ns_solver) {}
  bool step() {
    if (!solver_) return false;
    return solver_->simpleStep();
  }
  bool advanceSteps(int n) {
    for (int i = 0; i < n; ++i)
      if (!step()) return false;
    return true;
  }
  bool runUntil(double target_time) {
    while (getSolver()->getTime() < target_time)
      if (!step()) return false;
    return true;
  }
  double getTime() const { return solver_->getTime(); }
  std::shared_ptr<NavierStokesSolver> getSolver() { return solver_; }

 private:
  std::shared_ptr<NavierStokesSolver> solver_;
};
