// NavierStokesSolver facade: forwards the reference class API to the C ABI (cfsa_ns.h).
// Reference line numbers are for src/FEM/NavierStokes.cpp unless noted.
#include "NavierStokes.hpp"

#include <cmath>
#include <iostream>

NavierStokesSolver::~NavierStokesSolver() {
  if (h_) cfsa_ns_destroy(h_);
}

bool NavierStokesSolver::status(int code, const char *what) const {
  if (code == CFSA_OK) return true;
  std::cerr << "[NS] " << what << " failed (status " << code << "): " << cfsa_ns_last_error(h_)
            << std::endl;
  return false;
}

void NavierStokesSolver::syncMirrors() const {
  if (!h_ || !mirrors_stale_) return;
  const size_t N2 = velocity_.size(), nv = pressure_.size();
  std::vector<double> buf(3 * N2);
  if (cfsa_ns_get_velocity(h_, buf.data()) == CFSA_OK)
    for (size_t i = 0; i < N2; ++i) velocity_[i] = Vec3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
  if (cfsa_ns_get_velocity_star(h_, buf.data()) == CFSA_OK)
    for (size_t i = 0; i < N2; ++i)
      velocity_star_[i] = Vec3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
  if (nv) {
    cfsa_ns_get_pressure(h_, pressure_.data());
    cfsa_ns_get_pressure_correction(h_, pressure_correction_.data());
  }
  mirrors_stale_ = false;
}

void NavierStokesSolver::pushInlet() {
  if (!h_) return;
  if (!inlet_profile_.empty()) {
    std::vector<double> buf(3 * inlet_profile_.size());
    for (size_t i = 0; i < inlet_profile_.size(); ++i)
      for (int c = 0; c < 3; ++c) buf[3 * i + c] = inlet_profile_[i][c];
    status(cfsa_ns_set_inlet_profile(h_, buf.data()), "set inlet profile");
  } else {
    status(cfsa_ns_set_inlet_uniform(h_, mean_inlet_velocity_.data()), "set inlet");
  }
}

void NavierStokesSolver::pushParameters() {
  status(cfsa_ns_set_dt(h_, dt_), "setDt");
  status(cfsa_ns_set_tolerances(h_, momentum_tol_, pressure_tol_), "setTolerance");
  status(cfsa_ns_set_max_iterations(h_, momentum_maxit_, pressure_maxit_), "setMaxIterations");
  status(cfsa_ns_set_num_corrections(h_, n_corrections_), "setNumberOfCorrections");
  status(cfsa_ns_set_relaxation(h_, relax_u_, relax_p_), "setRelax");
  status(cfsa_ns_set_outlet(h_, (int)outlet_type_, outlet_pressure_), "setOutlet");
  status(cfsa_ns_set_reference_node(h_, reference_node_), "setReferencePressureNode");
  status(cfsa_ns_set_pressure_solver(h_, krylov_), "setPressureSolver");
  status(cfsa_ns_set_coarse_target(h_, coarse_target_), "setCoarseTarget");
  status(cfsa_ns_set_precision(h_, precision_), "setPrecision");
  status(cfsa_ns_set_momentum_solver(h_, mom_krylov_), "setMomentumSolver");
  status(cfsa_ns_set_convergence_norm(h_, conv_norm_), "setConvergenceNorm");
  pushInlet();
}

// NavierStokes.cpp:10-68
void NavierStokesSolver::initialize(const std::shared_ptr<Mesh> mesh_ptr, const Fluid &fluid_props) {
  mesh_ptr_ = mesh_ptr;
  fluid_properties_ = fluid_props;
  const Mesh &m = *mesh_ptr_;
  const size_t nv = m.nVertices(), nt = m.nTets(), ne = m.getNumberOfEdgeNodes();
  fluid_properties_.effective_viscosity.assign(nv + ne, fluid_props.viscosity);

  std::vector<double> xyz(3 * nv);
  for (size_t i = 0; i < nv; ++i)
    for (int c = 0; c < 3; ++c) xyz[3 * i + c] = m.getVertexPositon(i)[c];
  std::vector<int32_t> tets(4 * nt), edges(6 * nt);
  for (size_t t = 0; t < nt; ++t) {
    for (int k = 0; k < 4; ++k) tets[4 * t + k] = m.tetAt(t).vertids[k];
    for (int k = 0; k < 6; ++k) edges[6 * t + k] = m.getTetEdgeNodes(t)[k];
  }
  std::vector<int8_t> p1(nv), p2(ne);
  for (size_t i = 0; i < nv; ++i) p1[i] = (int8_t)m.getFluidVertexBC(i);
  for (size_t k = 0; k < ne; ++k) p2[k] = (int8_t)m.getP2FluidVertexBC(k);
  std::vector<int32_t> bverts, btet;
  std::vector<double> bnorm, barea;
  for (const Face &f : m.getFaces()) {
    if (f.tet_b != -1) continue;
    for (int k = 0; k < 3; ++k) bverts.push_back(f.vertids[k]);
    btet.push_back(f.tet_a);
    for (int c = 0; c < 3; ++c) bnorm.push_back(f.normal[c]);
    barea.push_back(f.area);
  }
  cfsa_mesh_view view{(int64_t)nv, (int64_t)nt, (int64_t)ne, xyz.data(), tets.data(), edges.data(),
                      p1.data(), p2.data(), (int64_t)btet.size(), bverts.data(), btet.data(),
                      bnorm.data(), barea.data()};
  cfsa_fluid fl{fluid_props.density, fluid_props.viscosity};
  if (h_) {
    cfsa_ns_destroy(h_);
    h_ = nullptr;
  }
  if (cfsa_ns_create(&view, &fl, &h_) != CFSA_OK) {
    std::cerr << "[NS] initialize failed: " << cfsa_ns_last_error(nullptr) << std::endl;
    h_ = nullptr;
    is_initialized_ = false;
    return;
  }
  is_initialized_ = true;
  velocity_.assign(nv + ne, Vec3::Zero());
  velocity_star_.assign(nv + ne, Vec3::Zero());
  pressure_.assign(nv, 0.0);
  pressure_correction_.assign(nv, 0.0);
  // Reference node for pressure null-space removal, Neumann outlets only (:48-67)
  if (reference_node_ < 0 && outlet_type_ == OutletType::Neumann) {
    for (size_t vi = 0; vi < nv; ++vi)
      if (m.getFluidVertexBC(vi) == FluidBCType::Internal) {
        reference_node_ = (int)vi;
        break;
      }
    if (reference_node_ < 0 && nv > 0) {
      reference_node_ = 0;
      std::cout << "[NS] Warning: No internal node found, using vertex 0 as pressure reference"
                << std::endl;
    }
  }
  pushParameters();
  status(cfsa_ns_initialize_fields(h_), "initialize fields");  // inlet nodes <- inlet (:33-46)
  mirrors_stale_ = true;
}

void NavierStokesSolver::build_sparse_matrices() {
  if (!h_) {
    std::cerr << "[NS] Error: mesh not initialized" << std::endl;
    return;
  }
  const Mesh &m = *mesh_ptr_;
  std::vector<double> xyz(3 * m.nVertices());
  for (size_t i = 0; i < m.nVertices(); ++i)
    for (int c = 0; c < 3; ++c) xyz[3 * i + c] = m.getVertexPositon(i)[c];
  std::vector<int8_t> p1(m.nVertices()), p2(m.getNumberOfEdgeNodes());
  for (size_t i = 0; i < p1.size(); ++i) p1[i] = (int8_t)m.getFluidVertexBC(i);
  for (size_t k = 0; k < p2.size(); ++k) p2[k] = (int8_t)m.getP2FluidVertexBC(k);
  status(cfsa_ns_update_boundary_tags(h_, p1.data(), p2.data()), "update boundary tags");
  status(cfsa_ns_update_vertices(h_, xyz.data()), "re-assemble");
}

bool NavierStokesSolver::pisoStep() {
  if (!is_initialized_) {
    std::cerr << "[NS] Error: solver not initialized" << std::endl;
    return false;
  }
  mirrors_stale_ = true;
  return status(cfsa_ns_piso_step(h_), "pisoStep");
}

bool NavierStokesSolver::pisoSteps(int n, int *n_done) {
  if (!is_initialized_) return false;
  mirrors_stale_ = true;
  return status(cfsa_ns_piso_steps(h_, n, n_done), "pisoSteps");
}

bool NavierStokesSolver::simpleStep() {
  if (!is_initialized_) {
    std::cerr << "[NS-Simple] Error: solver not initialized" << std::endl;
    return false;
  }
  mirrors_stale_ = true;
  return status(cfsa_ns_simple_step(h_), "simpleStep");
}

bool NavierStokesSolver::solveMomentumPredictor() {
  mirrors_stale_ = true;
  return status(cfsa_ns_momentum_predictor(h_), "momentum predictor");
}

bool NavierStokesSolver::solvePressurePoisson() {
  mirrors_stale_ = true;
  return status(cfsa_ns_pressure_poisson(h_), "pressure Poisson");
}

bool NavierStokesSolver::correctVelocity() {
  mirrors_stale_ = true;
  return status(cfsa_ns_correct_velocity(h_), "velocity correction");
}

bool NavierStokesSolver::solvePressureCG(const std::vector<double> &, std::vector<double> &) {
  std::cerr << "[NS] solvePressureCG: not provided (declared only in the reference)" << std::endl;
  return false;
}

// src/FEM/NavierStokes.cpp:773-802: Jacobi BiCGSTAB (tol 1e-8, maxit 1000, zero initial guess)
// on the raw Poisson matrix, no boundary penalty. As in the reference, the first x.size()
// entries of the solution are copied into x.
bool NavierStokesSolver::solvePressureBiCGSTAB(const std::vector<double> &rhs, std::vector<double> &x) {
  if (!h_) {
    std::cerr << "[NS] Error: solver not initialized" << std::endl;
    return false;
  }
  if (rhs.size() != pressure_.size() || x.size() > pressure_.size()) {
    std::cerr << "[NS] solvePressureBiCGSTAB: rhs needs one entry per pressure node" << std::endl;
    return false;
  }
  std::vector<double> sol(pressure_.size(), 0.0);
  const int code = cfsa_ns_solve_pressure_bicgstab(h_, rhs.data(), sol.data(), 1e-8, 1000);
  if (code != CFSA_OK) {
    std::cerr << "[NS] " << cfsa_ns_last_error(h_) << std::endl;
    return false;
  }
  std::copy(sol.begin(), sol.begin() + (std::ptrdiff_t)x.size(), x.begin());
  return true;
}

void NavierStokesSolver::computeDivergence(const std::vector<Vec3> &u, std::vector<double> &div_out) {
  std::vector<double> buf(3 * u.size());
  for (size_t i = 0; i < u.size(); ++i)
    for (int c = 0; c < 3; ++c) buf[3 * i + c] = u[i][c];
  div_out.assign(pressure_.size(), 0.0);
  status(cfsa_ns_compute_divergence(h_, buf.data(), div_out.data()), "computeDivergence");
}

std::vector<Vec3> NavierStokesSolver::computeAdvectionRHS() {
  std::vector<double> buf(3 * velocity_.size());
  std::vector<Vec3> out(velocity_.size());
  if (status(cfsa_ns_compute_advection(h_, buf.data()), "computeAdvectionRHS"))
    for (size_t i = 0; i < out.size(); ++i) out[i] = Vec3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
  return out;
}

// normalizePressire (:804-813) on the device-held pressure
bool NavierStokesSolver::normalizePressire() {
  syncMirrors();
  if (reference_node_ >= 0 && reference_node_ < (int)pressure_.size()) {
    const double ref = pressure_[reference_node_];
    for (auto &p : pressure_) p -= ref;
    return status(cfsa_ns_set_fields(h_, nullptr, pressure_.data()), "normalizePressire");
  }
  return true;
}

// NavierStokes.hpp:116-138
bool NavierStokesSolver::hasNans() {
  syncMirrors();
  for (const auto &v : velocity_)
    if (v.hasNaN()) return true;
  for (const auto &v : velocity_star_)
    if (v.hasNaN()) return true;
  for (double p : pressure_)
    if (std::isnan(p)) return true;
  for (double p : pressure_correction_)
    if (std::isnan(p)) return true;
  return false;
}

static std::vector<Vec3> to_vec3(const std::vector<double> &buf) {
  std::vector<Vec3> out(buf.size() / 3);
  for (size_t i = 0; i < out.size(); ++i) out[i] = Vec3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
  return out;
}

std::vector<Vec3> NavierStokesSolver::computePressureForces() const {
  std::vector<double> buf(3 * pressure_.size());
  if (!status(cfsa_ns_compute_pressure_forces(h_, buf.data()), "computePressureForces")) return {};
  return to_vec3(buf);
}

std::vector<Vec3> NavierStokesSolver::computeShearStress() const {
  std::vector<double> buf(3 * pressure_.size());
  if (!status(cfsa_ns_compute_shear_stress(h_, buf.data()), "computeShearStress")) return {};
  return to_vec3(buf);
}

std::vector<Vec3> NavierStokesSolver::computeTotalFluidForces() const {
  std::vector<double> buf(3 * pressure_.size());
  if (!status(cfsa_ns_compute_total_fluid_forces(h_, buf.data()), "computeTotalFluidForces")) return {};
  return to_vec3(buf);
}

// NavierStokes.cpp:357-372
double NavierStokesSolver::getMeanFacePressure(size_t fi) const {
  assert(mesh_ptr_ && fi < mesh_ptr_->nFaces());
  syncMirrors();
  const Face &f = mesh_ptr_->getFaces()[fi];
  double s = 0.0;
  for (const int vid : f.vertids) s += pressure_[vid];
  return s / static_cast<double>(f.vertids.size());
}

Vec3 NavierStokesSolver::getPressureForceAtFace(size_t fi) const {
  const double p = getMeanFacePressure(fi);
  const Face &f = mesh_ptr_->getFaces()[fi];
  return -f.normal * f.area * p;
}

void NavierStokesSolver::setMeanInletVelocity(const Vec3 &vel) {
  mean_inlet_velocity_ = vel;
  inlet_profile_.clear();
  pushInlet();
}

void NavierStokesSolver::setInletVelocityProfile(const std::vector<Vec3> &per_node) {
  inlet_profile_ = per_node;
  pushInlet();
}

void NavierStokesSolver::setOutletType(OutletType type) {
  outlet_type_ = type;
  if (h_) status(cfsa_ns_set_outlet(h_, (int)outlet_type_, outlet_pressure_), "setOutletType");
}

// NavierStokes.hpp:171-178 (warning kept)
void NavierStokesSolver::setOutletPressure(double p) {
  if (outlet_type_ != OutletType::DirichletPressure) {
    std::cout << "[NS Solver] Warning: setting outlet pressure without dirichlet outlet being the "
                 "outlet type"
              << std::endl;
  }
  outlet_pressure_ = p;
  if (h_) status(cfsa_ns_set_outlet(h_, (int)outlet_type_, outlet_pressure_), "setOutletPressure");
}

void NavierStokesSolver::setNumberOfCorrections(int n) {
  n_corrections_ = n;
  if (h_) status(cfsa_ns_set_num_corrections(h_, n), "setNumberOfCorrections");
}

void NavierStokesSolver::setRelaxU(double relax) {
  relax_u_ = relax;
  if (h_) status(cfsa_ns_set_relaxation(h_, relax_u_, relax_p_), "setRelaxU");
}

void NavierStokesSolver::setRelaxP(double relax) {
  relax_p_ = relax;
  if (h_) status(cfsa_ns_set_relaxation(h_, relax_u_, relax_p_), "setRelaxP");
}

void NavierStokesSolver::setReferencePressureNode(int node) {
  reference_node_ = node;
  if (h_) status(cfsa_ns_set_reference_node(h_, node), "setReferencePressureNode");
}

void NavierStokesSolver::setDt(double dt) {
  dt_ = dt;
  if (h_) status(cfsa_ns_set_dt(h_, dt), "setDt");
}

void NavierStokesSolver::setTolerance(double tol) {
  tolerance_ = tol;
  setKrylovTolerances(tol, tol);
}

void NavierStokesSolver::setKrylovTolerances(double momentum, double pressure) {
  momentum_tol_ = momentum;
  pressure_tol_ = pressure;
  if (h_) status(cfsa_ns_set_tolerances(h_, momentum, pressure), "setKrylovTolerances");
}

void NavierStokesSolver::setMaxIterations(int momentum, int pressure) {
  momentum_maxit_ = momentum;
  pressure_maxit_ = pressure;
  if (h_) status(cfsa_ns_set_max_iterations(h_, momentum, pressure), "setMaxIterations");
}

void NavierStokesSolver::setPressureSolver(int krylov) {
  krylov_ = krylov;
  if (h_) status(cfsa_ns_set_pressure_solver(h_, krylov), "setPressureSolver");
}

void NavierStokesSolver::setMomentumSolver(int krylov) {
  mom_krylov_ = krylov;
  if (h_) status(cfsa_ns_set_momentum_solver(h_, krylov), "setMomentumSolver");
}

bool NavierStokesSolver::saveState(const std::string &path) {
  if (!h_) return false;
  return status(cfsa_ns_save_state(h_, path.c_str()), "saveState");
}

bool NavierStokesSolver::loadState(const std::string &path) {
  if (!h_) return false;
  const bool ok = status(cfsa_ns_load_state(h_, path.c_str()), "loadState");
  invalidateMirrors();
  return ok;
}

void NavierStokesSolver::setCoarseTarget(int target) {
  coarse_target_ = target;
  if (h_) status(cfsa_ns_set_coarse_target(h_, target), "setCoarseTarget");
}

void NavierStokesSolver::setPrecision(int precision) {
  precision_ = precision;
  if (h_) status(cfsa_ns_set_precision(h_, precision), "setPrecision");
}

void NavierStokesSolver::setConvergenceNorm(int norm) {
  conv_norm_ = norm;
  if (h_) status(cfsa_ns_set_convergence_norm(h_, norm), "setConvergenceNorm");
}

double NavierStokesSolver::getTime() const {
  double t = 0.0;
  if (h_) cfsa_ns_get_time(h_, &t);
  return t;
}

cfsa_ns_stats NavierStokesSolver::getStats() const {
  cfsa_ns_stats s{};
  if (h_) cfsa_ns_get_stats(h_, &s);
  return s;
}
