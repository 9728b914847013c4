// Forward/backward operator pair over the GPU discrete adjoint of the PISO step (the C ABI's
// cfsa_ns_adjoint_*), used the way a torch.autograd.Function is: forward(n) advances the solver n
// pisoStep()s and records what the backward pass needs (checkpoints every `checkpoint_every`
// steps, recomputation of earlier segments); backward(objective) returns J and its gradients
// with respect to the inlet nodal values and the viscosity, plus the adjoint of the state the
// forward pass started from. No counterpart in the reference (it has no differentiation).
#pragma once

#include "NavierStokes.hpp"

#include <iostream>
#include <memory>
#include <vector>

struct AdjointObjective {
  int kind = CFSA_OBJECTIVE_WALL_SHEAR;
  int axis = 0;
  double lo = 0.0, hi = 0.0;
  // mean over wall vertices with lo <= x[axis] <= hi of |computeShearStress()_v|^2
  static AdjointObjective wallShear(int axis, double lo, double hi) {
    return {CFSA_OBJECTIVE_WALL_SHEAR, axis, lo, hi};
  }
  // mean pressure over inlet vertices minus mean pressure over outlet vertices
  static AdjointObjective pressureDrop() { return {CFSA_OBJECTIVE_PRESSURE_DROP, 0, 0.0, 0.0}; }
};

struct AdjointGradients {
  double J = 0.0;
  std::vector<Vec3> inlet;  // dJ/d(inlet value) per P2 node (zero off inlet nodes)
  double viscosity = 0.0;   // dJ/d(viscosity)
  std::vector<Vec3> u0;     // dJ/du at the start of the forward pass
  std::vector<double> p0;   // dJ/dp at the start of the forward pass
};

class NavierStokesAdjoint {
 public:
  explicit NavierStokesAdjoint(std::shared_ptr<NavierStokesSolver> solver, int checkpoint_every = 0)
      : solver_(std::move(solver)), checkpoint_every_(checkpoint_every) {}

  bool forward(int nsteps) {
    if (!solver_ || !solver_->handle()) return false;
    int done = 0;
    const int code = cfsa_ns_adjoint_forward(solver_->handle(), nsteps, checkpoint_every_, &done);
    solver_->invalidateMirrors();
    return report(code, "adjoint forward");
  }

  bool backward(const AdjointObjective &obj, AdjointGradients &out) {
    if (!solver_ || !solver_->handle()) return false;
    const cfsa_objective o{obj.kind, obj.axis, obj.lo, obj.hi};
    std::vector<double> gin, gu0, gp0;
    size(gin, gu0, gp0);
    const int code = cfsa_ns_adjoint_backward(solver_->handle(), &o, &out.J, gin.data(), &out.viscosity,
                                              gu0.data(), gp0.data());
    solver_->invalidateMirrors();
    if (!report(code, "adjoint backward")) return false;
    unpack(gin, gu0, gp0, out);
    return true;
  }

  // Backward pass from a caller seed: dJ/du [N2] and dJ/dp [nv] of the final state and the
  // explicit dJ/d(viscosity) (the grad_output of an autograd function).
  bool backward(const std::vector<Vec3> &dJ_du, const std::vector<double> &dJ_dp, double dJ_dnu,
                AdjointGradients &out) {
    if (!solver_ || !solver_->handle()) return false;
    std::vector<double> du(3 * dJ_du.size()), gin, gu0, gp0;
    for (size_t i = 0; i < dJ_du.size(); ++i)
      for (int c = 0; c < 3; ++c) du[3 * i + c] = dJ_du[i][c];
    size(gin, gu0, gp0);
    if (du.size() != gin.size() || dJ_dp.size() != gp0.size()) return false;
    out.J = 0.0;
    const int code = cfsa_ns_adjoint_backward_seed(solver_->handle(), du.data(), dJ_dp.data(), dJ_dnu,
                                                   gin.data(), &out.viscosity, gu0.data(), gp0.data());
    solver_->invalidateMirrors();
    if (!report(code, "adjoint backward")) return false;
    unpack(gin, gu0, gp0, out);
    return true;
  }

  double objective(const AdjointObjective &obj) const {
    const cfsa_objective o{obj.kind, obj.axis, obj.lo, obj.hi};
    double J = 0.0;
    cfsa_ns_objective(solver_->handle(), &o, &J);
    return J;
  }

  cfsa_adjoint_stats stats() const {
    cfsa_adjoint_stats s{};
    if (solver_ && solver_->handle()) cfsa_ns_get_adjoint_stats(solver_->handle(), &s);
    return s;
  }

 private:
  std::shared_ptr<NavierStokesSolver> solver_;
  int checkpoint_every_;

  void size(std::vector<double> &gin, std::vector<double> &gu0, std::vector<double> &gp0) const {
    int64_t sz[4] = {0, 0, 0, 0};
    cfsa_ns_sizes(solver_->handle(), sz);
    gin.assign(3 * (size_t)sz[2], 0.0);
    gu0.assign(3 * (size_t)sz[2], 0.0);
    gp0.assign((size_t)sz[0], 0.0);
  }
  static void unpack(const std::vector<double> &gin, const std::vector<double> &gu0,
                     const std::vector<double> &gp0, AdjointGradients &out) {
    const size_t n2 = gin.size() / 3;
    out.inlet.resize(n2);
    out.u0.resize(n2);
    for (size_t i = 0; i < n2; ++i) {
      out.inlet[i] = Vec3(gin[3 * i], gin[3 * i + 1], gin[3 * i + 2]);
      out.u0[i] = Vec3(gu0[3 * i], gu0[3 * i + 1], gu0[3 * i + 2]);
    }
    out.p0 = gp0;
  }
  bool report(int code, const char *what) const {
    if (code == CFSA_OK) return true;
    std::cerr << "[NS-Adjoint] " << what << " failed (status " << code
              << "): " << cfsa_ns_last_error(solver_->handle()) << std::endl;
    return false;
  }
};
