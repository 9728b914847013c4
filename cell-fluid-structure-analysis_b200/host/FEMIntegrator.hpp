// Time integrator over the GPU NavierStokesSolver: same class and behaviour as the reference's
// NavierStokesIntegrator (include/Numerics/FEMIntegrator.hpp:10-92); its commented-out CFL
// diagnostic is omitted.
#pragma once

#include "NavierStokes.hpp"

#include <memory>

class NavierStokesIntegrator {
 public:
  NavierStokesIntegrator(std::shared_ptr<NavierStokesSolver> solver)
      : solver_(solver), time_(0.0), step_count_(0) {}

  bool step() {
    if (!solver_) return false;
    const bool success = solver_->pisoStep();
    if (success) {
      time_ = solver_->getTime();
      step_count_++;
    }
    return success;
  }

  bool advanceSteps(int n) {
    for (int i = 0; i < n; ++i)
      if (!step()) return false;
    return true;
  }

  bool runUntil(double target_time) {
    while (time_ < target_time)
      if (!step()) return false;
    return true;
  }

  double getTime() const { return time_; }
  int getStepCount() const { return step_count_; }
  std::shared_ptr<NavierStokesSolver> getSolver() { return solver_; }

 private:
  std::shared_ptr<NavierStokesSolver> solver_;
  double time_;
  int step_count_;
};
