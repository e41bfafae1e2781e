// Stand-in for frehg::swe::SurfaceSolver, so that the reference's own
// coupling::Coupler (src/coupling/Coupler.cpp, Exchange.cpp) compiles and runs
// unmodified in the oracle harness.  Test infrastructure: the shallow-water
// solve is out of the groundwater drop-in's scope, so this surface has no
// lateral flow.  Its free-surface phase adds a per-column rain depth
// rain * dt to eta, and its depth refresh is the surface solver's
// updateDepth rule (depth = eta - bottom, zero at or below min_depth,
// src/swe/WetDry.cpp:24-43).  The other phases the coupler calls are no-ops;
// ET and the paired store are off unless the harness switches the store on.
#ifndef FREHG_SHIM_SWE_SURFACE_SOLVER_HPP
#define FREHG_SHIM_SWE_SURFACE_SOLVER_HPP

#include <cstddef>

#include "core/Types.hpp"

namespace frehg::swe {

class SurfaceSolver {
 public:
  SurfaceSolver(std::size_t ny2, std::size_t nx2, real_t minDepth)
      : eta_("eta", ny2, nx2),
        dept_("dept", ny2, nx2),
        bottom_("bottom", ny2, nx2),
        rain_("rain", ny2, nx2),
        wetFrac_("wet_frac", ny2, nx2),
        wetClock_("wet_clock", ny2, nx2),
        minDepth_(minDepth) {}

  void setTimeStep(real_t dt) { dt_ = dt; }
  void beginStep(real_t) {}
  void solveFreeSurface() {
    for (std::size_t j = 0; j < eta_.extent(0); ++j)
      for (std::size_t i = 0; i < eta_.extent(1); ++i) eta_(j, i) += rain_(j, i) * dt_;
  }
  void refreshDepth() {
    for (std::size_t j = 0; j < eta_.extent(0); ++j)
      for (std::size_t i = 0; i < eta_.extent(1); ++i) {
        real_t d = eta_(j, i) - bottom_(j, i);
        if (d <= minDepth_) d = 0.0;
        dept_(j, i) = d;
      }
  }
  void routeStageDeposits(const Field2<real_t>&) {}
  void sweepAndRelease() {}
  void updateVelocity() {}

  bool etActive() const { return false; }
  bool pairedStore() const { return paired_; }
  void setPairedStore(bool on) { paired_ = on; }

  const Field2<real_t>& eta() const { return eta_; }
  const Field2<real_t>& depth() const { return dept_; }
  const Field2<real_t>& bottom() const { return bottom_; }
  const Field2<real_t>& wetFrac() const { return wetFrac_; }
  const Field2<real_t>& wetClockStepStart() const { return wetClock_; }
  Field2<real_t>& rain() { return rain_; }

 private:
  Field2<real_t> eta_, dept_, bottom_, rain_, wetFrac_, wetClock_;
  real_t minDepth_ = 0.0;
  real_t dt_ = 0.0;
  bool paired_ = false;
};

}  // namespace frehg::swe

#endif  // FREHG_SHIM_SWE_SURFACE_SOLVER_HPP
