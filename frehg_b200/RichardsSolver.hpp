// RichardsSolver.hpp — C++20 host mirror of frehg2's gw::RichardsSolver over
// the B200 C ABI (include/frehg_gw.h).
//
// The class keeps the reference's member names and meanings
// (src/gw/RichardsSolver.hpp:166-423): step(t, dtg) with t the end-of-step
// time, nextDt(), head(), waterContent(), the volumetric flux accessors,
// audit(), lastSolve() and ownedVolume().  Non-OK ABI statuses throw
// frehg_b200::FatalError, as the reference's log::fatal throws
// frehg::FatalError (src/core/Types.hpp:53-62), so driver-side error
// semantics are unchanged.  Fields come back in the ABI shapes (interior
// cells, k fastest); a driver that keeps the reference's halo-layout views
// copies them into their interiors.
#pragma once

#include <array>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/frehg_gw.h"

namespace frehg_b200 {

class FatalError : public std::runtime_error {
 public:
  FatalError(int status, const std::string& message)
      : std::runtime_error(message), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

/// The reference's GwStepAudit terms returned by the step.
struct GwStepAudit {
  double boundaryIn = 0.0;
  double ssStorage = 0.0;
  double reallocAdjust = 0.0;
  double reallocDropped = 0.0;
  double vloss = 0.0;
};

/// The groundwater state of a checkpoint (Simulation::checkpointFields3 and
/// the "dtg" scalar, driver/Simulation.cpp:707-722, 1211-1216).
struct GwCheckpoint {
  double t = 0.0, dtg = 0.0;
  std::vector<double> h, wc, vloss;
};

/// The reference's SolveStats of the predictor solve.
struct SolveStats {
  int iterations = 0;
  int outerSweeps = 0;
  double residualNorm = 0.0;
};

class RichardsSolver {
 public:
  /// Build the domain from a rasterized descriptor and set the initial state
  /// (`icForm` is FREHG_GW_IC_*; `icField` null means the constant).
  RichardsSolver(const frehg_gw_desc& desc, int icForm, double icConstant,
                 const double* icField = nullptr, void* cudaStream = nullptr)
      : nx_(desc.nx), ny_(desc.ny), nz_(desc.nz) {
    check(frehg_gw_create(&desc, &h_));
    if (cudaStream) check(frehg_gw_set_stream(h_, cudaStream));
    check(frehg_gw_init_state(h_, icForm, icConstant, icField));
  }
  RichardsSolver(const RichardsSolver&) = delete;
  RichardsSolver& operator=(const RichardsSolver&) = delete;
  ~RichardsSolver() { frehg_gw_destroy(h_); }

  /// RichardsSolver::updateBoundaryValues with the caller's value(t); null
  /// arrays keep their current values.
  void setBoundaryValues(const double* top, const double* bottom, const double* xm,
                         const double* xp, const double* ym, const double* yp) {
    check(frehg_gw_set_bc_values(h_, top, bottom, xm, xp, ym, yp));
  }

  /// RichardsSolver::step(t, dtg).
  void step(double t, double dtg) {
    frehg_gw_step_info info{};
    check(frehg_gw_step(h_, t, dtg, &info));
    audit_ = {info.boundary_in, info.ss_storage, info.realloc_adjust, info.realloc_dropped,
              info.vloss};
    last_ = {info.cg_iterations, info.outer_iterations, info.residual_norm};
  }

  double nextDt() const {
    double v = 0.0;
    check(frehg_gw_next_dt(h_, &v));
    return v;
  }

  std::vector<double> head() const { return field(FREHG_GW_FIELD_HEAD); }
  std::vector<double> waterContent() const { return field(FREHG_GW_FIELD_WC); }
  std::vector<double> waterContentStart() const { return field(FREHG_GW_FIELD_WC_START); }
  std::vector<double> fluxXVolumetric() const { return field(FREHG_GW_FIELD_QX); }
  std::vector<double> fluxYVolumetric() const { return field(FREHG_GW_FIELD_QY); }
  std::vector<double> fluxZFaceVolumetric() const { return field(FREHG_GW_FIELD_QZ); }
  std::vector<double> faceConductivityX() const { return field(FREHG_GW_FIELD_KX); }
  std::vector<double> faceConductivityY() const { return field(FREHG_GW_FIELD_KY); }
  std::vector<double> faceConductivityZFace() const { return field(FREHG_GW_FIELD_KZ); }

  /// The state a checkpoint stores, at time t.
  GwCheckpoint checkpoint(double t) const {
    return GwCheckpoint{t, nextDt(), head(), waterContent(), field(FREHG_GW_FIELD_VLOSS)};
  }

  /// Simulation::restoreFromCheckpoint for the groundwater step (:756-792).
  void restore(const GwCheckpoint& ck) {
    check(frehg_gw_restore(h_, ck.h.data(), ck.wc.data(),
                           ck.vloss.empty() ? nullptr : ck.vloss.data(), ck.dtg));
  }

  /// Restart read + refreshDerivedState (interior arrays).
  void setState(const double* head, const double* wc) { check(frehg_gw_set_state(h_, head, wc)); }

  const GwStepAudit& audit() const { return audit_; }
  const SolveStats& lastSolve() const { return last_; }

  double ownedVolume() const {
    double v = 0.0;
    check(frehg_gw_owned_volume(h_, &v));
    return v;
  }

  long long activeCells() const { return frehg_gw_active_cells(h_); }
  frehg_gw_handle* handle() const { return h_; }

  /// RichardsSolver::attachCoupling (RichardsSolver.hpp:180-186): the
  /// GwCoupling views as device arrays ((ny+2)*(nx+2) each; null entries are
  /// allocated by the library).
  void attachCoupling(const frehg_gw_coupling& c) { check(frehg_gw_attach_coupling(h_, &c)); }
  /// Host copy of a coupled surface field (FREHG_GW_SURF_*).
  std::vector<double> surface(int which) const {
    std::vector<double> out(static_cast<size_t>(ny_ + 2) * static_cast<size_t>(nx_ + 2));
    check(frehg_gw_get_surface(h_, which, out.data()));
    return out;
  }
  void setSurface(int which, const double* host) { check(frehg_gw_set_surface(h_, which, host)); }
  /// The GwStepAudit cpl* terms of the last step and pcClampVolume.
  frehg_gw_coupled_audit couplingAudit() const {
    frehg_gw_coupled_audit a{};
    check(frehg_gw_coupled_audit_get(h_, &a));
    return a;
  }

  /// RichardsSolver::attachScalar (baroclinic on) / attachTemperature /
  /// setDensityCoefficients (RichardsSolver.hpp:191-225): the scalars'
  /// device fields are allocated here; hand them over before each step with
  /// setScalar (host) or write scalarPointer (device).
  void attachDensity(bool saline, bool thermal, const frehg_gw_density& c) {
    check(frehg_gw_attach_density(h_, saline ? 1 : 0, thermal ? 1 : 0, &c));
  }
  void setScalar(int which, const double* host) { check(frehg_gw_set_scalar(h_, which, host)); }
  double* scalarPointer(int which) { return frehg_gw_scalar_ptr(h_, which); }
  /// densityRatio / viscosityRatio / densityRatioFaceY / densityRatioFaceZ
  /// (RichardsSolver.hpp:392-400), in the ABI shapes.
  std::vector<double> densityRatio() const { return field(FREHG_GW_FIELD_RHO); }
  std::vector<double> viscosityRatio() const { return field(FREHG_GW_FIELD_VISC); }
  std::vector<double> densityRatioFaceY() const { return field(FREHG_GW_FIELD_RHO_Y); }
  std::vector<double> densityRatioFaceZ() const { return field(FREHG_GW_FIELD_RHO_Z); }

 private:
  static void check(int rc) {
    if (rc != FREHG_GW_OK) throw FatalError(rc, frehg_gw_last_error());
  }
  std::vector<double> field(int which) const {
    std::vector<double> out(frehg_gw_field_size(h_, which));
    check(frehg_gw_get_field(h_, which, out.data()));
    return out;
  }

  frehg_gw_handle* h_ = nullptr;
  int nx_, ny_, nz_;
  GwStepAudit audit_;
  SolveStats last_;
};

/// coupling::Coupler (src/coupling/Coupler.hpp) for one coupled solver: the
/// subsurface side of the coupled step.  The caller's surface solve (its
/// free-surface phase and depth refresh) runs before step(t, dt), on the
/// solver's surface fields; its velocity phase after.
class Coupler {
 public:
  Coupler(RichardsSolver& gw, bool sync, double dt, double dtInit, double tStart = 0.0)
      : gw_(gw) {
    const frehg_gw_coupler_opts o{sync ? 1 : 0, dt, dtInit, tStart};
    check(frehg_gw_coupler_init(gw_.handle(), &o));
  }
  /// Coupler::step(t, dt): open the window, take the sync step or the
  /// subcycled steps that fit, apply the seepage, reduce the audit.
  void step(double t, double dt) { check(frehg_gw_coupler_step(gw_.handle(), t, dt, &audit_)); }
  double nextDt() const { return state(0.0)[0]; }
  double currentDtg() const { return state(0.0)[1]; }
  double gwLag(double t) const { return state(t)[2]; }
  void restore(double t, double dtg, double lag) {
    check(frehg_gw_coupler_restore(gw_.handle(), t, dtg, lag));
  }
  const frehg_gw_window_audit& audit() const { return audit_; }
  std::vector<double> seepageRate() const { return gw_.surface(FREHG_GW_SURF_QSS); }
  std::vector<double> gain() const { return gw_.surface(FREHG_GW_SURF_GAIN); }
  std::vector<double> seepAccum() const { return gw_.surface(FREHG_GW_SURF_SEEP_ACCUM); }

 private:
  static void check(int rc) {
    if (rc != FREHG_GW_OK) throw FatalError(rc, frehg_gw_last_error());
  }
  std::array<double, 3> state(double t) const {
    std::array<double, 3> v{};
    check(frehg_gw_coupler_state(gw_.handle(), t, &v[0], &v[1], &v[2]));
    return v;
  }
  RichardsSolver& gw_;
  frehg_gw_window_audit audit_{};
};

}  // namespace frehg_b200
