// C entry points around the reference's own, unmodified frehg::gw::
// RichardsSolver (compiled from the reference's sources against the host
// shims in oracle/shim/include).  Test infrastructure only: it builds the
// solver exactly the way the reference's unit-test harness does
// (tests/unit/test_gw.cpp:33-61, MiniGw::build) from an in-code FrehgConfig,
// so python tests can drive the real reference step and read its fields.
//
// Field transfers use the reference's own (ny+2, nx+2, nz[+1]) halo layout
// with k fastest (src/core/Types.hpp:35-43).

#include "bc/BoundarySet.hpp"
#include "coupling/Coupler.hpp"
#include "core/Config.hpp"
#include "core/Grid.hpp"
#include "core/HaloExchanger.hpp"
#include "core/Types.hpp"
#include "gw/RichardsSolver.hpp"
#include "gw/TerrainMetric.hpp"

#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

extern "C" void frehg_shim_set_pc(const char* pc);

extern "C" {

/// Flat description of one groundwater case.  Soil types carry 8 numbers
/// each: ksx, ksy, ksz, theta_s, theta_r, alpha, n, aev.  Boundary
/// conditions: target (1 top, 2 bottom, 3 side), kind (4 head, 5 flux), value
/// form (0 constant, 2 gravity, 3 hydrostatic), value, hydrostatic stage and
/// polygon vertices (x, y pairs; bc_npts per condition, concatenated).
typedef struct ref_case {
  int nx, ny, nz;
  double dx, dy, dz, dz_stretch;
  int follow_terrain, terrain_uniform;
  const double* bath;  // ny*nx (j*nx + i), or NULL for a flat bed at 0
  int n_soil_types;
  const double* soil_types;
  const int* soil_map;  // ny*nx*nz ids ((j*nx + i)*nz + k), or NULL
  int ic_form;          // 0 moisture, 1 head, 2 water table
  double ic_const;
  const double* ic_field;  // 3D for moisture/head, 2D for water table, or NULL
  double ss;
  int use_full3d, pc_consistent, harmonic, realloc_off, surplus_redistribute, sc_head;
  double dt_init, dt_min, dt_max, dq_grow, dq_shrink, courant_max;
  double rtol, atol;
  int maxit;
  int n_bc;
  const int* bc_target;
  const int* bc_kind;
  const int* bc_form;
  const double* bc_value;
  const double* bc_eta;
  const int* bc_npts;
  const double* bc_pts;
  const char* workdir;
  const char* pc;  // "jacobi" | "icc"
} ref_case;

}  // extern "C"

namespace {

struct RefSim {
  frehg::FrehgConfig cfg;
  std::unique_ptr<frehg::Grid> grid;
  std::unique_ptr<frehg::HaloExchanger> halo;
  std::unique_ptr<frehg::gw::TerrainMetric> mesh;
  std::unique_ptr<frehg::BoundarySet> boundaries;
  std::unique_ptr<frehg::gw::RichardsSolver> gw;
  // coupled top: harness-owned GwCoupling views (ref_attach_coupling), or the
  // reference's Coupler over the stand-in surface (ref_coupler_create)
  frehg::gw::GwCoupling coupling;
  std::unique_ptr<frehg::swe::SurfaceSolver> surface;
  std::unique_ptr<frehg::coupling::Coupler> coupler;
  // density coupling: harness-owned scalar views (ref_attach_density)
  frehg::Field3<double> salt, temp;
  frehg::Field2<double> saltSurf, tempSurf;
};

std::string g_error;

void writeFlat(const std::string& path, const double* v, std::size_t n) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw frehg::FatalError("cannot write " + path);
  for (std::size_t k = 0; k < n; ++k) std::fprintf(f, "%.17g\n", v[k]);
  std::fclose(f);
}

void copyOut(const frehg::Field3<double>& f, double* out) {
  std::memcpy(out, f.data(), f.span() * sizeof(double));
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

void* ref_create(const ref_case* c) {
  try {
    frehg_shim_set_pc(c->pc ? c->pc : "");
    auto sim = std::make_unique<RefSim>();
    frehg::FrehgConfig& cfg = sim->cfg;
    const std::string dir = c->workdir ? c->workdir : ".";
    std::filesystem::create_directories(dir);
    cfg.configDir = dir;
    cfg.simulation.id = "oracle-ref";
    cfg.domain.nx = c->nx;
    cfg.domain.ny = c->ny;
    cfg.domain.nz = c->nz;
    cfg.domain.dx = c->dx;
    cfg.domain.dy = c->dy;
    cfg.domain.dz = c->dz;
    cfg.domain.dzStretch = c->dz_stretch;
    cfg.domain.followTerrain = c->follow_terrain != 0;
    cfg.domain.terrainLayers = c->terrain_uniform ? frehg::DomainConfig::TerrainLayers::Uniform
                                                  : frehg::DomainConfig::TerrainLayers::Scaled;
    const std::size_t ncol = static_cast<std::size_t>(c->nx) * static_cast<std::size_t>(c->ny);
    const std::size_t ncell = ncol * static_cast<std::size_t>(c->nz);
    if (c->bath) {
      writeFlat(dir + "/bath.dat", c->bath, ncol);
      cfg.domain.bottomElevation.fromFile = true;
      cfg.domain.bottomElevation.file = "bath.dat";
    } else {
      cfg.domain.bottomElevation.constant = 0.0;
    }
    cfg.time.dt = c->dt_init;
    cfg.time.tEnd = 1.0e9;
    cfg.time.outputInterval = 1.0e9;
    cfg.modules.groundwater = true;
    auto& gw = cfg.groundwater;
    gw.timestep.dtInit = c->dt_init;
    gw.timestep.dtMin = c->dt_min;
    gw.timestep.dtMax = c->dt_max;
    gw.timestep.dqGrow = c->dq_grow;
    gw.timestep.dqShrink = c->dq_shrink;
    gw.timestep.courantMax = c->courant_max;
    gw.specificStorage = c->ss;
    gw.useFull3d = c->use_full3d != 0;
    gw.predictorCorrector = c->pc_consistent
                                ? frehg::GroundwaterConfig::PredictorCorrector::Consistent
                                : frehg::GroundwaterConfig::PredictorCorrector::Legacy;
    gw.faceConductivity = c->harmonic ? frehg::GroundwaterConfig::FaceConductivity::Harmonic
                                      : frehg::GroundwaterConfig::FaceConductivity::Arithmetic;
    gw.reallocation = c->realloc_off ? frehg::GroundwaterConfig::Reallocation::Off
                                     : frehg::GroundwaterConfig::Reallocation::Legacy;
    gw.reallocationSurplus = c->surplus_redistribute
                                 ? frehg::GroundwaterConfig::ReallocationSurplus::Redistribute
                                 : frehg::GroundwaterConfig::ReallocationSurplus::Drop;
    gw.saturatedContact = c->sc_head ? frehg::GroundwaterConfig::SaturatedContact::Head
                                     : frehg::GroundwaterConfig::SaturatedContact::Legacy;
    cfg.solver.groundwater.rtol = c->rtol;
    cfg.solver.groundwater.atol = c->atol;
    cfg.solver.groundwater.maxIterations = c->maxit;

    cfg.soil.types.clear();
    for (int t = 0; t < c->n_soil_types; ++t) {
      const double* s = c->soil_types + 8 * t;
      frehg::SoilType st;
      st.name = "type" + std::to_string(t);
      st.ksx = s[0];
      st.ksy = s[1];
      st.ksz = s[2];
      st.thetaS = s[3];
      st.thetaR = s[4];
      st.vgAlpha = s[5];
      st.vgN = s[6];
      st.aev = s[7];
      cfg.soil.types.push_back(st);
    }
    if (c->soil_map) {
      std::vector<double> ids(ncell);
      for (std::size_t n = 0; n < ncell; ++n) ids[n] = c->soil_map[n];
      writeFlat(dir + "/soil_id.dat", ids.data(), ncell);
      cfg.soil.map.fromFile = true;
      cfg.soil.map.file = "soil_id.dat";
    } else {
      cfg.soil.map.constantName = "type0";
    }

    auto& ic = cfg.initialConditions.groundwater;
    ic.form = (c->ic_form == 0)   ? frehg::GroundwaterInitialConfig::Form::Moisture
              : (c->ic_form == 1) ? frehg::GroundwaterInitialConfig::Form::Head
                                  : frehg::GroundwaterInitialConfig::Form::WaterTable;
    if (c->ic_field) {
      writeFlat(dir + "/ic.dat", c->ic_field, c->ic_form == 2 ? ncol : ncell);
      ic.value.fromFile = true;
      ic.value.file = "ic.dat";
    } else {
      ic.value.constant = c->ic_const;
    }

    int off = 0;
    for (int b = 0; b < c->n_bc; ++b) {
      frehg::BoundaryConditionConfig bc;
      bc.name = "bc" + std::to_string(b);
      bc.target = static_cast<frehg::BcTarget>(c->bc_target[b]);
      bc.kind = static_cast<frehg::BcKind>(c->bc_kind[b]);
      bc.value.form = static_cast<frehg::BcValueConfig::Form>(c->bc_form[b]);
      bc.value.constant = c->bc_value[b];
      bc.value.hydrostaticEta = c->bc_eta[b];
      for (int p = 0; p < c->bc_npts[b]; ++p) {
        bc.polygon.push_back({c->bc_pts[2 * (off + p)], c->bc_pts[2 * (off + p) + 1]});
      }
      off += c->bc_npts[b];
      cfg.boundaryConditions.push_back(bc);
    }

    sim->grid = std::make_unique<frehg::Grid>(MPI_COMM_WORLD, cfg.domain);
    sim->halo = std::make_unique<frehg::HaloExchanger>(*sim->grid, false);
    sim->mesh = std::make_unique<frehg::gw::TerrainMetric>(*sim->grid, cfg, *sim->halo);
    sim->grid->buildGlobalIds(sim->mesh->ktop());
    sim->boundaries =
        std::make_unique<frehg::BoundarySet>(*sim->grid, cfg.boundaryConditions, cfg.configDir);
    sim->gw = std::make_unique<frehg::gw::RichardsSolver>(*sim->grid, cfg, *sim->mesh,
                                                          *sim->boundaries, *sim->halo);
    return sim.release();
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

void ref_destroy(void* h) { delete static_cast<RefSim*>(h); }

/// One RichardsSolver::step(t, dtg); t is the end-of-step time.
int ref_step(void* h, double t, double dtg) {
  try {
    static_cast<RefSim*>(h)->gw->step(t, dtg);
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

double ref_next_dt(void* h) { return static_cast<RefSim*>(h)->gw->nextDt(); }

double ref_owned_volume(void* h) { return static_cast<RefSim*>(h)->gw->ownedVolume(); }

/// audit[0..6] = boundaryIn, ssStorage, reallocAdjust, reallocDropped, vloss,
/// cplVent, pcClampVolume.
void ref_audit(void* h, double* out) {
  const auto& gw = *static_cast<RefSim*>(h)->gw;
  const auto& a = gw.audit();
  out[0] = a.boundaryIn;
  out[1] = a.ssStorage;
  out[2] = a.reallocAdjust;
  out[3] = a.reallocDropped;
  out[4] = a.vloss;
  out[5] = a.cplVent;
  out[6] = gw.pcClampVolume();
}

void ref_last_solve(void* h, int* iterations, double* residual) {
  const auto& s = static_cast<RefSim*>(h)->gw->lastSolve();
  *iterations = s.iterations;
  *residual = s.residualNorm;
}

double ref_elevation_offset(void* h) { return static_cast<RefSim*>(h)->mesh->elevationOffset(); }

/// Copy a named field out in the reference's halo layout.
int ref_get(void* h, const char* name, double* out) {
  RefSim& s = *static_cast<RefSim*>(h);
  auto& gw = *s.gw;
  auto& mesh = *s.mesh;
  const std::string n(name);
  if (n == "h") copyOut(gw.head(), out);
  else if (n == "wc") copyOut(gw.waterContent(), out);
  else if (n == "wcn") copyOut(gw.waterContentStart(), out);
  else if (n == "qx") copyOut(gw.fluxXVolumetric(), out);
  else if (n == "qy") copyOut(gw.fluxYVolumetric(), out);
  else if (n == "qz") copyOut(gw.fluxZFaceVolumetric(), out);
  else if (n == "kx") copyOut(gw.faceConductivityX(), out);
  else if (n == "ky") copyOut(gw.faceConductivityY(), out);
  else if (n == "kz") copyOut(gw.faceConductivityZFace(), out);
  else if (n == "vloss") copyOut(gw.vlossField(), out);
  else if (n == "rho") copyOut(gw.densityRatio(), out);
  else if (n == "visc") copyOut(gw.viscosityRatio(), out);
  else if (n == "rho_y") copyOut(gw.densityRatioFaceY(), out);
  else if (n == "rho_z") copyOut(gw.densityRatioFaceZ(), out);
  else if (n == "dz3d") copyOut(mesh.dz3d(), out);
  else if (n == "bot3d") copyOut(mesh.bot3d(), out);
  else if (n == "ax") copyOut(mesh.areaX(), out);
  else if (n == "ay") copyOut(mesh.areaY(), out);
  else if (n == "sinx") copyOut(mesh.sinX(), out);
  else if (n == "cosx") copyOut(mesh.cosX(), out);
  else if (n == "siny") copyOut(mesh.sinY(), out);
  else if (n == "cosy") copyOut(mesh.cosY(), out);
  else if (n == "bath") std::memcpy(out, mesh.bath().data(), mesh.bath().span() * sizeof(double));
  else {
    g_error = "unknown field " + n;
    return 1;
  }
  return 0;
}

/// Overwrite h and wc (halo layout; interiors authoritative) and rebuild the
/// derived state, as a restart read does (RichardsSolver::refreshDerivedState).
void ref_set_state(void* h, const double* head, const double* wc) {
  auto& gw = *static_cast<RefSim*>(h)->gw;
  std::memcpy(gw.head().data(), head, gw.head().span() * sizeof(double));
  std::memcpy(gw.waterContent().data(), wc, gw.waterContent().span() * sizeof(double));
  gw.refreshDerivedState();
}

/// Global ids (halo layout, -1 inactive) and the per-column ktop.
void ref_gid(void* h, int* gid, int* ktop) {
  RefSim& s = *static_cast<RefSim*>(h);
  const auto& g = s.grid->gid3Host();
  for (std::size_t n = 0; n < g.span(); ++n) gid[n] = g.data()[n];
  const auto& kt = s.mesh->ktop();
  for (std::size_t n = 0; n < kt.span(); ++n) ktop[n] = kt.data()[n];
}

/// The rasterized boundary markers, rebuilt from the BoundarySet exactly as
/// RichardsSolver::buildBoundaryLists / updateBoundaryValues do
/// (RichardsSolver.cpp:429-566), each (ny+2)*(nx+2): codes[0..5] =
/// top, bottom, xm, xp, ym, yp; values likewise at time t.
void ref_bc_masks(void* h, double t, int* codes, double* values) {
  RefSim& s = *static_cast<RefSim*>(h);
  const std::size_t n2 = static_cast<std::size_t>(s.grid->nyLocal() + 2) *
                         static_cast<std::size_t>(s.grid->nxLocal() + 2);
  const std::size_t nx2 = static_cast<std::size_t>(s.grid->nxLocal() + 2);
  std::memset(codes, 0, 6 * n2 * sizeof(int));
  std::memset(values, 0, 6 * n2 * sizeof(double));
  for (const frehg::BoundaryCondition& bc : s.boundaries->all()) {
    if (bc.target() != frehg::BcTarget::GroundwaterTop &&
        bc.target() != frehg::BcTarget::GroundwaterBottom &&
        bc.target() != frehg::BcTarget::GroundwaterSide) {
      continue;
    }
    int code = 0;
    if (bc.kind() == frehg::BcKind::Head) {
      code = (bc.valueForm() == frehg::BcValueConfig::Form::Hydrostatic) ? 4 : 1;
    } else if (bc.kind() == frehg::BcKind::Flux) {
      code = (bc.valueForm() == frehg::BcValueConfig::Form::Gravity) ? 3 : 2;
    } else {
      continue;
    }
    double v = bc.value(t);
    if (code == 4) v += s.mesh->elevationOffset();
    for (const frehg::BcCell& cell : bc.cells()) {
      frehg::BcFace face = cell.face;
      if (bc.target() == frehg::BcTarget::GroundwaterTop) face = frehg::BcFace::Top;
      if (bc.target() == frehg::BcTarget::GroundwaterBottom) face = frehg::BcFace::Bottom;
      int slot = 0;
      switch (face) {
        case frehg::BcFace::Top: slot = 0; break;
        case frehg::BcFace::Bottom: slot = 1; break;
        case frehg::BcFace::XMinus: slot = 2; break;
        case frehg::BcFace::XPlus: slot = 3; break;
        case frehg::BcFace::YMinus: slot = 4; break;
        case frehg::BcFace::YPlus: slot = 5; break;
      }
      const std::size_t at = static_cast<std::size_t>(cell.j) * nx2 + static_cast<std::size_t>(cell.i);
      codes[static_cast<std::size_t>(slot) * n2 + at] = code;
      values[static_cast<std::size_t>(slot) * n2 + at] = v;
    }
  }
}

void ref_reallocate_only(void* h) { static_cast<RefSim*>(h)->gw->reallocateWaterContent(); }

/// Attach harness-owned coupled surface views (zeroed) to the solver, as the
/// coupler's constructor does (src/coupling/Coupler.cpp:40-60).
int ref_attach_coupling(void* h, double min_depth, int vent_all, int book_bounce) {
  RefSim& s = *static_cast<RefSim*>(h);
  const std::size_t ny2 = static_cast<std::size_t>(s.grid->nyLocal()) + 2;
  const std::size_t nx2 = static_cast<std::size_t>(s.grid->nxLocal()) + 2;
  frehg::gw::GwCoupling& c = s.coupling;
  c.active = true;
  c.minDepth = min_depth;
  c.eta = frehg::Field2<double>("eta", ny2, nx2);
  c.dept = frehg::Field2<double>("dept", ny2, nx2);
  c.seepAccum = frehg::Field2<double>("seep", ny2, nx2);
  c.avail = frehg::Field2<double>("avail", ny2, nx2);
  c.gain = frehg::Field2<double>("gain", ny2, nx2);
  if (book_bounce) c.bounce = frehg::Field2<double>("bounce", ny2, nx2);
  c.ventAll = vent_all != 0;
  s.gw->attachCoupling(c);
  return 0;
}

namespace {
frehg::Field2<double> surfaceView(RefSim& s, int which) {
  if (s.coupler) {
    switch (which) {
      case 0: return s.surface->eta();
      case 1: return s.surface->depth();
      case 2: return s.coupler->seepAccum();
      case 4: return s.coupler->gain();
      case 5: return s.coupler->bounce();
      case 6: return s.coupler->seepageRate();
      case 7: return s.surface->bottom();
      case 9: return s.surface->rain();
      default: return frehg::Field2<double>();
    }
  }
  switch (which) {
    case 0: return s.coupling.eta;
    case 1: return s.coupling.dept;
    case 2: return s.coupling.seepAccum;
    case 3: return s.coupling.avail;
    case 4: return s.coupling.gain;
    case 5: return s.coupling.bounce;
    default: return frehg::Field2<double>();
  }
}
}  // namespace

/// Surface field `which` (0 eta, 1 depth, 2 seepAccum, 3 avail, 4 gain,
/// 5 bounce, 6 qss, 7 bottom, 9 rain of the stand-in surface), (ny+2)*(nx+2):
/// copied out when out is given, then overwritten from in when in is given.
int ref_surface(void* h, int which, double* out, const double* in) {
  RefSim& s = *static_cast<RefSim*>(h);
  frehg::Field2<double> v = surfaceView(s, which);
  if (!v.is_allocated()) {
    g_error = "surface field not available";
    return 1;
  }
  if (out) std::memcpy(out, v.data(), v.span() * sizeof(double));
  if (in) std::memcpy(v.data(), in, v.span() * sizeof(double));
  return 0;
}

/// cpl[0..4] = cplExchanged, cplBounce, cplVent, cplVentThin, cplEvap of the
/// last step; cpl[5] = pcClampVolume (cumulative).
void ref_coupled_audit(void* h, double* out) {
  const auto& gw = *static_cast<RefSim*>(h)->gw;
  const auto& a = gw.audit();
  out[0] = a.cplExchanged;
  out[1] = a.cplBounce;
  out[2] = a.cplVent;
  out[3] = a.cplVentThin;
  out[4] = a.cplEvap;
  out[5] = gw.pcClampVolume();
}

/// The reference's coupling::Coupler over the stand-in surface: sync or
/// subcycled, surface dt, groundwater dt_init, start time, min_depth, the
/// paired-store switch (every vent deposits).
int ref_coupler_create(void* h, int sync, double dt, double dt_init, double t_start,
                       double min_depth, int paired) {
  try {
    RefSim& s = *static_cast<RefSim*>(h);
    frehg::FrehgConfig cfg = s.cfg;
    cfg.coupling.mode = sync ? frehg::CouplingConfig::Mode::Sync
                             : frehg::CouplingConfig::Mode::Subcycled;
    cfg.time.dt = dt;
    cfg.time.tStart = t_start;
    cfg.groundwater.timestep.dtInit = dt_init;
    cfg.surfaceWater.minDepth = min_depth;
    cfg.modules.transport = false;
    const std::size_t ny2 = static_cast<std::size_t>(s.grid->nyLocal()) + 2;
    const std::size_t nx2 = static_cast<std::size_t>(s.grid->nxLocal()) + 2;
    s.surface = std::make_unique<frehg::swe::SurfaceSolver>(ny2, nx2, min_depth);
    s.surface->setPairedStore(paired != 0);
    s.coupler = std::make_unique<frehg::coupling::Coupler>(*s.grid, cfg, *s.surface, *s.gw);
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

/// Coupler::step(t, dt).  out[0..] = the CouplingAudit: gw boundaryIn,
/// ssStorage, reallocAdjust, reallocDropped, vloss, cplExchanged, cplBounce,
/// cplVent, cplVentThin, cplEvap, applied, discarded, surfaceGain,
/// accumVolume, substeps.
int ref_coupler_step(void* h, double t, double dt, double* out) {
  try {
    RefSim& s = *static_cast<RefSim*>(h);
    s.coupler->step(t, dt);
    const frehg::coupling::CouplingAudit& a = s.coupler->audit();
    const double v[] = {a.gw.boundaryIn, a.gw.ssStorage, a.gw.reallocAdjust, a.gw.reallocDropped,
                        a.gw.vloss, a.gw.cplExchanged, a.gw.cplBounce, a.gw.cplVent,
                        a.gw.cplVentThin, a.gw.cplEvap, a.applied, a.discarded, a.surfaceGain,
                        a.accumVolume, static_cast<double>(a.substeps)};
    std::memcpy(out, v, sizeof v);
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

/// RichardsSolver::enableTransportWindow / resetTransportWindow.
void ref_enable_transport_window(void* h) { static_cast<RefSim*>(h)->gw->enableTransportWindow(); }
void ref_reset_transport_window(void* h) { static_cast<RefSim*>(h)->gw->resetTransportWindow(); }

/// Window volumes: 0 windowVolumeX (qx layout), 1 windowVolumeY, 2
/// windowVolumeZ (qzF layout), 3 windowVentVolume ((ny+2)*(nx+2)).
int ref_window(void* h, int which, double* out) {
  const auto& gw = *static_cast<RefSim*>(h)->gw;
  if (which == 0) copyOut(gw.windowVolumeX(), out);
  else if (which == 1) copyOut(gw.windowVolumeY(), out);
  else if (which == 2) copyOut(gw.windowVolumeZ(), out);
  else if (which == 3)
    std::memcpy(out, gw.windowVentVolume().data(), gw.windowVentVolume().span() * sizeof(double));
  else return 1;
  return 0;
}

/// RichardsSolver::attachScalar (baroclinic on) / attachTemperature /
/// setDensityCoefficients with harness-owned scalar views, zeroed.
int ref_attach_density(void* h, int saline, int thermal, double beta_s, double beta_sv,
                       double beta_t, double t_ref, int dgrad) {
  RefSim& s = *static_cast<RefSim*>(h);
  const std::size_t ny2 = static_cast<std::size_t>(s.grid->nyLocal()) + 2;
  const std::size_t nx2 = static_cast<std::size_t>(s.grid->nxLocal()) + 2;
  const std::size_t nz = static_cast<std::size_t>(s.grid->nz());
  frehg::DensityCouplingConfig dc;
  dc.enabled = true;
  dc.betaSaline = beta_s;
  dc.betaSalineViscosity = beta_sv;
  dc.thermalExpansion = beta_t;
  dc.referenceTemperature = t_ref;
  dc.densityReallocationGradient = dgrad != 0;
  s.gw->setDensityCoefficients(dc);
  if (saline) {
    s.salt = frehg::Field3<double>("salt", ny2, nx2, nz);
    s.saltSurf = frehg::Field2<double>("salt_surf", ny2, nx2);
  }
  s.gw->attachScalar(s.salt, s.saltSurf, true);
  if (thermal) {
    s.temp = frehg::Field3<double>("temp", ny2, nx2, nz);
    s.tempSurf = frehg::Field2<double>("temp_surf", ny2, nx2);
    s.gw->attachTemperature(s.temp, s.tempSurf);
  }
  return 0;
}

/// Scalar `which` (0 salinity, 1 surface salinity, 2 temperature, 3 surface
/// temperature): copied out when out is given, then overwritten from in.
int ref_scalar(void* h, int which, double* out, const double* in) {
  RefSim& s = *static_cast<RefSim*>(h);
  double* f = nullptr;
  std::size_t n = 0;
  if (which == 0 && s.salt.size()) { f = s.salt.data(); n = s.salt.span(); }
  else if (which == 1 && s.saltSurf.size()) { f = s.saltSurf.data(); n = s.saltSurf.span(); }
  else if (which == 2 && s.temp.size()) { f = s.temp.data(); n = s.temp.span(); }
  else if (which == 3 && s.tempSurf.size()) { f = s.tempSurf.data(); n = s.tempSurf.span(); }
  if (!f) {
    g_error = "scalar not attached";
    return 1;
  }
  if (out) std::memcpy(out, f, n * sizeof(double));
  if (in) std::memcpy(f, in, n * sizeof(double));
  return 0;
}

/// Coupler::nextDt, currentDtg, gwLag(t).
void ref_coupler_state(void* h, double t, double* out) {
  const auto& c = *static_cast<RefSim*>(h)->coupler;
  out[0] = c.nextDt();
  out[1] = c.currentDtg();
  out[2] = c.gwLag(t);
}

}  // extern "C"
