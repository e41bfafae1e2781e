// Drives the C++20 RichardsSolver mirror (frehg_b200/RichardsSolver.hpp) the
// way the reference's driver loop does (Simulation::runGroundwaterLoop,
// src/driver/Simulation.cpp:1695-1700): t += nextDt(); step(t, dtg).  A
// 4x3x10 box with a ponded top and free drainage; exits non-zero unless the
// mass audit identity closes every step.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../frehg_b200/RichardsSolver.hpp"

int main() {
  const int nx = 4, ny = 3, nz = 10;
  const size_t n = static_cast<size_t>(nx) * ny * nz, ncol = static_cast<size_t>(nx) * ny;
  std::vector<double> dz(nz, 0.05), ks(n, 1e-5), alpha(n, 1.0), vgn(n, 2.0), ts(n, 0.40),
      tr(n, 0.05), aev(n, 0.0);
  std::vector<int> top(ncol, FREHG_GW_BC_HEAD), bot(ncol, FREHG_GW_BC_GRAVITY);
  std::vector<int> xs(ny, FREHG_GW_BC_NOFLUX), ys(nx, FREHG_GW_BC_NOFLUX);
  frehg_gw_desc d{};
  d.abi_version = FREHG_GW_ABI_VERSION;
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.dx = d.dy = 1.0;
  d.dz_layers = dz.data();
  d.dz_stretch = 1.0;
  d.ksx = d.ksy = d.ksz = ks.data();
  d.vg_alpha = alpha.data();
  d.vg_n = vgn.data();
  d.theta_s = ts.data();
  d.theta_r = tr.data();
  d.aev = aev.data();
  d.specific_storage = 1e-5;
  d.top_code = top.data();
  d.bot_code = bot.data();
  d.xm_code = d.xp_code = xs.data();
  d.ym_code = d.yp_code = ys.data();
  d.use_full3d = 1;
  d.pc_consistent = 1;
  d.saturated_contact_head = 1;
  d.dt_init = 10.0;
  d.dt_min = 1e-3;
  d.dt_max = 600.0;
  d.dq_grow = 0.01;
  d.dq_shrink = 0.02;
  d.courant_max = 2.0;
  d.rtol = 1e-8;
  d.atol = 1e-14;
  d.max_iterations = 1000;
  d.precision = FREHG_GW_PRECISION_FP64;
  try {
    frehg_b200::RichardsSolver gw(d, FREHG_GW_IC_HEAD, -1.0);
    std::vector<double> pond(ncol, 0.01), zero(ncol, 0.0);
    gw.setBoundaryValues(pond.data(), zero.data(), nullptr, nullptr, nullptr, nullptr);
    double t = 0.0, prev = gw.ownedVolume();
    for (int s = 0; s < 5; ++s) {
      const double dtg = gw.nextDt();
      t += dtg;
      gw.step(t, dtg);
      const double v = gw.ownedVolume();
      const auto& a = gw.audit();
      const double resid =
          (v - prev) - (a.boundaryIn - a.ssStorage + a.reallocAdjust - a.vloss);
      std::printf("step %d dtg %.4g its %d volume %.12g audit residual %.3e\n", s, dtg,
                  gw.lastSolve().iterations, v, resid);
      if (!(std::fabs(resid) <= 1e-12 * std::fmax(v, 1.0))) return 2;
      prev = v;
    }
    // The coupled top under the Coupler mirror: a 2 cm pond over the box,
    // sync windows of 5 s, the surface a stand-in without lateral flow (its
    // depth refreshed from eta before each window).  The coupled budget
    // closes: d(V_gw + V_surface + held seepage) = the external boundary
    // inflow + bounce - evaporation - Ss storage + reallocation - clamp loss
    // + the infiltration the bed clamp could not take from the surface.
    std::vector<int> flux_top(ncol, FREHG_GW_BC_FLUX);
    d.top_code = flux_top.data();
    frehg_b200::RichardsSolver cg(d, FREHG_GW_IC_HEAD, -1.0);
    frehg_gw_coupling c{};
    c.min_depth = 1e-3;
    cg.attachCoupling(c);
    const size_t n2 = static_cast<size_t>(nx + 2) * (ny + 2);
    const double off = frehg_gw_elevation_offset(cg.handle());
    std::vector<double> bottom(n2, off), eta(n2, off + 0.02), dep(n2, 0.02);
    cg.setSurface(FREHG_GW_SURF_BOTTOM, bottom.data());
    cg.setSurface(FREHG_GW_SURF_ETA, eta.data());
    frehg_b200::Coupler cp(cg, true, 5.0, 5.0);
    auto surface_volume = [&](const std::vector<double>& e, const std::vector<double>& acc) {
      double v = 0.0;
      for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          const size_t k = static_cast<size_t>(j) * (nx + 2) + i;
          v += (e[k] - bottom[k]) + acc[k];
        }
      return v * d.dx * d.dy;
    };
    double total = cg.ownedVolume() + surface_volume(eta, cg.surface(FREHG_GW_SURF_SEEP_ACCUM));
    double tc = 0.0;
    for (int w = 0; w < 6; ++w) {
      const double dt = cp.nextDt();
      tc += dt;
      eta = cg.surface(FREHG_GW_SURF_ETA);
      for (size_t k = 0; k < n2; ++k) {
        const double dd = eta[k] - bottom[k];
        dep[k] = dd <= c.min_depth ? 0.0 : dd;
      }
      cg.setSurface(FREHG_GW_SURF_DEPTH, dep.data());
      cp.step(tc, dt);
      const auto& a = cp.audit();
      const double now = cg.ownedVolume() + surface_volume(cg.surface(FREHG_GW_SURF_ETA),
                                                           cg.surface(FREHG_GW_SURF_SEEP_ACCUM));
      const double src = (a.gw.boundary_in + a.cpl.exchanged + a.cpl.vent) + a.cpl.bounce -
                         a.cpl.evap - a.gw.ss_storage + a.gw.realloc_adjust - a.gw.vloss +
                         a.discarded;
      const double resid = (now - total) - src;
      std::printf("window %d dt %.4g substeps %ld exchanged %.4e applied %.4e residual %.3e\n", w,
                  dt, a.substeps, a.cpl.exchanged, a.applied, resid);
      if (!(std::fabs(resid) <= 1e-12 * std::fmax(now, 1.0))) return 3;
      if (!(a.cpl.exchanged < 0.0)) return 4;  // the pond infiltrates
      total = now;
    }
  } catch (const frehg_b200::FatalError& e) {
    std::fprintf(stderr, "FatalError(%d): %s\n", e.status(), e.what());
    return 1;
  }
  return 0;
}
