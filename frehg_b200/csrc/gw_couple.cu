// The coupled top of the groundwater step and the coupler window around it
// (include/frehg_gw.h, "coupled top").  The step's coupled branches live in
// the kernels (gw_kernels.cu: k_cpl_mode, the coupled face / assembly /
// flux / classification / walk rules, k_cpl_book); this file attaches the
// surface fields, moves them to and from the host and runs the subsurface
// part of coupling::Coupler::step (src/coupling/Coupler.cpp:69-131,
// Exchange.cpp:21-127) over frehg_gw_step.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "gw_handle.h"

using fgw_api::cuda_fail;
using fgw_api::fail;

#define CUDA_TRY(call, what)                           \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

namespace {

constexpr int kSurfFields = 8;  // FREHG_GW_SURF_ETA .. FREHG_GW_SURF_BOTTOM

int need_coupling(const frehg_gw_handle* h) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  if (!h->D.f.cpl) return fail(FREHG_GW_ESTATE, "no coupling attached (frehg_gw_attach_coupling)");
  return FREHG_GW_OK;
}

}  // namespace

extern "C" {

int frehg_gw_attach_coupling(frehg_gw_handle* h, const frehg_gw_coupling* c) {
  if (!h || !c) return fail(FREHG_GW_EINVAL, "attach_coupling: null argument");
  FGW_ON_DEVICE(h);
  if (!(c->min_depth >= 0.0) || !std::isfinite(c->min_depth))
    return fail(FREHG_GW_EINVAL, "attach_coupling: min_depth must be finite and >= 0");
  fgw::Device& D = h->D;
  const size_t n2 = static_cast<size_t>(D.d.ncol);
  CUDA_TRY(cudaStreamSynchronize(D.stream), "attach_coupling");
  for (int w = 0; w < kSurfFields; ++w) {
    if (c->field[w]) {
      D.surf[w] = c->field[w];
      D.surf_own[w] = false;
    } else if (!D.surf[w] || !D.surf_own[w]) {
      void* p = nullptr;
      const cudaError_t e = cudaMalloc(&p, n2 * sizeof(double));
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FREHG_GW_ENOMEM, "attach_coupling: surface field allocation failed");
      }
      D.allocs.push_back(p);
      CUDA_TRY(cudaMemsetAsync(p, 0, n2 * sizeof(double), D.stream), "attach_coupling");
      D.surf[w] = static_cast<double*>(p);
      D.surf_own[w] = true;
    }
  }
  if (!D.cmode) {
    void* p = nullptr;
    if (cudaMalloc(&p, n2) != cudaSuccess) {
      cudaGetLastError();
      return fail(FREHG_GW_ENOMEM, "attach_coupling: mode allocation failed");
    }
    D.allocs.push_back(p);
    CUDA_TRY(cudaMemsetAsync(p, 0, n2, D.stream), "attach_coupling");
    D.cmode = static_cast<int8_t*>(p);
  }
  if (!D.cpl_dev) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(fgw::CplDev)) != cudaSuccess) {
      cudaGetLastError();
      return fail(FREHG_GW_ENOMEM, "attach_coupling: allocation failed");
    }
    D.allocs.push_back(p);
    D.cpl_dev = static_cast<fgw::CplDev*>(p);
  }
  fgw::CplDev& k = D.cpl_host;
  k.vent_all = c->vent_all != 0;
  k.book_bounce = c->book_bounce != 0;
  k.min_depth = c->min_depth;
  k.bath = h->bath_dev;
  k.eta = D.surf[FREHG_GW_SURF_ETA];
  k.dept = D.surf[FREHG_GW_SURF_DEPTH];
  k.seep = D.surf[FREHG_GW_SURF_SEEP_ACCUM];
  k.avail = D.surf[FREHG_GW_SURF_AVAIL];
  k.gain = D.surf[FREHG_GW_SURF_GAIN];
  k.bounce = D.surf[FREHG_GW_SURF_BOUNCE];
  k.cmode = D.cmode;
  CUDA_TRY(cudaMemcpyAsync(D.cpl_dev, &k, sizeof(k), cudaMemcpyHostToDevice, D.stream),
           "attach_coupling");
  D.f.cpl = D.cpl_dev;
  h->cpl_last = frehg_gw_coupled_audit{};
  CUDA_TRY(cudaStreamSynchronize(D.stream), "attach_coupling");
  return FREHG_GW_OK;
}

int frehg_gw_get_surface(frehg_gw_handle* h, int which, double* host_out) {
  if (int rc = need_coupling(h)) return rc;
  FGW_ON_DEVICE(h);
  if (!host_out) return fail(FREHG_GW_EINVAL, "get_surface: null output");
  fgw::Device& D = h->D;
  const size_t n2 = static_cast<size_t>(D.d.ncol);
  if (which == FREHG_GW_SURF_MODE) {
    std::vector<int8_t> m(n2);
    CUDA_TRY(cudaMemcpyAsync(m.data(), D.cmode, n2, cudaMemcpyDeviceToHost, D.stream),
             "get_surface");
    CUDA_TRY(cudaStreamSynchronize(D.stream), "get_surface");
    for (size_t n = 0; n < n2; ++n) host_out[n] = m[n];
    return FREHG_GW_OK;
  }
  if (which < 0 || which >= kSurfFields) return fail(FREHG_GW_EINVAL, "get_surface: bad field");
  CUDA_TRY(cudaMemcpyAsync(host_out, D.surf[which], n2 * sizeof(double), cudaMemcpyDeviceToHost,
                           D.stream), "get_surface");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "get_surface");
  return FREHG_GW_OK;
}

int frehg_gw_set_surface(frehg_gw_handle* h, int which, const double* host_in) {
  if (int rc = need_coupling(h)) return rc;
  FGW_ON_DEVICE(h);
  if (!host_in) return fail(FREHG_GW_EINVAL, "set_surface: null input");
  if (which < 0 || which >= kSurfFields)
    return fail(FREHG_GW_EINVAL, "set_surface: bad or read-only field");
  fgw::Device& D = h->D;
  CUDA_TRY(cudaMemcpyAsync(D.surf[which], host_in, static_cast<size_t>(D.d.ncol) * sizeof(double),
                           cudaMemcpyHostToDevice, D.stream), "set_surface");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "set_surface");
  return FREHG_GW_OK;
}

int frehg_gw_surface_ptr(frehg_gw_handle* h, int which, double** dev_out) {
  if (int rc = need_coupling(h)) return rc;
  if (!dev_out || which < 0 || which >= kSurfFields)
    return fail(FREHG_GW_EINVAL, "surface_ptr: bad argument");
  *dev_out = h->D.surf[which];
  return FREHG_GW_OK;
}

int frehg_gw_coupled_audit_get(frehg_gw_handle* h, frehg_gw_coupled_audit* out) {
  if (int rc = need_coupling(h)) return rc;
  if (!out) return fail(FREHG_GW_EINVAL, "coupled_audit: null output");
  *out = h->cpl_last;
  return FREHG_GW_OK;
}

double frehg_gw_elevation_offset(const frehg_gw_handle* h) { return h ? h->offset : 0.0; }

int frehg_gw_coupler_init(frehg_gw_handle* h, const frehg_gw_coupler_opts* o) {
  if (int rc = need_coupling(h)) return rc;
  FGW_ON_DEVICE(h);
  if (!o) return fail(FREHG_GW_EINVAL, "coupler_init: null options");
  const double first = o->sync ? o->dt : o->dt_init;
  if (!(o->dt > 0.0) || !(first > 0.0))
    return fail(FREHG_GW_EINVAL, "coupler_init: dt (and dt_init when subcycled) must be positive");
  h->coupler = true;
  h->csync = o->sync != 0;
  h->cdt = o->dt;
  h->cdtg = first;
  h->ctsub = o->t_start;
  return FREHG_GW_OK;
}

int frehg_gw_coupler_step(frehg_gw_handle* h, double t, double dt, frehg_gw_window_audit* out) {
  if (int rc = need_coupling(h)) return rc;
  FGW_ON_DEVICE(h);
  if (!h->coupler) return fail(FREHG_GW_ESTATE, "coupler_step before frehg_gw_coupler_init");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(FREHG_GW_EINVAL, "coupler_step: dt <= 0");
  fgw::Device& D = h->D;
  frehg_gw_window_audit a{};
  fgw::launch_cpl_begin_window(D);
  CUDA_TRY(cudaGetLastError(), "coupler window");
  for (;;) {
    double tt, dtg;
    if (h->csync) {
      if (a.substeps > 0) break;
      h->ctsub = t;
      tt = t;
      dtg = dt;
    } else {
      // Coupler.cpp:106-112: advance while a whole dtg fits
      if (!(h->ctsub + h->cdtg <= t + 1.0e-9)) break;
      h->ctsub += h->cdtg;
      tt = h->ctsub;
      dtg = h->cdtg;
    }
    frehg_gw_step_info info{};
    const int rc = frehg_gw_step(h, tt, dtg, &info);
    if (rc != FREHG_GW_OK) return rc;
    h->cdtg = h->next_dt;
    a.gw.boundary_in += info.boundary_in;
    a.gw.ss_storage += info.ss_storage;
    a.gw.realloc_adjust += info.realloc_adjust;
    a.gw.realloc_dropped += info.realloc_dropped;
    a.gw.vloss += info.vloss;
    a.gw.cg_iterations += info.cg_iterations;
    a.gw.outer_iterations += info.outer_iterations;
    a.cpl.exchanged += h->cpl_last.exchanged;
    a.cpl.bounce += h->cpl_last.bounce;
    a.cpl.vent += h->cpl_last.vent;
    a.cpl.vent_thin += h->cpl_last.vent_thin;
    a.cpl.evap += h->cpl_last.evap;
    ++a.substeps;
  }
  a.cpl.pc_clamp_volume = h->pc_clamp_total;
  a.gw.next_dt = h->cdtg;
  fgw::launch_cpl_seepage(D, dt);
  CUDA_TRY(cudaMemcpyAsync(D.out_host->win, D.out->win, sizeof(D.out->win),
                           cudaMemcpyDeviceToHost, D.stream), "coupler seepage");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "coupler seepage");
  CUDA_TRY(cudaGetLastError(), "coupler seepage");
  const double cell = D.d.dx * D.d.dy;
  a.applied = D.out_host->win[0] * cell;
  a.discarded = D.out_host->win[1] * cell;
  a.surface_gain = D.out_host->win[2] * cell;
  a.accum_volume = D.out_host->win[3] * cell;
  if (out) *out = a;
  return FREHG_GW_OK;
}

int frehg_gw_coupler_state(frehg_gw_handle* h, double t, double* next_dt, double* dtg,
                           double* lag) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  if (!h->coupler) return fail(FREHG_GW_ESTATE, "coupler_state before frehg_gw_coupler_init");
  if (next_dt) *next_dt = h->csync ? h->cdtg : h->cdt;
  if (dtg) *dtg = h->cdtg;
  if (lag) *lag = h->csync ? 0.0 : (t - h->ctsub);
  return FREHG_GW_OK;
}

int frehg_gw_coupler_restore(frehg_gw_handle* h, double t, double dtg, double lag) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  if (!h->coupler) return fail(FREHG_GW_ESTATE, "coupler_restore before frehg_gw_coupler_init");
  if (!(dtg > 0.0)) return fail(FREHG_GW_EINVAL, "coupler_restore: dtg must be positive");
  h->cdtg = dtg;
  h->ctsub = t - lag;
  return FREHG_GW_OK;
}

}  // extern "C"
