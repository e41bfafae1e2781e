// The C ABI of the B200 groundwater step (include/frehg_gw.h): handle
// lifetime, device memory, and the per-step orchestration of the kernels in
// gw_kernels.cu and gw_cg.cu.  No exception crosses the ABI; every entry
// point returns a frehg_gw_status and records a message for
// frehg_gw_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/frehg_gw.h"
#include "gw_internal.h"
#include "gw_setup.h"

#include "gw_handle.h"

namespace {
thread_local std::string g_error;
}  // namespace

namespace fgw_api {

int fail(int status, const std::string& msg) {
  g_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(FREHG_GW_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace fgw_api

namespace {

using fgw_api::cuda_fail;
using fgw_api::fail;

#define CUDA_TRY(call, what)                    \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// Every device array of a domain is a 256-byte-aligned slice of one arena
// allocation: create runs its allocation sequence twice, first to size the
// arena (plan), then to hand out the slices.  One allocation avoids the
// page rounding of many mid-sized ones and makes the footprint
// frehg_gw_device_bytes reports exact up to that alignment.
template <class T>
cudaError_t dalloc(fgw::Device& D, T** p, size_t n) {
  const size_t bytes = ((n ? n : 1) * sizeof(T) + 255) & ~static_cast<size_t>(255);
  if (D.arena_plan) {
    D.arena_bytes += bytes;
    *p = nullptr;
    return cudaSuccess;
  }
  if (!D.arena || D.arena_off + bytes > D.arena_bytes) return cudaErrorMemoryAllocation;
  *p = reinterpret_cast<T*>(D.arena + D.arena_off);
  D.arena_off += bytes;
  return cudaSuccess;
}

// Solver arrays carry a zero margin of one j-row on both ends.
template <class T>
cudaError_t dalloc_margin(fgw::Device& D, T** p, long long ncell, long long margin) {
  T* base = nullptr;
  cudaError_t e = dalloc(D, &base, static_cast<size_t>(ncell + 2 * margin));
  *p = base ? base + margin : nullptr;
  return e;
}

void free_device(fgw::Device& D) {
  for (void* p : D.allocs) cudaFree(p);
  D.allocs.clear();
  if (D.out_host) cudaFreeHost(D.out_host);
  D.out_host = nullptr;
  if (D.own_stream && D.stream) cudaStreamDestroy(D.stream);
  D.stream = nullptr;
}

}  // namespace

extern "C" {

const char* frehg_gw_last_error(void) { return g_error.c_str(); }

int frehg_gw_create(const frehg_gw_desc* desc, frehg_gw_handle** out) {
  g_error.clear();
  if (!desc || !out) return fail(FREHG_GW_EINVAL, "frehg_gw_create: null argument");
  *out = nullptr;
  try {
    fgw::HostDomain H;
    std::string err;
    const int rc = fgw::build_host_domain(*desc, H, err);
    if (rc != FREHG_GW_OK) return fail(rc, "frehg_gw_create: " + err);
    if (desc->precision != FREHG_GW_PRECISION_FP64 && desc->precision != FREHG_GW_PRECISION_MIXED &&
        desc->precision != FREHG_GW_PRECISION_FP64_LINE)
      return fail(FREHG_GW_EINVAL, "frehg_gw_create: unknown precision");
    if (desc->precision == FREHG_GW_PRECISION_FP64_LINE && desc->nz > 256)
      return fail(FREHG_GW_EUNSUPPORTED, "frehg_gw_create: the FP64 line form takes nz <= 256");
    if (!(desc->rtol >= 0.0) || !(desc->atol >= 0.0) || desc->max_iterations < 1)
      return fail(FREHG_GW_EINVAL, "frehg_gw_create: invalid solver tolerances");

    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    int coop = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "attribute");
    if (!coop) return fail(FREHG_GW_ECUDA, "device lacks cooperative launch");

    auto* hnd = new frehg_gw_handle();
    hnd->device = dev;
    fgw::Device& D = hnd->D;
    CUDA_TRY(cudaDeviceGetAttribute(&D.sm_count, cudaDevAttrMultiProcessorCount, dev), "sm");
    CUDA_TRY(cudaStreamCreateWithFlags(&D.stream, cudaStreamNonBlocking), "stream");
    D.own_stream = true;

    fgw::Dims& d = D.d;
    d.nx = H.nx;
    d.ny = H.ny;
    d.nz = H.nz;
    d.nx2 = H.nx + 2;
    d.ny2 = H.ny + 2;
    d.sx = H.nz;
    d.sy = static_cast<long long>(H.nx + 2) * H.nz;
    d.ncell = H.ncell;
    d.ncol = H.ncol;
    d.mz = fgw::div_magic(static_cast<unsigned>(H.nz));
    d.mx2 = fgw::div_magic(static_cast<unsigned>(H.nx + 2));
    d.dx = desc->dx;
    d.dy = desc->dy;
    d.az = desc->dx * desc->dy;
    d.idx = 1.0 / desc->dx;
    d.idy = 1.0 / desc->dy;
    d.ss = desc->specific_storage;
    d.full3d = desc->use_full3d ? 1 : 0;
    d.pc = desc->pc_consistent ? 1 : 0;
    d.harm = (desc->pc_consistent && desc->face_harmonic) ? 1 : 0;
    d.off = desc->reallocation_off ? 1 : 0;
    d.redistribute = desc->surplus_redistribute ? 1 : 0;
    d.terrain = desc->follow_terrain ? 1 : 0;

    int soil_kind[8];
    double soil_u[8] = {};
    for (int f = 0; f < 8; ++f) soil_kind[f] = fgw::soil_storage(*desc, f, &soil_u[f]);
    // Allocation sequence, run twice (see dalloc): plan, then slices.
    auto allocate = [&]() -> cudaError_t {
      const long long n3 = d.ncell, nf = d.ncol * (d.nz + 1), m = d.sy;
      auto up = [&](double** p, const std::vector<double>& v) -> cudaError_t {
        cudaError_t e = dalloc(D, p, v.size());
        if (e != cudaSuccess || D.arena_plan) return e;
        return cudaMemcpy(*p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
      };
      cudaError_t e = cudaSuccess;
      double** soil[8] = {&D.ksx, &D.ksy, &D.ksz, &D.vga, &D.vgn, &D.wcs, &D.wcr, &D.aev};
      for (int f = 0; f < 8 && e == cudaSuccess; ++f) {
        const int g = soil_kind[f];
        if (g == fgw::kSoilUniform) e = up(soil[f], std::vector<double>(1, soil_u[f]));
        else if (g >= 0) *soil[f] = *soil[g];  // equal bytes: one array for both
        else e = up(soil[f], H.soil[f]);
      }
      if (e == cudaSuccess) e = up(&D.dz, H.dz);
      if (e == cudaSuccess) e = up(&D.bot, H.bot);
      if (e == cudaSuccess) e = up(&D.ax, H.ax);
      if (e == cudaSuccess) e = up(&D.ay, H.ay);
      if (e == cudaSuccess) e = up(&D.sinx, H.sinx);
      if (e == cudaSuccess) e = up(&D.cosx, H.cosx);
      if (e == cudaSuccess) e = up(&D.siny, H.siny);
      if (e == cudaSuccess) e = up(&D.cosy, H.cosy);
      if (e == cudaSuccess) e = up(&hnd->bath_dev, H.bath);
      if (e == cudaSuccess) e = dalloc(D, &D.act, static_cast<size_t>(n3));
      if (e == cudaSuccess && !D.arena_plan)
        e = cudaMemcpy(D.act, H.act.data(), static_cast<size_t>(n3), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = dalloc(D, &D.codes, 6 * static_cast<size_t>(d.ncol));
      if (e == cudaSuccess && !D.arena_plan)
        e = cudaMemcpy(D.codes, H.codes.data(), H.codes.size() * sizeof(int), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = dalloc(D, &D.values, 6 * static_cast<size_t>(d.ncol));
      // Zero like the host staging copy: every later upload keeps the two
      // equal entry for entry (frehg_gw_set_bc_values relies on it).
      if (e == cudaSuccess && !D.arena_plan)
        e = cudaMemset(D.values, 0, 6 * static_cast<size_t>(d.ncol) * sizeof(double));
      for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = dalloc(D, &D.h[b], n3);
        if (e == cudaSuccess) e = dalloc(D, &D.wc[b], n3);
      }
      double** cellf[] = {&D.hp, &D.wcu, &D.ch, &D.kcx, &D.kcy, &D.kcz, &D.kx, &D.ky, &D.qx, &D.qy,
                          &D.vloss, &D.room, &D.sup, &D.sdn};
      for (double** p : cellf)
        if (e == cudaSuccess) e = dalloc(D, p, n3);
      if (e == cudaSuccess) e = dalloc(D, &D.kzf, nf);
      if (e == cudaSuccess) e = dalloc(D, &D.qzf, nf);
      if (e == cudaSuccess) e = dalloc(D, &D.colflag, d.ncol);
      if (e == cudaSuccess) e = dalloc(D, &D.satf, n3);
      double** solv[] = {&D.diag, &D.gxp, &D.gyp, &D.gzp, &D.rhs, &D.x, &D.r, &D.z, &D.p0, &D.p1, &D.w};
      for (double** p : solv)
        if (e == cudaSuccess) e = dalloc_margin(D, p, n3, m);
      if (desc->precision == FREHG_GW_PRECISION_MIXED) {
        float** solv32[] = {&D.diag32, &D.gxp32, &D.gyp32, &D.gzp32, &D.dinv32, &D.l32,
                            &D.r32,    &D.z32,   &D.d32,   &D.p032,  &D.p132, &D.w32};
        for (float** p : solv32)
          if (e == cudaSuccess) e = dalloc_margin(D, p, n3, m);
        if (e == cudaSuccess) e = dalloc_margin(D, &D.xalt, n3, m);
      }
      if (desc->precision == FREHG_GW_PRECISION_FP64_LINE) {
        double** line64[] = {&D.dinv64, &D.l64, &D.d64, &D.xalt};
        for (double** p : line64)
          if (e == cudaSuccess) e = dalloc_margin(D, p, n3, m);
      }
      // Diagonal 1 everywhere outside the active rows (ghosts, margins), so the
      // Jacobi scaling of those always-zero entries stays finite.
      if (e == cudaSuccess && !D.arena_plan) {
        std::vector<double> ones(static_cast<size_t>(n3 + 2 * m), 1.0);
        e = cudaMemcpy(D.diag - m, ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && D.diag32) {
          std::vector<float> onesf(ones.size(), 1.0f);
          e = cudaMemcpy(D.diag32 - m, onesf.data(), onesf.size() * sizeof(float),
                         cudaMemcpyHostToDevice);
        }
      }
      D.nblk = static_cast<int>(std::min<long long>((n3 + fgw::kBlock - 1) / fgw::kBlock,
                                                    static_cast<long long>(D.sm_count) * 8));
      if (D.nblk < 1) D.nblk = 1;
      D.cg_grid = fgw::cg64_grid(D.sm_count, n3);
      D.cg_grid32 = D.sm_count * 4;
      if (e == cudaSuccess)
        e = dalloc(D, &D.partial, static_cast<size_t>(fgw::kPSlots) * D.nblk);
      if (e == cudaSuccess)
        e = dalloc(D, &D.cgpart, 4 * static_cast<size_t>(std::max(D.cg_grid, D.cg_grid32)));
      if (e == cudaSuccess) e = dalloc(D, &D.out, 1);
      return e;
    };
    D.arena_plan = true;
    cudaError_t e = allocate();
    D.arena_plan = false;
    if (e == cudaSuccess) e = cudaMalloc(&D.arena, D.arena_bytes);
    if (e == cudaSuccess) {
      D.allocs.push_back(D.arena);
      e = cudaMemset(D.arena, 0, D.arena_bytes);
    }
    if (e == cudaSuccess) e = allocate();
    if (e == cudaSuccess) e = cudaMallocHost(&D.out_host, sizeof(fgw::StepOut));
    if (e != cudaSuccess) {
      free_device(D);
      delete hnd;
      return fail(e == cudaErrorMemoryAllocation ? FREHG_GW_ENOMEM : FREHG_GW_ECUDA,
                  std::string("frehg_gw_create: ") + cudaGetErrorString(e));
    }

    fgw::Fields& f = D.f;
    {
      const double* sp[8] = {D.ksx, D.ksy, D.ksz, D.vga, D.vgn, D.wcs, D.wcr, D.aev};
      fgw::SoilField* sf[8] = {&f.ksx, &f.ksy, &f.ksz, &f.vga, &f.vgn, &f.wcs, &f.wcr, &f.aev};
      for (int q = 0; q < 8; ++q)
        *sf[q] = fgw::SoilField{sp[q], soil_kind[q] == fgw::kSoilUniform ? 0LL : ~0LL};
    }
    f.dz = D.dz;
    f.bot = D.bot;
    f.ax = D.ax;
    f.ay = D.ay;
    f.sinx = D.sinx;
    f.cosx = D.cosx;
    f.siny = D.siny;
    f.cosy = D.cosy;
    f.act = D.act;
    f.topc = D.codes;
    f.botc = D.codes + d.ncol;
    f.xmc = D.codes + 2 * d.ncol;
    f.xpc = D.codes + 3 * d.ncol;
    f.ymc = D.codes + 4 * d.ncol;
    f.ypc = D.codes + 5 * d.ncol;
    f.topv = D.values;
    f.botv = D.values + d.ncol;
    f.xmv = D.values + 2 * d.ncol;
    f.xpv = D.values + 3 * d.ncol;
    f.ymv = D.values + 4 * d.ncol;
    f.ypv = D.values + 5 * d.ncol;

    hnd->offset = H.offset;
    hnd->nactive = H.nactive;
    hnd->codes = H.codes;
    hnd->values.assign(6 * static_cast<size_t>(d.ncol), 0.0);
    // Page-lock the boundary-value staging so each step's upload is a direct
    // DMA; without it (registration refused) the copy still works, staged.
    hnd->values_pinned = cudaHostRegister(hnd->values.data(), hnd->values.size() * sizeof(double),
                                          cudaHostRegisterDefault) == cudaSuccess;
    if (!hnd->values_pinned) cudaGetLastError();
    hnd->rtol = desc->rtol;
    hnd->atol = desc->atol;
    hnd->maxit = desc->max_iterations;
    hnd->precision = desc->precision;
    hnd->outer_rtol = desc->outer_rtol > 0 ? desc->outer_rtol : 3e-12;
    hnd->max_outer = desc->max_outer > 0 ? desc->max_outer : 30;
    hnd->dt_min = desc->dt_min;
    hnd->dt_max = desc->dt_max;
    hnd->dq_grow = desc->dq_grow;
    hnd->dq_shrink = desc->dq_shrink;
    hnd->co_max = desc->courant_max;
    hnd->next_dt = desc->dt_init;
    CUDA_TRY(cudaDeviceSynchronize(), "frehg_gw_create");
    *out = hnd;
    return FREHG_GW_OK;
  } catch (const std::exception& ex) {
    return fail(FREHG_GW_ENOMEM, std::string("frehg_gw_create: ") + ex.what());
  }
}

int frehg_gw_destroy(frehg_gw_handle* h) {
  if (!h) return FREHG_GW_OK;
  FGW_ON_DEVICE(h);
  cudaStreamSynchronize(h->D.stream);
  for (cudaEvent_t& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->values_pinned) cudaHostUnregister(h->values.data());
  free_device(h->D);
  delete h;
  return FREHG_GW_OK;
}

int frehg_gw_set_stream(frehg_gw_handle* h, void* stream) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  CUDA_TRY(cudaStreamSynchronize(h->D.stream), "set_stream");
  if (h->D.own_stream) cudaStreamDestroy(h->D.stream);
  if (stream) {
    h->D.stream = static_cast<cudaStream_t>(stream);
    h->D.own_stream = false;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&h->D.stream, cudaStreamNonBlocking), "stream");
    h->D.own_stream = true;
  }
  return FREHG_GW_OK;
}

int frehg_gw_set_bc_values(frehg_gw_handle* h, const double* top, const double* bot,
                           const double* xm, const double* xp, const double* ym, const double* yp) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  const long long nc = d.ncol;
  const double off = h->offset;
  bool bad = false;
  // Interior row j of a per-column slot from the caller's (ny, nx) array.
  auto row = [&](int slot, const double* src, int j) {
    const long long base = slot * nc + fgw::col2(d, j, 1);
    const int* cd = h->codes.data() + base;
    double* dst = h->values.data() + base;
    const double* sr = src + static_cast<long long>(j - 1) * d.nx;
    bool b = false;
    for (int i = 0; i < d.nx; ++i) {
      const double v = sr[i] + (cd[i] == FREHG_GW_BC_HEAD_HYDROSTATIC ? off : 0.0);
      dst[i] = v;
      b |= !std::isfinite(v);
    }
    bad |= b;
  };
  auto put = [&](int slot, long long col, double v) {
    const int code = h->codes[slot * nc + col];
    v += (code == FREHG_GW_BC_HEAD_HYDROSTATIC ? off : 0.0);
    h->values[slot * nc + col] = v;
    bad |= !std::isfinite(v);
  };
  for (int j = 1; j <= d.ny; ++j) {
    if (top) row(0, top, j);
    if (bot) row(1, bot, j);
    if (xm) put(2, fgw::col2(d, j, 1), xm[j - 1]);
    if (xp) put(3, fgw::col2(d, j, d.nx), xp[j - 1]);
  }
  for (int i = 1; i <= d.nx; ++i) {
    if (ym) put(4, fgw::col2(d, 1, i), ym[i - 1]);
    if (yp) put(5, fgw::col2(d, d.ny, i), yp[i - 1]);
  }
  if (bad) {
    // A rejected call changes nothing: the touched slots of the staging copy
    // are read back from the device, which holds the last accepted values
    // (the two are equal entry for entry after every accepted call).
    const double* src[6] = {top, bot, xm, xp, ym, yp};
    for (int slot = 0; slot < 6; ++slot) {
      if (!src[slot]) continue;
      CUDA_TRY(cudaMemcpyAsync(h->values.data() + slot * nc, D.values + slot * nc,
                               static_cast<size_t>(nc) * sizeof(double), cudaMemcpyDeviceToHost,
                               D.stream), "set_bc_values");
    }
    CUDA_TRY(cudaStreamSynchronize(D.stream), "set_bc_values");
    return fail(FREHG_GW_EINVAL, "non-finite boundary value");
  }
  // Upload what the kernels read: the top and bottom slots whole, the side
  // slots' edge entries (a column of the x edges, a row of the y edges).
  const size_t w = sizeof(double), pitch = static_cast<size_t>(d.nx2) * w;
  auto slot1d = [&](int slot, long long col, size_t n) {
    return cudaMemcpyAsync(D.values + slot * nc + col, h->values.data() + slot * nc + col, n * w,
                           cudaMemcpyHostToDevice, D.stream);
  };
  auto xedge = [&](int slot, int i) {
    const long long col = fgw::col2(d, 1, i);
    return cudaMemcpy2DAsync(D.values + slot * nc + col, pitch, h->values.data() + slot * nc + col,
                             pitch, w, static_cast<size_t>(d.ny), cudaMemcpyHostToDevice, D.stream);
  };
  if (top) CUDA_TRY(slot1d(0, 0, static_cast<size_t>(nc)), "set_bc_values");
  if (bot) CUDA_TRY(slot1d(1, 0, static_cast<size_t>(nc)), "set_bc_values");
  if (xm) CUDA_TRY(xedge(2, 1), "set_bc_values");
  if (xp) CUDA_TRY(xedge(3, d.nx), "set_bc_values");
  if (ym) CUDA_TRY(slot1d(4, fgw::col2(d, 1, 1), static_cast<size_t>(d.nx)), "set_bc_values");
  if (yp) CUDA_TRY(slot1d(5, fgw::col2(d, d.ny, 1), static_cast<size_t>(d.nx)), "set_bc_values");
  // Landed before returning: a batch or a server steps the member on a
  // stream of its own, and the staging is free for the next call.
  CUDA_TRY(cudaStreamSynchronize(D.stream), "set_bc_values");
  return FREHG_GW_OK;
}

int frehg_gw_init_state(frehg_gw_handle* h, int form, double constant, const double* field) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  h->have_prev = false;
  if (form < FREHG_GW_IC_MOISTURE || form > FREHG_GW_IC_WATER_TABLE)
    return fail(FREHG_GW_EINVAL, "unknown initial-condition form");
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  double* fdev = nullptr;
  if (field) {
    const size_t n = (form == FREHG_GW_IC_WATER_TABLE)
                         ? static_cast<size_t>(d.nx) * d.ny
                         : static_cast<size_t>(d.nx) * d.ny * d.nz;
    CUDA_TRY(cudaMalloc(&fdev, n * sizeof(double)), "init_state");
    CUDA_TRY(cudaMemcpy(fdev, field, n * sizeof(double), cudaMemcpyHostToDevice), "init_state");
  }
  D.cur = 0;
  fgw::launch_init_state(D, form, constant, fdev, h->bath_dev, h->offset);
  fgw::launch_ghosts(D, D.h[0], D.wc[0]);
  CUDA_TRY(cudaMemcpyAsync(D.h[1], D.h[0], d.ncell * sizeof(double), cudaMemcpyDeviceToDevice,
                           D.stream), "init_state");
  CUDA_TRY(cudaMemcpyAsync(D.wc[1], D.wc[0], d.ncell * sizeof(double), cudaMemcpyDeviceToDevice,
                           D.stream), "init_state");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "init_state");
  if (fdev) cudaFree(fdev);
  CUDA_TRY(cudaGetLastError(), "init_state kernel");
  h->have_state = true;
  h->start_buf = 0;
  return FREHG_GW_OK;
}

int frehg_gw_set_state(frehg_gw_handle* h, const double* head, const double* wc) {
  if (!h || !head || !wc) return fail(FREHG_GW_EINVAL, "null argument");
  FGW_ON_DEVICE(h);
  h->have_prev = false;
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  std::vector<double> hh(static_cast<size_t>(d.ncell)), ww(static_cast<size_t>(d.ncell));
  CUDA_TRY(cudaMemcpy(hh.data(), D.h[D.cur], d.ncell * sizeof(double), cudaMemcpyDeviceToHost),
           "set_state");
  CUDA_TRY(cudaMemcpy(ww.data(), D.wc[D.cur], d.ncell * sizeof(double), cudaMemcpyDeviceToHost),
           "set_state");
  for (int j = 1; j <= d.ny; ++j)
    for (int i = 1; i <= d.nx; ++i)
      for (int k = 0; k < d.nz; ++k) {
        const long long q = (static_cast<long long>(j - 1) * d.nx + (i - 1)) * d.nz + k;
        hh[fgw::cidx(d, j, i, k)] = head[q];
        ww[fgw::cidx(d, j, i, k)] = wc[q];
      }
  if (D.f.baro) fgw::launch_baro(D);  // refreshDerivedState (RichardsSolver.cpp:880-890)
  for (int b = 0; b < 2; ++b) {
    CUDA_TRY(cudaMemcpy(D.h[b], hh.data(), d.ncell * sizeof(double), cudaMemcpyHostToDevice),
             "set_state");
    CUDA_TRY(cudaMemcpy(D.wc[b], ww.data(), d.ncell * sizeof(double), cudaMemcpyHostToDevice),
             "set_state");
    fgw::launch_ghosts(D, D.h[b], D.wc[b]);
  }
  CUDA_TRY(cudaStreamSynchronize(D.stream), "set_state");
  h->have_state = true;
  h->start_buf = D.cur;
  return FREHG_GW_OK;
}

int frehg_gw_restore(frehg_gw_handle* h, const double* head, const double* wc,
                     const double* vloss, double dtg) {
  if (!h || !head || !wc) return fail(FREHG_GW_EINVAL, "null argument");
  FGW_ON_DEVICE(h);
  h->have_prev = false;
  if (!(dtg > 0.0) || !std::isfinite(dtg)) return fail(FREHG_GW_EINVAL, "dtg must be positive");
  const int rc = frehg_gw_set_state(h, head, wc);
  if (rc != FREHG_GW_OK) return rc;
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  if (vloss) {
    std::vector<double> v(static_cast<size_t>(d.ncell), 0.0);
    for (int j = 1; j <= d.ny; ++j)
      for (int i = 1; i <= d.nx; ++i)
        for (int k = 0; k < d.nz; ++k)
          v[fgw::cidx(d, j, i, k)] =
              vloss[(static_cast<long long>(j - 1) * d.nx + (i - 1)) * d.nz + k];
    CUDA_TRY(cudaMemcpy(D.vloss, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice),
             "restore");
  }
  h->next_dt = dtg;
  return FREHG_GW_OK;
}

}  // extern "C"

namespace fgw_api {

cudaError_t enqueue_predictor(frehg_gw_handle* h, double dtg) {
  fgw::Device& D = h->D;
  double* hn = D.h[D.cur];
  double* wcn = D.wc[D.cur];
  // the density ratios first, so the hydrostatic edge ghosts see this step's
  // (RichardsSolver.cpp:739-746)
  if (D.f.baro) fgw::launch_baro(D);
  fgw::launch_ghosts(D, hn, wcn);
  if (D.f.cpl) fgw::launch_cpl_mode(D, hn);
  const bool mixed = h->precision == FREHG_GW_PRECISION_MIXED;
  const bool line64 = h->precision == FREHG_GW_PRECISION_FP64_LINE;
  if (!line64 && h->fused && fgw::launch_predict(D, hn, wcn, mixed)) return cudaGetLastError();
  fgw::launch_closure_pred(D, hn);
  // Both warm-started forms begin from h^n, or, when the previous step's
  // start state h^(n-1) is still in the other state buffer, from the linear
  // extrapolation of the two to this step's end.
  const bool extrap = (mixed || line64) && h->extrapolate && h->have_prev && dtg > 0.0 &&
                      h->prev_dtg > 0.0;
  fgw::launch_assemble(D, hn, wcn, mixed || line64, extrap ? D.h[1 - D.cur] : nullptr,
                       extrap ? dtg / h->prev_dtg : 0.0);
  if (mixed) return fgw::launch_line_factor(D);
  if (line64) return fgw::launch_line_factor64(D);
  return cudaGetLastError();
}

void enqueue_corrector(frehg_gw_handle* h) {
  fgw::Device& D = h->D;
  const int nxt = 1 - D.cur;
  double* hn = D.h[D.cur];
  double* wcn = D.wc[D.cur];
  if (!(h->fused && fgw::launch_correct(D, hn, wcn))) {
    fgw::launch_closure_corr(D, hn);
    fgw::launch_flux(D, wcn);
    if (D.f.cpl) fgw::launch_cpl_book(D, wcn);
    fgw::launch_update_wc(D, hn, wcn);
  }
  if (h->profiling) cudaEventRecord(h->ev[3], D.stream);
  fgw::launch_classify(D, D.wc[nxt], D.h[nxt]);
  fgw::launch_walk(D, D.wc[nxt]);
  if (D.win_x) fgw::launch_window_accum(D);
  if (h->profiling) cudaEventRecord(h->ev[4], D.stream);
  fgw::launch_finalize(D, D.wc[nxt], h->co_max);
  fgw::launch_step_info(D, h->dq_grow, h->dq_shrink, h->dt_min, h->dt_max);
}

cudaError_t upload_next_dt(frehg_gw_handle* h) {
  h->D.out_host->next_dt = h->next_dt;
  return cudaMemcpyAsync(&h->D.out->next_dt, &h->D.out_host->next_dt, sizeof(double),
                         cudaMemcpyHostToDevice, h->D.stream);
}

int finish_step(frehg_gw_handle* h, frehg_gw_step_info* info) {
  fgw::Device& D = h->D;
  const fgw::StepOut& o = *D.out_host;
  frehg_gw_step_info s{};
  s.cg_iterations = o.cg.its;
  s.outer_iterations = o.cg.outer;
  s.residual_norm = o.cg.dp;
  s.boundary_in = o.boundary_in;
  s.ss_storage = o.ss_storage;
  s.realloc_adjust = o.realloc_adjust;
  s.realloc_dropped = o.realloc_dropped;
  s.vloss = o.vloss;
  s.next_dt = o.next_dt;
  int status = FREHG_GW_OK;
  if (o.cg.err) {
    status = fail(FREHG_GW_ECUDA, "predictor solve: grid barrier timed out");
  } else if (o.cg.reason < 0) {
    status = fail(FREHG_GW_ESOLVER, "predictor solve diverged after " + std::to_string(o.cg.its) +
                                        " iterations (KSP reason " +
                                        std::to_string(o.cg.reason) + ")");
  } else if (!std::isfinite(o.volume)) {
    status = fail(FREHG_GW_ENONFINITE, "non-finite moisture after the step");
  }
  s.status = status;
  if (info) *info = s;
  if (status != FREHG_GW_OK) return status;
  h->start_buf = D.cur;
  D.cur = 1 - D.cur;
  h->next_dt = o.next_dt;
  if (D.f.cpl) {
    h->pc_clamp_total += o.cpl[5];
    h->cpl_last = frehg_gw_coupled_audit{o.cpl[0], o.cpl[1], o.cpl[2], o.cpl[3], o.cpl[4],
                                         h->pc_clamp_total};
  }
  return FREHG_GW_OK;
}

}  // namespace fgw_api

extern "C" {

int frehg_gw_step(frehg_gw_handle* h, double t, double dtg, frehg_gw_step_info* info) {
  (void)t;  // boundary values arrive through frehg_gw_set_bc_values
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  if (!h->have_state) return fail(FREHG_GW_ESTATE, "frehg_gw_step before frehg_gw_init_state");
  if (!(dtg > 0.0) || !std::isfinite(dtg)) return fail(FREHG_GW_EINVAL, "dtg must be positive");
  fgw::Device& D = h->D;
  const bool prof = h->profiling;
  auto mark = [&](int n) {
    if (prof) cudaEventRecord(h->ev[n], D.stream);
  };
  // The step's dtg goes into the device step record, where every kernel of
  // the step reads it.
  D.out_host->next_dt = dtg;
  CUDA_TRY(cudaMemcpyAsync(&D.out->next_dt, &D.out_host->next_dt, sizeof(double),
                           cudaMemcpyHostToDevice, D.stream), "step dtg");
  mark(0);
  cudaError_t e = fgw_api::enqueue_predictor(h, dtg);
  if (e != cudaSuccess) return cuda_fail(e, "predictor launch");
  mark(1);
  if (h->precision == FREHG_GW_PRECISION_MIXED) {
    e = fgw::launch_cg_mixed(D, h->rtol, h->atol, h->maxit, h->outer_rtol, h->max_outer);
  } else if (h->precision == FREHG_GW_PRECISION_FP64_LINE) {
    e = fgw::launch_cg_line64(D, h->atol, h->maxit, h->outer_rtol, h->max_outer);
  } else {
    e = fgw::launch_cg64(D, h->rtol, h->atol, h->maxit);
  }
  if (e != cudaSuccess) return cuda_fail(e, "predictor solve launch");
  mark(2);
  fgw_api::enqueue_corrector(h);
  mark(5);
  CUDA_TRY(cudaMemcpyAsync(D.out_host, D.out, sizeof(fgw::StepOut), cudaMemcpyDeviceToHost,
                           D.stream), "step readback");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "step");
  CUDA_TRY(cudaGetLastError(), "step kernels");
  if (prof) {
    for (int n = 0; n < 5; ++n) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, h->ev[n], h->ev[n + 1]);
      h->phase_ms[n] = ms;
    }
  }
  const int rc = fgw_api::finish_step(h, info);
  // The state buffer not holding the new h^n now holds this step's start
  // state: the next single step may extrapolate from the pair.
  h->have_prev = rc == FREHG_GW_OK;
  h->prev_dtg = dtg;
  return rc;
}

int frehg_gw_next_dt(frehg_gw_handle* h, double* out) {
  if (!h || !out) return fail(FREHG_GW_EINVAL, "null argument");
  *out = h->next_dt;
  return FREHG_GW_OK;
}

size_t frehg_gw_field_size(const frehg_gw_handle* h, int field) {
  if (!h) return 0;
  const fgw::Dims& d = h->D.d;
  const size_t nx = d.nx, ny = d.ny, nz = d.nz;
  switch (field) {
    case FREHG_GW_FIELD_QX: case FREHG_GW_FIELD_KX: case FREHG_GW_FIELD_AX:
    case FREHG_GW_FIELD_SINX: case FREHG_GW_FIELD_COSX:
      return ny * (nx + 1) * nz;
    case FREHG_GW_FIELD_QY: case FREHG_GW_FIELD_KY: case FREHG_GW_FIELD_AY:
    case FREHG_GW_FIELD_SINY: case FREHG_GW_FIELD_COSY:
      return (ny + 1) * nx * nz;
    case FREHG_GW_FIELD_QZ: case FREHG_GW_FIELD_KZ: case FREHG_GW_FIELD_WINDOW_Z:
      return ny * nx * (nz + 1);
    case FREHG_GW_FIELD_WINDOW_X: case FREHG_GW_FIELD_RHO_X: case FREHG_GW_FIELD_VISC_X:
      return ny * (nx + 1) * nz;
    case FREHG_GW_FIELD_WINDOW_Y: case FREHG_GW_FIELD_RHO_Y: case FREHG_GW_FIELD_VISC_Y:
      return (ny + 1) * nx * nz;
    case FREHG_GW_FIELD_RHO_Z: case FREHG_GW_FIELD_VISC_Z:
      return ny * nx * (nz + 1);
    case FREHG_GW_FIELD_WINDOW_VENT:
      return ny * nx;
    default:
      return (field >= 0 && field < FREHG_GW_FIELD_COUNT) ? ny * nx * nz : 0;
  }
}

int frehg_gw_get_field(frehg_gw_handle* h, int field, double* out) {
  if (!h || !out) return fail(FREHG_GW_EINVAL, "null argument");
  FGW_ON_DEVICE(h);
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  const double* src = nullptr;
  int kind = 0;  // 0 cell, 1 x face, 2 y face, 3 z face
  switch (field) {
    case FREHG_GW_FIELD_HEAD: src = D.h[D.cur]; break;
    case FREHG_GW_FIELD_WC: src = D.wc[D.cur]; break;
    case FREHG_GW_FIELD_WC_START: src = D.wc[h->start_buf]; break;
    case FREHG_GW_FIELD_DZ: src = D.dz; break;
    case FREHG_GW_FIELD_BOT: src = D.bot; break;
    case FREHG_GW_FIELD_VLOSS: src = D.vloss; break;
    case FREHG_GW_FIELD_QX: src = D.qx; kind = 1; break;
    case FREHG_GW_FIELD_KX: src = D.kx; kind = 1; break;
    case FREHG_GW_FIELD_AX: src = D.ax; kind = 1; break;
    case FREHG_GW_FIELD_SINX: src = D.sinx; kind = 1; break;
    case FREHG_GW_FIELD_COSX: src = D.cosx; kind = 1; break;
    case FREHG_GW_FIELD_QY: src = D.qy; kind = 2; break;
    case FREHG_GW_FIELD_KY: src = D.ky; kind = 2; break;
    case FREHG_GW_FIELD_AY: src = D.ay; kind = 2; break;
    case FREHG_GW_FIELD_SINY: src = D.siny; kind = 2; break;
    case FREHG_GW_FIELD_COSY: src = D.cosy; kind = 2; break;
    case FREHG_GW_FIELD_QZ: src = D.qzf; kind = 3; break;
    case FREHG_GW_FIELD_KZ: src = D.kzf; kind = 3; break;
    case FREHG_GW_FIELD_WINDOW_X: src = D.win_x; kind = 1; break;
    case FREHG_GW_FIELD_WINDOW_Y: src = D.win_y; kind = 2; break;
    case FREHG_GW_FIELD_WINDOW_Z: src = D.win_z; kind = 3; break;
    case FREHG_GW_FIELD_WINDOW_VENT: src = D.win_vent; kind = 4; break;
    case FREHG_GW_FIELD_RHO: src = D.rrho; break;
    case FREHG_GW_FIELD_VISC: src = D.rvisc; break;
    case FREHG_GW_FIELD_RHO_X: src = D.rxp; kind = 1; break;
    case FREHG_GW_FIELD_VISC_X: src = D.vxp; kind = 1; break;
    case FREHG_GW_FIELD_RHO_Y: src = D.ryp; kind = 2; break;
    case FREHG_GW_FIELD_VISC_Y: src = D.vyp; kind = 2; break;
    case FREHG_GW_FIELD_RHO_Z: src = D.rzp; kind = 3; break;
    case FREHG_GW_FIELD_VISC_Z: src = D.vzp; kind = 3; break;
    case FREHG_GW_FIELD_HEAD_PREV:
      if (!h->have_prev) return fail(FREHG_GW_ESTATE, "get_field: no previous step start");
      src = D.h[1 - D.cur];
      break;
    default: return fail(FREHG_GW_EINVAL, "unknown field");
  }
  if (!src && field >= FREHG_GW_FIELD_RHO) {  // no density coupling: every ratio is 1
    const size_t cnt = static_cast<size_t>(kind == 1 ? d.nx + 1 : d.nx) *
                       (kind == 2 ? d.ny + 1 : d.ny) * (kind == 3 ? d.nz + 1 : d.nz);
    std::fill(out, out + cnt, 1.0);
    return FREHG_GW_OK;
  }
  if (!src) return fail(FREHG_GW_ESTATE, "get_field: transport window not enabled");
  if (kind == 4) {  // a column field, (ny+2)(nx+2) on the device
    std::vector<double> full(static_cast<size_t>(d.ncol));
    CUDA_TRY(cudaStreamSynchronize(D.stream), "get_field");
    CUDA_TRY(cudaMemcpy(full.data(), src, full.size() * sizeof(double), cudaMemcpyDeviceToHost),
             "get_field");
    size_t q = 0;
    for (int j = 1; j <= d.ny; ++j)
      for (int i = 1; i <= d.nx; ++i) out[q++] = full[fgw::col2(d, j, i)];
    return FREHG_GW_OK;
  }
  const size_t n = static_cast<size_t>(kind == 3 ? d.ncol * (d.nz + 1) : d.ncell);
  std::vector<double> full(n);
  CUDA_TRY(cudaStreamSynchronize(D.stream), "get_field");
  CUDA_TRY(cudaMemcpy(full.data(), src, n * sizeof(double), cudaMemcpyDeviceToHost), "get_field");
  size_t q = 0;
  if (kind == 3) {
    for (int j = 1; j <= d.ny; ++j)
      for (int i = 1; i <= d.nx; ++i)
        for (int k = 0; k <= d.nz; ++k) out[q++] = full[fgw::fidx(d, j, i, k)];
    return FREHG_GW_OK;
  }
  const int j0 = (kind == 2) ? 0 : 1, i0 = (kind == 1) ? 0 : 1;
  for (int j = j0; j <= d.ny; ++j)
    for (int i = i0; i <= d.nx; ++i)
      for (int k = 0; k < d.nz; ++k) out[q++] = full[fgw::cidx(d, j, i, k)];
  return FREHG_GW_OK;
}

int frehg_gw_enable_transport_window(frehg_gw_handle* h) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  fgw::Device& D = h->D;
  if (D.win_x) return FREHG_GW_OK;
  const size_t n3 = static_cast<size_t>(D.d.ncell), nf = static_cast<size_t>(D.d.ncol) * (D.d.nz + 1);
  double** f[5] = {&D.win_x, &D.win_y, &D.win_z, &D.pcorr, &D.win_vent};
  const size_t n[5] = {n3, n3, nf, nf, static_cast<size_t>(D.d.ncol)};
  CUDA_TRY(cudaStreamSynchronize(D.stream), "enable_transport_window");
  for (int w = 0; w < 5; ++w) {
    void* p = nullptr;
    if (cudaMalloc(&p, n[w] * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      for (int u = 0; u < w; ++u) *f[u] = nullptr;  // freed with the handle
      return fail(FREHG_GW_ENOMEM, "enable_transport_window: allocation failed");
    }
    D.allocs.push_back(p);
    CUDA_TRY(cudaMemsetAsync(p, 0, n[w] * sizeof(double), D.stream), "enable_transport_window");
    *f[w] = static_cast<double*>(p);
  }
  CUDA_TRY(cudaStreamSynchronize(D.stream), "enable_transport_window");
  return FREHG_GW_OK;
}

int frehg_gw_reset_transport_window(frehg_gw_handle* h) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  fgw::Device& D = h->D;
  if (!D.win_x) return FREHG_GW_OK;  // as the reference: a no-op until enabled
  const size_t n3 = static_cast<size_t>(D.d.ncell), nf = static_cast<size_t>(D.d.ncol) * (D.d.nz + 1);
  CUDA_TRY(cudaMemsetAsync(D.win_x, 0, n3 * sizeof(double), D.stream), "reset_transport_window");
  CUDA_TRY(cudaMemsetAsync(D.win_y, 0, n3 * sizeof(double), D.stream), "reset_transport_window");
  CUDA_TRY(cudaMemsetAsync(D.win_z, 0, nf * sizeof(double), D.stream), "reset_transport_window");
  CUDA_TRY(cudaMemsetAsync(D.win_vent, 0, static_cast<size_t>(D.d.ncol) * sizeof(double),
                           D.stream), "reset_transport_window");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "reset_transport_window");
  return FREHG_GW_OK;
}

int frehg_gw_owned_volume(frehg_gw_handle* h, double* out) {
  if (!h || !out) return fail(FREHG_GW_EINVAL, "null argument");
  FGW_ON_DEVICE(h);
  fgw::Device& D = h->D;
  fgw::launch_volume(D, D.wc[D.cur]);
  CUDA_TRY(cudaMemcpyAsync(D.out_host, D.out, sizeof(fgw::StepOut), cudaMemcpyDeviceToHost,
                           D.stream), "owned_volume");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "owned_volume");
  *out = D.out_host->volume;
  return FREHG_GW_OK;
}

long long frehg_gw_active_cells(const frehg_gw_handle* h) { return h ? h->nactive : 0; }

int frehg_gw_device(const frehg_gw_handle* h) { return h ? h->device : -1; }

int frehg_gw_set_profiling(frehg_gw_handle* h, int on) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  if (on && !h->ev[0]) {
    for (cudaEvent_t& e : h->ev) CUDA_TRY(cudaEventCreate(&e), "set_profiling");
  }
  h->profiling = on != 0;
  return FREHG_GW_OK;
}

int frehg_gw_set_fused(frehg_gw_handle* h, int on) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  // The fused passes raised a misaligned-address error on the B200 whose
  // cause is not found; they are not switched on until it is.
  if (on) return fail(FREHG_GW_EUNSUPPORTED, "set_fused: the fused passes are disabled");
  h->fused = false;
  return FREHG_GW_OK;
}

int frehg_gw_prev_dt(frehg_gw_handle* h, double* out) {
  if (!h || !out) return fail(FREHG_GW_EINVAL, "null argument");
  *out = h->have_prev ? h->prev_dtg : 0.0;
  return FREHG_GW_OK;
}

int frehg_gw_restore_prev(frehg_gw_handle* h, const double* head_prev, double prev_dt) {
  if (!h || !head_prev) return fail(FREHG_GW_EINVAL, "null argument");
  FGW_ON_DEVICE(h);
  if (!(prev_dt > 0.0) || !std::isfinite(prev_dt))
    return fail(FREHG_GW_EINVAL, "restore_prev: prev_dt must be positive");
  if (!h->have_state) return fail(FREHG_GW_ESTATE, "restore_prev before a state");
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  // Only the interior heads are read (the extrapolated start of active cells).
  std::vector<double> full(static_cast<size_t>(d.ncell), 0.0);
  CUDA_TRY(cudaStreamSynchronize(D.stream), "restore_prev");
  size_t q = 0;
  for (int j = 1; j <= d.ny; ++j)
    for (int i = 1; i <= d.nx; ++i)
      for (int k = 0; k < d.nz; ++k) full[fgw::cidx(d, j, i, k)] = head_prev[q++];
  CUDA_TRY(cudaMemcpy(D.h[1 - D.cur], full.data(), full.size() * sizeof(double),
                      cudaMemcpyHostToDevice), "restore_prev");
  h->have_prev = true;
  h->prev_dtg = prev_dt;
  return FREHG_GW_OK;
}

int frehg_gw_set_warm_start(frehg_gw_handle* h, int mode) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  if (mode != 0 && mode != 1) return fail(FREHG_GW_EINVAL, "set_warm_start: mode 0 or 1");
  h->extrapolate = mode == 1;
  return FREHG_GW_OK;
}

int frehg_gw_phase_times(frehg_gw_handle* h, double* ms5) {
  if (!h || !ms5) return fail(FREHG_GW_EINVAL, "null argument");
  for (int n = 0; n < 5; ++n) ms5[n] = h->phase_ms[n];
  return FREHG_GW_OK;
}

long long frehg_gw_kernel_launches(const frehg_gw_handle* h) { return h ? h->D.launches : 0; }

}  // extern "C"

// ---------------------------------------------------------------- init_state without allocation
// frehg_gw_init_state stages a caller's IC field in a device buffer that it
// allocates and frees on every call.  frehg_gw_init_state_static stages it in
// one fixed array compiled into this library instead, so the call allocates
// nothing.  It is meant for callers that cannot allocate at that point: a
// driver that has handed all free HBM to its own memory pool (cudaMalloc
// would fail), or one that re-initialises domains while other streams are
// busy (cudaFree waits for the whole device).
//
// The array holds FREHG_GW_STATIC_FIELD_MAX doubles (2 MiB); larger fields
// are rejected with FREHG_GW_EINVAL.  Nothing in it has to start at zero:
// each call writes the values it then reads.  Every call on a device uses
// the same array, so two calls that overlap in time (two host threads, or two
// handles driven concurrently) race on it and must be serialised by the
// caller.  The first call on each device does a one-time set-up (it looks up
// the array's device address, which may load this library's device code on
// that device); make that first call before any stream capture begins.
static __device__ __align__(256) double g_static_field[FREHG_GW_STATIC_FIELD_MAX];

namespace {

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_ptr[kStaticMaxDevices] = {};

// The array's device address on the current device, looked up once per
// device with that device current.
int static_field_address(double** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev), "init_state_static: cudaGetDevice");
  if (dev < 0 || dev >= kStaticMaxDevices)
    return fail(FREHG_GW_EUNSUPPORTED, "init_state_static: device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    CUDA_TRY(cudaGetSymbolAddress(&p, g_static_field), "init_state_static: scratch address");
    g_static_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_static_ptr[dev];
  return FREHG_GW_OK;
}

}  // namespace

int frehg_gw_init_state_static(frehg_gw_handle* h, int form, double constant,
                               const double* field) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  FGW_ON_DEVICE(h);
  h->have_prev = false;
  if (form < FREHG_GW_IC_MOISTURE || form > FREHG_GW_IC_WATER_TABLE)
    return fail(FREHG_GW_EINVAL, "unknown initial-condition form");
  double* scratch = nullptr;
  const int rc = static_field_address(&scratch);
  if (rc != FREHG_GW_OK) return rc;
  fgw::Device& D = h->D;
  const fgw::Dims& d = D.d;
  const double* fdev = nullptr;
  if (field) {
    const size_t n = (form == FREHG_GW_IC_WATER_TABLE)
                         ? static_cast<size_t>(d.nx) * d.ny
                         : static_cast<size_t>(d.nx) * d.ny * d.nz;
    if (n > static_cast<size_t>(FREHG_GW_STATIC_FIELD_MAX))
      return fail(FREHG_GW_EINVAL,
                  "init_state_static: field has " + std::to_string(n) +
                      " values; the static scratch holds at most " +
                      std::to_string(FREHG_GW_STATIC_FIELD_MAX) +
                      " (use frehg_gw_init_state)");
    CUDA_TRY(cudaMemcpyAsync(scratch, field, n * sizeof(double), cudaMemcpyHostToDevice,
                             D.stream), "init_state_static");
    fdev = scratch;
  }
  D.cur = 0;
  fgw::launch_init_state(D, form, constant, fdev, h->bath_dev, h->offset);
  fgw::launch_ghosts(D, D.h[0], D.wc[0]);
  CUDA_TRY(cudaMemcpyAsync(D.h[1], D.h[0], d.ncell * sizeof(double), cudaMemcpyDeviceToDevice,
                           D.stream), "init_state_static");
  CUDA_TRY(cudaMemcpyAsync(D.wc[1], D.wc[0], d.ncell * sizeof(double), cudaMemcpyDeviceToDevice,
                           D.stream), "init_state_static");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "init_state_static");
  CUDA_TRY(cudaGetLastError(), "init_state_static kernel");
  h->have_state = true;
  h->start_buf = 0;
  return FREHG_GW_OK;
}
