// Density coupling of the groundwater step (include/frehg_gw.h, "density
// coupling"): the scalars a transport module hands over, and the cell and
// face density / viscosity ratios the step computes from them at its start
// (RichardsSolver::updateBaroclinicFaces, src/gw/Baroclinic.cpp:46-186).  The
// ratios enter the ghost, assembly, flux, theta-update and classification
// kernels of gw_kernels.cu through Fields::baro.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "gw_handle.h"

using fgw_api::cuda_fail;
using fgw_api::fail;

#define CUDA_TRY(call, what)                           \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

namespace fgw {

namespace {

struct BaroCoef {
  double bs, bsv, bt, t0;  // beta_saline, beta_saline_visc, beta_T, T0
  int saline, thermal, coupled;
};

// r_rho = 1 + beta_s s - beta_T (T - T0) and r_visc = 1 / (1 + beta_sv s)
// over every cell of the halo box (update_rhovisc's extended range).
__global__ void k_baro_cells(Dims d, BaroCoef k, const double* __restrict__ s,
                             const double* __restrict__ t, double* __restrict__ rrho,
                             double* __restrict__ rvisc) {
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double sv = k.saline ? s[c] : 0.0;
    const double dtv = k.thermal ? t[c] - k.t0 : 0.0;
    rrho[c] = 1.0 + k.bs * sv - k.bt * dtv;
    rvisc[c] = 1.0 / (1.0 + k.bsv * sv);
  }
}

__device__ inline bool head_code(int code) { return code == kHead || code == kHydro; }

// The face means, one thread per (j, i, plane) slot of the z-face layout:
// plane k < nz also owns the x face slot (j, i, k) and the y face slot
// (j, i, k).  Interior faces average two active flanks (1 otherwise); the
// minus-side domain-edge faces average the edge cell with its ghost, or take
// the ghost's ratio under a head edge; the plus-side edge faces take the
// ghost's ratio under a head edge and stay 1 otherwise; the face above a
// column's top cell averages it with the surface scalar's ratio (coupled) or
// its own; the bottom boundary face stays 1.
__global__ void k_baro_faces(Dims d, Fields f, BaroCoef k, const double* __restrict__ s,
                             const double* __restrict__ s2, const double* __restrict__ t,
                             const double* __restrict__ t2, const double* __restrict__ rrho,
                             const double* __restrict__ rvisc, double* __restrict__ rxp,
                             double* __restrict__ vxp, double* __restrict__ ryp,
                             double* __restrict__ vyp, double* __restrict__ rzp,
                             double* __restrict__ vzp) {
  const int nzp = d.nz + 1;
  const long long n = d.ncol * nzp;
  for (long long u = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; u < n;
       u += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long col = u / nzp;
    const int kk = static_cast<int>(u - col * nzp);
    const int j = static_cast<int>(col / d.nx2);
    const int i = static_cast<int>(col - static_cast<long long>(j) * d.nx2);
    if (kk < d.nz) {
      const long long c = cidx(d, j, i, kk);
      if (j >= 1 && j <= d.ny && i <= d.nx) {  // x face slot (j, i): face i + 1/2
        double rr = 1.0, rv = 1.0;
        if (i == 0) {
          const long long a = c + d.sx;
          if (f.act[a]) {
            if (head_code(f.xmc[col2(d, j, 1)])) {
              rr = rrho[c];
              rv = rvisc[c];
            } else {
              rr = 0.5 * (rrho[a] + rrho[c]);
              rv = 0.5 * (rvisc[a] + rvisc[c]);
            }
          }
        } else if (i == d.nx) {
          if (f.act[c] && head_code(f.xpc[col])) {
            rr = rrho[c + d.sx];
            rv = rvisc[c + d.sx];
          }
        } else if (f.act[c] && f.act[c + d.sx]) {
          rr = 0.5 * (rrho[c] + rrho[c + d.sx]);
          rv = 0.5 * (rvisc[c] + rvisc[c + d.sx]);
        }
        rxp[c] = rr;
        vxp[c] = rv;
      }
      if (i >= 1 && i <= d.nx && j <= d.ny) {  // y face slot (j, i): face j + 1/2
        double rr = 1.0, rv = 1.0;
        if (j == 0) {
          const long long a = c + d.sy;
          if (f.act[a]) {
            if (head_code(f.ymc[col2(d, 1, i)])) {
              rr = rrho[c];
              rv = rvisc[c];
            } else {
              rr = 0.5 * (rrho[a] + rrho[c]);
              rv = 0.5 * (rvisc[a] + rvisc[c]);
            }
          }
        } else if (j == d.ny) {
          if (f.act[c] && head_code(f.ypc[col])) {
            rr = rrho[c + d.sy];
            rv = rvisc[c + d.sy];
          }
        } else if (f.act[c] && f.act[c + d.sy]) {
          rr = 0.5 * (rrho[c] + rrho[c + d.sy]);
          rv = 0.5 * (rvisc[c] + rvisc[c + d.sy]);
        }
        ryp[c] = rr;
        vyp[c] = rv;
      }
    }
    if (j >= 1 && j <= d.ny && i >= 1 && i <= d.nx) {  // z plane kk above cell kk
      const long long cb = cidx(d, j, i, kk < d.nz ? kk : d.nz - 1);
      const bool below = kk < d.nz && f.act[cb];
      const bool above = kk >= 1 && f.act[cidx(d, j, i, kk - 1)];
      double rr = 1.0, rv = 1.0;
      if (below && above) {
        const long long a = cb - 1;
        rr = 0.5 * (rrho[a] + rrho[cb]);
        rv = 0.5 * (rvisc[a] + rvisc[cb]);
      } else if (below) {
        const double sg = k.saline ? (k.coupled ? s2[col] : s[cb]) : 0.0;
        const double tg = k.thermal ? (k.coupled ? t2[col] : t[cb]) - k.t0 : 0.0;
        rr = 0.5 * (rrho[cb] + 1.0 + k.bs * sg - k.bt * tg);
        rv = 0.5 * (rvisc[cb] + 1.0 / (1.0 + k.bsv * sg));
      }
      rzp[fidx(d, j, i, kk)] = rr;
      vzp[fidx(d, j, i, kk)] = rv;
    }
  }
}

__global__ void k_fill(double* __restrict__ p, long long n, double v) {
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
       c += static_cast<long long>(gridDim.x) * blockDim.x)
    p[c] = v;
}

}  // namespace

void launch_baro(const Device& D) {
  const BaroCoef k{D.beta_s, D.beta_sv, D.beta_t, D.t_ref, D.saline, D.thermal,
                   D.f.cpl != nullptr};
  const double* s = D.scal[FREHG_GW_SCALAR_SALINE];
  const double* s2 = D.scal[FREHG_GW_SCALAR_SALINE_SURF];
  const double* t = D.scal[FREHG_GW_SCALAR_TEMP];
  const double* t2 = D.scal[FREHG_GW_SCALAR_TEMP_SURF];
  const unsigned g = static_cast<unsigned>(D.nblk);
  k_baro_cells<<<g, kBlock, 0, D.stream>>>(D.d, k, s, t, D.rrho, D.rvisc);
  k_baro_faces<<<g, kBlock, 0, D.stream>>>(D.d, D.f, k, s, s2, t, t2, D.rrho, D.rvisc, D.rxp,
                                           D.vxp, D.ryp, D.vyp, D.rzp, D.vzp);
  D.launches += 2;
}

}  // namespace fgw

namespace {

int need_density(const frehg_gw_handle* h) {
  if (!h) return fail(FREHG_GW_EINVAL, "null handle");
  if (!h->D.f.baro) return fail(FREHG_GW_ESTATE, "no density coupling (frehg_gw_attach_density)");
  return FREHG_GW_OK;
}

bool cell_scalar(int which) {
  return which == FREHG_GW_SCALAR_SALINE || which == FREHG_GW_SCALAR_TEMP;
}

cudaError_t alloc_zero(fgw::Device& D, double** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(double));
  if (e != cudaSuccess) return e;
  D.allocs.push_back(q);
  *p = static_cast<double*>(q);
  return cudaMemsetAsync(q, 0, n * sizeof(double), D.stream);
}

}  // namespace

extern "C" {

int frehg_gw_attach_density(frehg_gw_handle* h, int saline, int thermal,
                            const frehg_gw_density* c) {
  if (!h || !c) return fail(FREHG_GW_EINVAL, "attach_density: null argument");
  FGW_ON_DEVICE(h);
  if (!saline && !thermal) return fail(FREHG_GW_EINVAL, "attach_density: no scalar");
  const double co[4] = {c->beta_saline, c->beta_saline_visc, c->thermal_expansion,
                        c->reference_temperature};
  for (double v : co)
    if (!std::isfinite(v)) return fail(FREHG_GW_EINVAL, "attach_density: non-finite coefficient");
  fgw::Device& D = h->D;
  if (D.f.baro) return fail(FREHG_GW_ESTATE, "attach_density: already attached");
  const size_t n3 = static_cast<size_t>(D.d.ncell), n2 = static_cast<size_t>(D.d.ncol);
  const size_t nf = n2 * static_cast<size_t>(D.d.nz + 1);
  CUDA_TRY(cudaStreamSynchronize(D.stream), "attach_density");
  const bool want[4] = {saline != 0, saline != 0, thermal != 0, thermal != 0};
  for (int w = 0; w < 4; ++w) {
    if (!want[w]) continue;
    if (alloc_zero(D, &D.scal[w], cell_scalar(w) ? n3 : n2) != cudaSuccess) {
      cudaGetLastError();
      return fail(FREHG_GW_ENOMEM, "attach_density: scalar allocation failed");
    }
  }
  double** r3[] = {&D.rrho, &D.rvisc, &D.rxp, &D.ryp, &D.vxp, &D.vyp};
  double** rf[] = {&D.rzp, &D.vzp};
  for (double** p : r3)
    if (alloc_zero(D, p, n3) != cudaSuccess) {
      cudaGetLastError();
      return fail(FREHG_GW_ENOMEM, "attach_density: ratio allocation failed");
    }
  for (double** p : rf)
    if (alloc_zero(D, p, nf) != cudaSuccess) {
      cudaGetLastError();
      return fail(FREHG_GW_ENOMEM, "attach_density: ratio allocation failed");
    }
  const unsigned g = static_cast<unsigned>(D.nblk);
  for (double** p : r3) fgw::k_fill<<<g, fgw::kBlock, 0, D.stream>>>(*p, static_cast<long long>(n3), 1.0);
  for (double** p : rf) fgw::k_fill<<<g, fgw::kBlock, 0, D.stream>>>(*p, static_cast<long long>(nf), 1.0);
  D.launches += 8;
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(fgw::BaroDev)) != cudaSuccess) {
    cudaGetLastError();
    return fail(FREHG_GW_ENOMEM, "attach_density: allocation failed");
  }
  D.allocs.push_back(p);
  D.baro_dev = static_cast<fgw::BaroDev*>(p);
  D.saline = saline != 0;
  D.thermal = thermal != 0;
  D.beta_s = c->beta_saline;
  D.beta_sv = c->beta_saline_visc;
  D.beta_t = c->thermal_expansion;
  D.t_ref = c->reference_temperature;
  fgw::BaroDev& b = D.baro_host;
  b.rrho = D.rrho;
  b.rxp = D.rxp;
  b.ryp = D.ryp;
  b.rzp = D.rzp;
  b.vxp = D.vxp;
  b.vyp = D.vyp;
  b.vzp = D.vzp;
  b.dgrad = c->reallocation_gradient != 0;
  CUDA_TRY(cudaMemcpyAsync(D.baro_dev, &b, sizeof(b), cudaMemcpyHostToDevice, D.stream),
           "attach_density");
  CUDA_TRY(cudaStreamSynchronize(D.stream), "attach_density");
  CUDA_TRY(cudaGetLastError(), "attach_density kernel");
  D.f.baro = D.baro_dev;
  return FREHG_GW_OK;
}

int frehg_gw_set_scalar(frehg_gw_handle* h, int which, const double* values) {
  if (int rc = need_density(h)) return rc;
  FGW_ON_DEVICE(h);
  if (which < 0 || which > 3 || !h->D.scal[which])
    return fail(FREHG_GW_EINVAL, "set_scalar: scalar not attached");
  if (!values) return fail(FREHG_GW_EINVAL, "set_scalar: null values");
  fgw::Device& D = h->D;
  const size_t n = static_cast<size_t>(cell_scalar(which) ? D.d.ncell : D.d.ncol);
  CUDA_TRY(cudaStreamSynchronize(D.stream), "set_scalar");
  CUDA_TRY(cudaMemcpy(D.scal[which], values, n * sizeof(double), cudaMemcpyHostToDevice),
           "set_scalar");
  return FREHG_GW_OK;
}

int frehg_gw_get_scalar(frehg_gw_handle* h, int which, double* out) {
  if (int rc = need_density(h)) return rc;
  FGW_ON_DEVICE(h);
  if (which < 0 || which > 3 || !h->D.scal[which])
    return fail(FREHG_GW_EINVAL, "get_scalar: scalar not attached");
  if (!out) return fail(FREHG_GW_EINVAL, "get_scalar: null output");
  fgw::Device& D = h->D;
  const size_t n = static_cast<size_t>(cell_scalar(which) ? D.d.ncell : D.d.ncol);
  CUDA_TRY(cudaStreamSynchronize(D.stream), "get_scalar");
  CUDA_TRY(cudaMemcpy(out, D.scal[which], n * sizeof(double), cudaMemcpyDeviceToHost),
           "get_scalar");
  return FREHG_GW_OK;
}

double* frehg_gw_scalar_ptr(frehg_gw_handle* h, int which) {
  if (!h || which < 0 || which > 3) return nullptr;
  return h->D.scal[which];
}

}  // extern "C"
