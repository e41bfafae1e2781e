// Cell and face kernels of the B200 groundwater step (everything except the
// predictor's linear solve, which lives in gw_cg.cu).
//
// One step is: ghosts -> predictor closure -> assembly -> CG -> corrector
// closure (+ head scatter and ghosts) -> faces and fluxes -> theta update ->
// post-allocation classification -> column send walks -> clamp, audit and
// controller terms -> one-block reduction into the step record.  Each kernel
// follows one phase of the reference step (src/gw/RichardsSolver.cpp:729-794);
// the per-kernel comments cite the reference code they restate.
//
// All reductions are two-level and fixed-shape: every reducing kernel runs on
// the same grid of D.nblk blocks, writes one partial per block, and
// k_step_info combines the partials in block order, so a step's audit is
// bit-reproducible run to run.
#include <cfloat>

#include "gw_internal.h"

namespace fgw {

namespace {

__device__ inline double ghost_head(int code, double value, double interior, double zc) {
  // enforceHeadBc / ghostHead, uncoupled (src/gw/Predictor.cpp:66-87).
  if (code == kHead) return value;
  if (code == kHydro) return value - zc;
  return interior;
}

struct SumOp {
  __device__ double operator()(double a, double b) const { return a + b; }
};
struct MaxOp {
  __device__ double operator()(double a, double b) const { return b > a ? b : a; }
};
struct MinOp {
  __device__ double operator()(double a, double b) const { return b < a ? b : a; }
};

// Block-wide reduction in a fixed order; the result is valid in thread 0.
template <class Op>
__device__ double block_reduce(double v, Op op, double identity) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (lane < nw) ? sh[lane] : identity;
  if (wid == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  __syncthreads();
  return v;
}

inline dim3 cells_grid(const Device& D) { return dim3(static_cast<unsigned>(D.nblk)); }

// ---------------------------------------------------------------- ghosts
// Domain-edge ghost heads and moisture (enforceHeadBc, Predictor.cpp:757-817;
// enforceMoistureBc, Corrector.cpp:709-756).  Either pointer may be null.
__global__ void k_ghosts(Dims d, Fields f, double* h, double* wc) {
  const long long nxg = 2LL * d.ny * d.nz, nyg = 2LL * d.nx * d.nz;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < nxg + nyg;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    long long g, c;
    int code;
    double val;
    if (t < nxg) {
      const int side = static_cast<int>(t / (static_cast<long long>(d.ny) * d.nz));
      const long long rem = t - static_cast<long long>(side) * d.ny * d.nz;
      const int j = static_cast<int>(rem / d.nz) + 1, k = static_cast<int>(rem % d.nz);
      const int ii = side == 0 ? 1 : d.nx;
      c = cidx(d, j, ii, k);
      g = side == 0 ? c - d.sx : c + d.sx;
      const long long cc = col2(d, j, ii);
      code = side == 0 ? f.xmc[cc] : f.xpc[cc];
      val = side == 0 ? f.xmv[cc] : f.xpv[cc];
    } else {
      const long long u = t - nxg;
      const int side = static_cast<int>(u / (static_cast<long long>(d.nx) * d.nz));
      const long long rem = u - static_cast<long long>(side) * d.nx * d.nz;
      const int i = static_cast<int>(rem / d.nz) + 1, k = static_cast<int>(rem % d.nz);
      const int jj = side == 0 ? 1 : d.ny;
      c = cidx(d, jj, i, k);
      g = side == 0 ? c - d.sy : c + d.sy;
      const long long cc = col2(d, jj, i);
      code = side == 0 ? f.ymc[cc] : f.ypc[cc];
      val = side == 0 ? f.ymv[cc] : f.ypv[cc];
    }
    if (h) h[g] = ghost_head(code, val, h[c], f.bot[c] + 0.5 * f.dz[c]);
    if (wc) wc[g] = is_head(code) ? f.wcs[c] : wc[c];
  }
}

// ---------------------------------------------------------------- closures
// Per-cell directional conductivities K(h, Ksx|Ksy|Ksz) of the predictor pass
// from the step-start head (ghosts included; Predictor.cpp:127-232 evaluates
// them for both flanks of every face).
// The same pass also evaluates C(h^n), the capacity of the storage term
// (Predictor.cpp:445-452), from the same powers.
__global__ void k_closure_pred(Dims d, Fields f, const double* __restrict__ h, double* kcx,
                               double* kcy, double* kcz, double* ch) {
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    const Soil so = soil_at(f, c);
    const double hc = h[c];
    const VgParts v = vg_parts(so, hc);
    const KrParts p = vg_kr_from(v, hc);
    kcx[c] = vg_k_from(p, f.ksx[c]);
    kcy[c] = vg_k_from(p, f.ksy[c]);
    kcz[c] = vg_k_from(p, f.ksz[c]);
    ch[c] = vg_capacity_from(so, v, hc);
  }
}

// Corrector pass: scatter the solved heads (fillAndSolve's gw_scatter_head,
// Predictor.cpp:745-754), re-impose the ghost heads (enforceHeadBc after the
// solve, RichardsSolver.cpp:762) and evaluate the per-cell conductivities of
// the predicted head (the corrector's computeFaceConductivity, :768).
__global__ void k_closure_corr(Dims d, Fields f, const double* __restrict__ x,
                               const double* __restrict__ hn, double* hp, double* kcx,
                               double* kcy, double* kcz) {
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const bool jin = j >= 1 && j <= d.ny, iin = i >= 1 && i <= d.nx;
    double hv = 0.0;
    if (jin && iin) {
      hv = f.act[c] ? x[c] : hn[c];
    } else if (jin && (i == 0 || i == d.nx + 1)) {
      const long long ci = (i == 0) ? c + d.sx : c - d.sx;
      const long long cc = col2(d, j, i == 0 ? 1 : d.nx);
      const double hi = f.act[ci] ? x[ci] : hn[ci];
      hv = ghost_head(i == 0 ? f.xmc[cc] : f.xpc[cc], i == 0 ? f.xmv[cc] : f.xpv[cc], hi,
                      f.bot[ci] + 0.5 * f.dz[ci]);
    } else if (iin && (j == 0 || j == d.ny + 1)) {
      const long long ci = (j == 0) ? c + d.sy : c - d.sy;
      const long long cc = col2(d, j == 0 ? 1 : d.ny, i);
      const double hi = f.act[ci] ? x[ci] : hn[ci];
      hv = ghost_head(j == 0 ? f.ymc[cc] : f.ypc[cc], j == 0 ? f.ymv[cc] : f.ypv[cc], hi,
                      f.bot[ci] + 0.5 * f.dz[ci]);
    }
    hp[c] = hv;
    const KrParts p = vg_kr_parts(soil_at(f, c), hv);
    kcx[c] = vg_k_from(p, f.ksx[c]);
    kcy[c] = vg_k_from(p, f.ksy[c]);
    kcz[c] = vg_k_from(p, f.ksz[c]);
  }
}

// ---------------------------------------------------------------- assembly
// The 7-point head system of one active cell (assembleSystemImpl,
// Predictor.cpp:400-698, uncoupled, density ratios 1): storage
// C(h^n) + Ss theta^n / theta_s, the six legs with the head-edge doubling,
// the flux-edge and Dirichlet-top diagonal rules, and the RHS with gravity,
// terrain and boundary terms.  The solver stores the diagonal and the three
// upper legs of each row; the lower legs are the neighbours' upper legs
// (the same expression on the same data, so the stored matrix is the
// reference's up to the rounding of its z legs).  Legs toward an inactive
// cell or out of the domain are stored as 0 (PETSc ignores column -1).
__global__ void __launch_bounds__(kBlock, 3)
    k_assemble(Dims d, Fields f, PassK pk, const double* __restrict__ hn,
               const double* __restrict__ wcn, const double* __restrict__ ch, double dtg,
               double* diag, double* gxps, double* gyps, double* gzps, double* rhs) {
  const double dx = d.dx, dy = d.dy;
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    if (j < 1 || j > d.ny || i < 1 || i > d.nx) continue;
    if (!f.act[c]) {
      diag[c] = 1.0;
      gxps[c] = 0.0;
      gyps[c] = 0.0;
      gzps[c] = 0.0;
      rhs[c] = 0.0;
      continue;
    }
    const long long cw = c - d.sx, ce = c + d.sx, cs = c - d.sy, cn = c + d.sy;
    const long long col = col2(d, j, i);
    const bool east = i == d.nx, west = i == 1, north = j == d.ny, south = j == 1;
    const bool top = (k == 0) || !f.act[c - 1];
    const double dzc = f.dz[c];
    const double volume = d.az * dzc;
    const double kxp = face_kx(d, f, pk, j, i, k), kxm = face_kx(d, f, pk, j, i - 1, k);
    const double kyp = face_ky(d, f, pk, j, i, k), kym = face_ky(d, f, pk, j - 1, i, k);
    const double kzm = face_kz(d, f, pk, j, i, k), kzp = face_kz(d, f, pk, j, i, k + 1);
    double gxp = -kxp * dtg * f.cosx[c] / (dx * dx) * (f.ax[c] * dx);
    double gxm = -kxm * dtg * f.cosx[cw] / (dx * dx) * (f.ax[cw] * dx);
    double gyp = -kyp * dtg * f.cosy[c] / (dy * dy) * (f.ay[c] * dy);
    double gym = -kym * dtg * f.cosy[cs] / (dy * dy) * (f.ay[cs] * dy);
    const int cxp = f.xpc[col], cxm = f.xmc[col], cyp = f.ypc[col], cym = f.ymc[col];
    if (east && is_head(cxp)) gxp *= 2.0;
    if (west && is_head(cxm)) gxm *= 2.0;
    if (north && is_head(cyp)) gyp *= 2.0;
    if (south && is_head(cym)) gym *= 2.0;
    double dzf = (k == d.nz - 1) ? 0.5 * dzc : 0.5 * (dzc + f.dz[c + 1]);
    const double gzp = -kzp * dtg / (dzc * dzf) * volume;
    dzf = top ? 0.5 * dzc : 0.5 * (dzc + f.dz[c - 1]);
    const double gzm = -kzm * dtg / (dzc * dzf) * volume;

    const double storage = ch[c] + d.ss * wcn[c] / f.wcs[c];
    double gct = storage * volume - (gxp + gxm + gyp + gym);
    if (east && cxp == kFlux) gct += gxp;
    if (west && cxm == kFlux) gct += gxm;
    if (north && cyp == kFlux) gct += gyp;
    if (south && cym == kFlux) gct += gym;
    const int botc = f.botc[col], topc = f.topc[col];
    if (!(k == d.nz - 1 && botc != kHead)) gct -= gzp;
    if (!top || topc == kHead) gct -= gzm;

    double b = storage * hn[c] * volume;
    b -= dtg * volume * kzp / dzc;
    b += dtg * volume * kzm / dzc;
    if (d.terrain) {
      double sg = (f.bot[ce] > f.bot[c]) ? 1.0 : -1.0;
      b += sg * dtg * f.ax[c] * kxp * f.sinx[c];
      sg = (f.bot[c] > f.bot[cw]) ? -1.0 : 1.0;
      b += sg * dtg * f.ax[cw] * kxm * f.sinx[cw];
      sg = (f.bot[cn] > f.bot[c]) ? 1.0 : -1.0;
      b += sg * dtg * f.ay[c] * kyp * f.siny[c];
      sg = (f.bot[c] > f.bot[cs]) ? -1.0 : 1.0;
      b += sg * dtg * f.ay[cs] * kym * f.siny[cs];
    }
    if (east) {
      if (cxp == kFlux) b += f.ax[c] * f.xpv[col] * dtg;
      else b -= gxp * hn[ce];
    }
    if (west) {
      if (cxm == kFlux) b += f.ax[cw] * f.xmv[col] * dtg;
      else b -= gxm * hn[cw];
    }
    if (north) {
      if (cyp == kFlux) b += f.ay[c] * f.ypv[col] * dtg;
      else b -= gyp * hn[cn];
    }
    if (south) {
      if (cym == kFlux) b += f.ay[cs] * f.ymv[col] * dtg;
      else b -= gym * hn[cs];
    }
    if (k == d.nz - 1) {
      if (botc == kFlux) b += dtg * volume * (f.botv[col] + kzp) / dzc;
      else if (botc == kHead) b -= gzp * f.botv[col];
    }
    if (top) {
      if (topc == kHead) b -= gzm * f.topv[col];
      else if (topc == kFlux) b += -dtg * volume * (f.topv[col] + kzm) / dzc;
    }
    diag[c] = gct;
    gxps[c] = (!east && f.act[ce]) ? gxp : 0.0;
    gyps[c] = (!north && f.act[cn]) ? gyp : 0.0;
    gzps[c] = (k + 1 < d.nz && f.act[c + 1]) ? gzp : 0.0;
    rhs[c] = b;
  }
}

// ---------------------------------------------------------------- fluxes
// Corrector faces and Darcy fluxes (computeFaceConductivity from the predicted
// head, Predictor.cpp:105-386, and computeFluxesImpl<PC, HARM>,
// Corrector.cpp:135-527, uncoupled).  Thread c owns the x+ and y+ faces of
// its cell and the z face above it (plus the bottom face for k = nz-1).
__device__ inline double flux_x(const Dims& d, const Fields& f, const PassK& pk,
                                const double* hp, const double* wcn, int j, int i, int k) {
  const long long c = cidx(d, j, i, k);
  const double faceA = f.ax[c];
  double q;
  if (i == 0) {
    const long long ci = c + d.sx;
    q = faceA * pk.kcx[ci] * f.cosx[c] * (hp[ci] - hp[c]) / (0.5 * d.dx);
    const int code = f.xmc[col2(d, j, 1)];
    if (code == kNoFlux) q = 0.0;
    else if (code == kFlux) q = -f.xmv[col2(d, j, 1)] * faceA;
    return q;
  }
  const long long e = c + d.sx;
  double kf, delta = d.dx;
  const double sg = (f.bot[e] > f.bot[c]) ? 1.0 : -1.0;
  if (i == d.nx) {
    kf = pk.kcx[c];
    delta = 0.5 * d.dx;
  } else {
    if (d.pc) {
      kf = d.harm ? face_harm(pk.kcx[c], f.ksx[c], 1.0, pk.kcx[e], f.ksx[e], 1.0)
                  : 0.5 * (pk.kcx[c] + pk.kcx[e]);
    } else {
      kf = 0.5 * (pk.kcx[c] + vg_k(soil_at(f, e), hp[e], f.ksx[c]));
    }
    if (!f.act[c] || !f.act[e]) kf = 0.0;
  }
  q = faceA * (kf * f.cosx[c] * (hp[e] - hp[c]) / delta + sg * kf * f.sinx[c]);
  if (!d.full3d && ((f.act[c] && wcn[c] < f.wcs[c]) || (f.act[e] && wcn[e] < f.wcs[e]))) q = 0.0;
  if (i == d.nx) {
    const int code = f.xpc[col2(d, j, d.nx)];
    if (code == kNoFlux) q = 0.0;
    else if (code == kFlux) q = f.xpv[col2(d, j, d.nx)] * faceA;
  }
  return q;
}

__device__ inline double flux_y(const Dims& d, const Fields& f, const PassK& pk,
                                const double* hp, const double* wcn, int j, int i, int k) {
  const long long c = cidx(d, j, i, k);
  const double faceA = f.ay[c];
  double q;
  if (j == 0) {
    const long long ci = c + d.sy;
    q = faceA * pk.kcy[ci] * f.cosy[c] * (hp[ci] - hp[c]) / (0.5 * d.dy);
    const int code = f.ymc[col2(d, 1, i)];
    if (code == kNoFlux) q = 0.0;
    else if (code == kFlux) q = -f.ymv[col2(d, 1, i)] * faceA;
    return q;
  }
  const long long n = c + d.sy;
  double kf, delta = d.dy;
  const double sg = (f.bot[n] > f.bot[c]) ? 1.0 : -1.0;
  if (j == d.ny) {
    kf = pk.kcy[c];
    delta = 0.5 * d.dy;
  } else {
    if (d.pc) {
      kf = d.harm ? face_harm(pk.kcy[c], f.ksy[c], 1.0, pk.kcy[n], f.ksy[n], 1.0)
                  : 0.5 * (pk.kcy[c] + pk.kcy[n]);
    } else {
      kf = 0.5 * (pk.kcy[c] + vg_k(soil_at(f, n), hp[n], f.ksy[c]));
    }
    if (!f.act[c] || !f.act[n]) kf = 0.0;
  }
  q = faceA * (kf * f.cosy[c] * (hp[n] - hp[c]) / delta + sg * kf * f.siny[c]);
  if (!d.full3d && ((f.act[c] && wcn[c] < f.wcs[c]) || (f.act[n] && wcn[n] < f.wcs[n]))) q = 0.0;
  if (j == d.ny) {
    const int code = f.ypc[col2(d, d.ny, i)];
    if (code == kNoFlux) q = 0.0;
    else if (code == kFlux) q = f.ypv[col2(d, d.ny, i)] * faceA;
  }
  return q;
}

__device__ inline double flux_z(const Dims& d, const Fields& f, const PassK& pk,
                                const double* hp, int j, int i, int k) {
  const long long base = cidx(d, j, i, 0), col = col2(d, j, i);
  const bool below = (k < d.nz) && f.act[base + k];
  const bool above = (k >= 1) && f.act[base + k - 1];
  if (below && !above) {  // face above a column's top cell
    const long long c = base + k;
    const int code = f.topc[col];
    if (code == kFlux) return f.topv[col] * d.az;
    if (code == kHead) {
      const double delta = 0.5 * f.dz[c];
      return d.az * f.ksz[c] * ((hp[c] - f.topv[col]) / delta - 1.0);
    }
    return 0.0;
  }
  if (k == d.nz && above) {  // bottom boundary face
    const long long c = base + d.nz - 1;
    const int code = f.botc[col];
    const double kf = pk.kcz[c];
    if (code == kFlux) return f.botv[col] * d.az;
    if (code == kGravity) return -kf * d.az;
    if (code == kHead) {
      const double delta = 0.5 * f.dz[c];
      return d.az * kf * ((f.botv[col] - hp[c]) / delta - 1.0);
    }
    return 0.0;
  }
  if (above && below) {
    const long long up = base + k - 1, lo = base + k;
    double kf;
    if (d.pc) {
      kf = d.harm ? face_harm(pk.kcz[up], f.ksz[up], f.dz[up], pk.kcz[lo], f.ksz[lo], f.dz[lo])
                  : 0.5 * (pk.kcz[up] + pk.kcz[lo]);
    } else {
      kf = 0.5 * (vg_k(soil_at(f, up), hp[up], f.ksz[lo]) + pk.kcz[lo]);
    }
    const double delta = 0.5 * (f.dz[up] + f.dz[lo]);
    return d.az * kf * ((hp[lo] - hp[up]) / delta - 1.0);
  }
  return 0.0;
}

__global__ void k_flux(Dims d, Fields f, PassK pk, const double* __restrict__ hp,
                       const double* __restrict__ wcn, double* kx, double* ky, double* kzf,
                       double* qx, double* qy, double* qzf) {
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const bool jin = j >= 1 && j <= d.ny, iin = i >= 1 && i <= d.nx;
    if (jin && i <= d.nx) {
      kx[c] = face_kx(d, f, pk, j, i, k);
      qx[c] = flux_x(d, f, pk, hp, wcn, j, i, k);
    }
    if (iin && j <= d.ny) {
      ky[c] = face_ky(d, f, pk, j, i, k);
      qy[c] = flux_y(d, f, pk, hp, wcn, j, i, k);
    }
    if (jin && iin) {
      const long long fz = fidx(d, j, i, k);
      kzf[fz] = face_kz(d, f, pk, j, i, k);
      qzf[fz] = flux_z(d, f, pk, hp, j, i, k);
      if (k == d.nz - 1) {
        kzf[fz + 1] = face_kz(d, f, pk, j, i, d.nz);
        qzf[fz + 1] = flux_z(d, f, pk, hp, j, i, d.nz);
      }
    }
  }
}

// ---------------------------------------------------------------- theta update
// theta from the flux divergence with the Ss factor, and the Ss audit term
// (updateWaterContent, Corrector.cpp:629-672).  Cells outside the update keep
// theta^n, so the output buffer is a full copy.
//
// The same pass writes the saturation flag of every cell (theta >= theta_s or
// h > h_ae on the corrected theta and predicted head, ghosts included) that
// the post-allocation classification tests on the six neighbours of a cell.
// All loads of a cell are issued before its first store and before any
// branch on loaded data, so one memory round trip serves the cell.
__global__ void __launch_bounds__(kBlock) k_update_wc(
    Dims d, Fields f, const double* __restrict__ hp, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ qx, const double* __restrict__ qy,
    const double* __restrict__ qzf, double dtg, double* __restrict__ wcu,
    uint8_t* __restrict__ satf, double* partial) {
  double acc = 0.0;
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const bool in = j >= 1 && j <= d.ny && i >= 1 && i <= d.nx;
    const double w0 = wcn[c], hpc = hp[c], ts = f.wcs[c], aev = f.aev[c];
    double upd = w0;
    if (in) {
      const long long fz = fidx(d, j, i, k);
      const int8_t ac = f.act[c];
      const double hnc = hn[c], dzc = f.dz[c];
      const double qxp = qx[c], qxm = qx[c - d.sx], qyp = qy[c], qym = qy[c - d.sy];
      const double qzt = qzf[fz], qzb = qzf[fz + 1];
      if (ac) {
        const double volume = d.az * dzc;
        const double dh = hpc - hnc;
        const double coeff = volume * (1.0 + d.ss * dh / ts);
        const double dqx = dtg * (qxp - qxm);
        const double dqy = dtg * (qyp - qym);
        const double dqz = dtg * (qzb - qzt);
        upd = (w0 * volume + dqx + dqy + dqz) / coeff;
        acc += upd * volume * d.ss * dh / ts;
      }
    }
    wcu[c] = upd;
    satf[c] = (upd >= ts || hpc > aev) ? 1 : 0;
  }
  const double s = block_reduce(acc, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// ---------------------------------------------------------------- post-allocation
// The six-direction gradient split (check_head_gradient as restated by
// Reallocate.cpp:205-274), on the pre-sweep head.
struct Split {
  double up, down;
};
// The six-face gradient split of a cell's surplus (Reallocate.cpp:235-300)
// on values the caller has already loaded: heads hR of the cell and its six
// neighbours (x+, x-, y+, y-, z+ below, z- above), the neighbours' activity,
// the face conductivities and the three layer thicknesses.
struct SplitIn {
  double hc, hxp, hxm, hyp, hym, hzp, hzm;
  double kxp, kxm, kyp, kym, kzb, kzt;
  double dzc, dzp, dzm;
  int8_t axp, axm, ayp, aym, azp, azm;
};

__device__ inline Split gradient_split(const Dims& d, const SplitIn& n, int k) {
  double dh0 = 0.0, dh1 = 0.0, dh2 = 0.0, dh3 = 0.0, dh4 = 0.0, dh5 = 0.0;
  if (d.full3d) {
    if (n.axp && n.kxp > 0.0) dh0 = (n.hxp - n.hc) / d.dx;
    if (n.axm && n.kxm > 0.0) dh1 = (n.hc - n.hxm) / d.dx;
    if (n.ayp && n.kyp > 0.0) dh2 = (n.hyp - n.hc) / d.dy;
    if (n.aym && n.kym > 0.0) dh3 = (n.hc - n.hym) / d.dy;
  }
  if (k + 1 < d.nz && n.azp && n.kzb > 0.0) {
    const double dzp = 0.5 * (n.dzc + n.dzp);
    dh4 = (n.hzp - n.hc) / dzp - 1.0;
  }
  if (k >= 1 && n.azm && n.kzt > 0.0) {
    const double dzm = 0.5 * (n.dzc + n.dzm);
    dh5 = (n.hc - n.hzm) / dzm - 1.0;
  }
  double tot = 0.0, gz;
  if (dh0 * dh1 >= 0.0) tot += fabs(0.5 * (dh0 + dh1));
  else tot += fabs(dh0) + fabs(dh1);
  if (dh2 * dh3 >= 0.0) tot += fabs(0.5 * (dh2 + dh3));
  else tot += fabs(dh2) + fabs(dh3);
  if (dh4 * dh5 >= 0.0) {
    gz = 0.5 * (dh4 + dh5);
    tot += fabs(gz);
  } else {
    gz = 0.0;
    tot += fabs(dh4) + fabs(dh5);
  }
  Split s{0.0, 0.0};
  if (tot > 0.0) {
    if (gz > 0.0) s.up = gz / tot;
    else if (gz < 0.0) s.down = -gz / tot;
    else {
      s.down = fabs(dh4) / tot;
      s.up = fabs(dh5) / tot;
    }
  }
  return s;
}

// Phase 1 of the post-allocation (reallocateWaterContent's classification,
// Reallocate.cpp:181-391, saturated_contact: head): reads the corrected theta
// and predicted head as the pre-sweep snapshot, writes the restored state to
// separate buffers, so the classification is race-free by construction.  The
// neighbour-saturation tests read the flags k_update_wc wrote from the same
// snapshot.  Every load of an interior cell, its neighbours included, is
// issued before the first branch on loaded data.
__global__ void __launch_bounds__(kBlock, 3) k_classify(
    Dims d, Fields f, const double* __restrict__ kx, const double* __restrict__ ky,
    const double* __restrict__ kzf, const double* __restrict__ wcR,
    const double* __restrict__ hR, const uint8_t* __restrict__ satf, double* __restrict__ wc_out,
    double* __restrict__ h_out, double* __restrict__ room, double* __restrict__ sup,
    double* __restrict__ sdn, int* colflag, double* part_adj, double* part_drop) {
  double adj = 0.0, drop = 0.0;
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const double before = wcR[c];
    double wout = before, hout = hR[c], rm = 0.0, up = 0.0, dn = 0.0;
    const bool in = j >= 1 && j <= d.ny && i >= 1 && i <= d.nx;
    if (in) {
      const long long col = col2(d, j, i), fz = fidx(d, j, i, k);
      const long long cp = (k + 1 < d.nz) ? c + 1 : c, cm = (k >= 1) ? c - 1 : c;
      SplitIn n;
      n.hc = hout;
      n.hxp = hR[c + d.sx];
      n.hxm = hR[c - d.sx];
      n.hyp = hR[c + d.sy];
      n.hym = hR[c - d.sy];
      n.hzp = hR[cp];
      n.hzm = hR[cm];
      n.kxp = kx[c];
      n.kxm = kx[c - d.sx];
      n.kyp = ky[c];
      n.kym = ky[c - d.sy];
      n.kzt = kzf[fz];
      n.kzb = kzf[fz + 1];
      n.dzc = f.dz[c];
      n.dzp = f.dz[cp];
      n.dzm = f.dz[cm];
      n.axp = f.act[c + d.sx];
      n.axm = f.act[c - d.sx];
      n.ayp = f.act[c + d.sy];
      n.aym = f.act[c - d.sy];
      n.azp = (k + 1 < d.nz) ? f.act[cp] : 0;
      n.azm = (k >= 1) ? f.act[cm] : 0;
      const int8_t ac = f.act[c];
      const uint8_t sxp = satf[c + d.sx], sxm = satf[c - d.sx], syp = satf[c + d.sy],
                    sym = satf[c - d.sy], szp = satf[cp], szm = satf[cm];
      const int topc = f.topc[col];
      const double topv = f.topv[col];
      const Soil so = soil_at(f, c);
      if (ac) {
        const double volume = d.az * n.dzc;
        if (before >= so.ts) {
          if (!d.off) {
            const double excess = (before - so.ts) * volume;
            const Split sp = gradient_split(d, n, k);
            up = excess * sp.up;
            dn = excess * sp.down;
            adj -= excess - up - dn;
            drop += excess - up - dn;
            wout = so.ts;
          }
        } else {
          rm = (so.ts - before) * volume;
          const bool top = (k == 0) || !n.azm;
          const bool adjsat = (n.azp && szp) || (n.kxp != 0.0 && sxp) ||
                              (n.kxm != 0.0 && sxm) || (n.kyp != 0.0 && syp) ||
                              (n.kym != 0.0 && sym) ||
                              (top ? (topc == kHead && topv >= 0.0) : (szm != 0));
          if (!adjsat) {
            if (before < 0.9999 * so.ts) hout = vg_head(so, before);
          } else if (!d.off) {
            const double after = vg_theta(so, hout);
            wout = after;
            rm = (so.ts - after) * volume;
            if (d.redistribute && after < before) {
              const double surplus = (before - after) * volume;
              const Split sp = gradient_split(d, n, k);
              up = surplus * sp.up;
              dn = surplus * sp.down;
              adj -= surplus - up - dn;
              drop += surplus - up - dn;
            } else {
              adj += (after - before) * volume;
              if (after < before) drop += (before - after) * volume;
            }
          }
        }
        if (up > 0.0 || dn > 0.0) colflag[col] = 1;
      }
    }
    wc_out[c] = wout;
    h_out[c] = hout;
    room[c] = rm;
    sup[c] = up;
    sdn[c] = dn;
  }
  const double s1 = block_reduce(adj, SumOp(), 0.0);
  if (threadIdx.x == 0) part_adj[blockIdx.x] = s1;
  const double s2 = block_reduce(drop, SumOp(), 0.0);
  if (threadIdx.x == 0) part_drop[blockIdx.x] = s2;
}

// Phase 2: the vertical send walks, one thread per flagged column, k
// ascending (Reallocate.cpp:410-540, uncoupled, no transport window).
__global__ void k_walk_thread(Dims d, Fields f, double* wc, double* room, const double* __restrict__ sup,
                       const double* __restrict__ sdn, double* qzf, const int* __restrict__ colflag,
                       double dtg, double* partial) {
  double lost = 0.0;
  const long long ncolint = static_cast<long long>(d.nx) * d.ny;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < ncolint;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    if (!colflag[col]) continue;
    const long long base = cidx(d, j, i, 0), fb = fidx(d, j, i, 0);
    const bool topHead = f.topc[col] == kHead;
    for (int k = 0; k < d.nz; ++k) {
      if (!f.act[base + k]) continue;
      double dv = sup[base + k];
      if (dv > 0.0) {
        int ll = k;
        while (ll > 0 && f.act[base + ll - 1] && dv > 0.0) {
          --ll;
          const long long c = base + ll;
          if (room[c] > 0.0) {
            const double take = (room[c] > dv) ? dv : room[c];
            wc[c] += take / (d.az * f.dz[c]);
            room[c] -= take;
            qzf[fb + ll + 1] += take / dtg;
            dv -= take;
          }
        }
        if (dv > 0.0) {
          if (topHead) {
            qzf[fb + ll] += dv / dtg;
          } else {
            while (ll + 1 < d.nz && dv > 0.0) {
              ++ll;
              const long long c = base + ll;
              if (room[c] > 0.0) {
                const double take = (room[c] > dv) ? dv : room[c];
                wc[c] += take / (d.az * f.dz[c]);
                room[c] -= take;
                qzf[fb + ll] -= take / dtg;
                dv -= take;
              }
            }
            lost -= dv;
          }
        }
      }
      dv = sdn[base + k];
      if (dv > 0.0) {
        int ll = k;
        while (ll + 1 < d.nz && dv > 0.0) {
          ++ll;
          const long long c = base + ll;
          if (room[c] > 0.0) {
            const double take = (room[c] > dv) ? dv : room[c];
            wc[c] += take / (d.az * f.dz[c]);
            room[c] -= take;
            qzf[fb + ll] -= take / dtg;
            dv -= take;
          }
        }
        lost -= dv;
      }
    }
  }
  const double s = block_reduce(lost, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// The same walk with one warp per flagged column.  The column's room, theta,
// cell volume and face fluxes are staged in shared memory (coalesced), with
// two bit sets per column: the cells that still have room and the inactive
// cells.  A ballot over each 32-cell chunk finds the surplus cells in
// ascending k, and lane 0 runs each walk on shared memory, jumping straight
// to the next cell with room (a cell without room takes nothing, so the walk
// may skip it) and stopping where the per-thread walk stops.  The deposit
// order and every rounding step are those of the per-thread walk above.
// Shared memory per warp: walk_warp_bytes(nz).
constexpr int kWalkWarps = kBlock / 32;
__host__ __device__ inline int walk_words(int nz) { return (nz + 31) / 32; }
__host__ __device__ inline size_t walk_warp_bytes(int nz) {
  return static_cast<size_t>(4 * nz + 1) * sizeof(double) +
         static_cast<size_t>(2 * walk_words(nz)) * sizeof(unsigned);
}

// Largest m in [lo, hi] whose bit is set, or -1.
__device__ inline int bits_highest(const unsigned* w, int lo, int hi) {
  if (hi < lo) return -1;
  int wi = hi >> 5;
  unsigned m = w[wi] & (0xffffffffu >> (31 - (hi & 31)));
  const int wlo = lo >> 5;
  for (;;) {
    if (m) {
      const int pos = (wi << 5) + 31 - __clz(m);
      return pos >= lo ? pos : -1;
    }
    if (--wi < wlo) return -1;
    m = w[wi];
  }
}

// Smallest m in [lo, hi] whose bit is set, or -1.
__device__ inline int bits_lowest(const unsigned* w, int lo, int hi) {
  if (hi < lo) return -1;
  int wi = lo >> 5;
  unsigned m = w[wi] & (0xffffffffu << (lo & 31));
  const int whi = hi >> 5;
  for (;;) {
    if (m) {
      const int pos = (wi << 5) + __ffs(m) - 1;
      return pos <= hi ? pos : -1;
    }
    if (++wi > whi) return -1;
    m = w[wi];
  }
}

// Deposit at cell m: take min(room, dv), add take / dtg to face `face` with
// `plus` (true: +=, false: -=), and clear m's room bit once its room is used up.
__device__ inline void walk_take(double& dv, int m, double* rs, double* ws, const double* vs,
                                 double* qs, unsigned* rbits, int face, bool plus, double dtg) {
  const double take = (rs[m] > dv) ? dv : rs[m];
  ws[m] += take / vs[m];
  rs[m] -= take;
  if (plus) {
    qs[face] += take / dtg;
  } else {
    qs[face] -= take / dtg;
  }
  dv -= take;
  if (!(rs[m] > 0.0)) rbits[m >> 5] &= ~(1u << (m & 31));
}

__global__ void __launch_bounds__(kBlock) k_walk(Dims d, Fields f, double* wc,
                                                 const double* __restrict__ room,
                                                 const double* __restrict__ sup,
                                                 const double* __restrict__ sdn, double* qzf,
                                                 const int* __restrict__ colflag, double dtg,
                                                 double* partial) {
  extern __shared__ __align__(16) unsigned char walk_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nz = d.nz, nw = walk_words(nz);
  double* rs = reinterpret_cast<double*>(walk_smem + warp * walk_warp_bytes(nz));
  double* ws = rs + nz;
  double* vs = ws + nz;
  double* qs = vs + nz;  // nz + 1 faces
  unsigned* rbits = reinterpret_cast<unsigned*>(qs + nz + 1);
  unsigned* ibits = rbits + nw;  // inactive cells
  double lost = 0.0;
  const long long ncolint = static_cast<long long>(d.nx) * d.ny;
  const long long nwarps = static_cast<long long>(gridDim.x) * kWalkWarps;
  for (long long t = blockIdx.x * static_cast<long long>(kWalkWarps) + warp; t < ncolint;
       t += nwarps) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    if (!colflag[col]) continue;
    const long long base = cidx(d, j, i, 0), fb = fidx(d, j, i, 0);
    const bool topHead = f.topc[col] == kHead;
    for (int k0 = 0; k0 < nz; k0 += 32) {
      const int k = k0 + lane;
      double r = 0.0;
      bool inact = false;
      if (k < nz) {
        r = room[base + k];
        rs[k] = r;
        ws[k] = wc[base + k];
        vs[k] = d.az * f.dz[base + k];
        inact = !f.act[base + k];
      }
      const unsigned rb = __ballot_sync(0xffffffffu, r > 0.0);
      const unsigned ib = __ballot_sync(0xffffffffu, inact);
      if (lane == 0) {
        rbits[k0 >> 5] = rb;
        ibits[k0 >> 5] = ib;
      }
    }
    for (int k = lane; k <= nz; k += 32) qs[k] = qzf[fb + k];
    __syncwarp();
    for (int k0 = 0; k0 < nz; k0 += 32) {
      const int k = k0 + lane;
      double su = 0.0, sd = 0.0;
      bool any = false;
      if (k < nz && f.act[base + k]) {
        su = sup[base + k];
        sd = sdn[base + k];
        any = su > 0.0 || sd > 0.0;
      }
      unsigned mask = __ballot_sync(0xffffffffu, any);
      while (mask) {
        const int b = __ffs(mask) - 1;
        mask &= mask - 1;
        const double upv = __shfl_sync(0xffffffffu, su, b);
        const double dnv = __shfl_sync(0xffffffffu, sd, b);
        if (lane == 0) {
          const int kk = k0 + b;
          double dv = upv;
          if (dv > 0.0) {
            // Upward: cells kk-1, kk-2, ... up to the first inactive cell above
            // kk (exclusive) or the surface.
            const int lim = bits_highest(ibits, 0, kk - 1) + 1;
            int ll = kk;
            while (dv > 0.0) {
              const int m = bits_highest(rbits, lim, ll - 1);
              if (m < 0) {
                ll = lim;
                break;
              }
              walk_take(dv, m, rs, ws, vs, qs, rbits, m + 1, true, dtg);
              ll = m;
            }
            if (dv > 0.0) {
              if (topHead) {
                qs[ll] += dv / dtg;
              } else {
                while (dv > 0.0) {
                  const int m = bits_lowest(rbits, ll + 1, nz - 1);
                  if (m < 0) break;
                  walk_take(dv, m, rs, ws, vs, qs, rbits, m, false, dtg);
                  ll = m;
                }
                lost -= dv;
              }
            }
          }
          dv = dnv;
          if (dv > 0.0) {
            int ll = kk;
            while (dv > 0.0) {
              const int m = bits_lowest(rbits, ll + 1, nz - 1);
              if (m < 0) break;
              walk_take(dv, m, rs, ws, vs, qs, rbits, m, false, dtg);
              ll = m;
            }
            lost -= dv;
          }
        }
        __syncwarp();
      }
    }
    for (int k = lane; k < nz; k += 32) wc[base + k] = ws[k];
    for (int k = lane; k <= nz; k += 32) qzf[fb + k] = qs[k];
    __syncwarp();
  }
  const double s = block_reduce(lost, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// ---------------------------------------------------------------- clamp, audit, controller
// finalizeWaterContent (Corrector.cpp:758-792), accumulateBoundaryFlux
// (RichardsSolver.cpp:961-1006), the adaptTimeStep inputs (AdaptiveStep.cpp:
// 58-98) and the owned volume (RichardsSolver.cpp:892-912), in one sweep.
__global__ void __launch_bounds__(kBlock, 3) k_finalize(Dims d, Fields f, double* wc, double* vloss,
                           const double* __restrict__ qx, const double* __restrict__ qy,
                           const double* __restrict__ qzf, double dtg, double co_max,
                           double* partial, int nblk) {
  double vl = 0.0, inflow = 0.0, dqmax = -DBL_MAX, dtco = DBL_MAX, vol = 0.0;
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    if (j < 1 || j > d.ny || i < 1 || i > d.nx || !f.act[c]) continue;
    const double volume = d.az * f.dz[c];
    double w = wc[c];
    if (w > f.wcs[c]) {
      const double ex = (w - f.wcs[c]) * volume;
      vloss[c] += ex;
      vl += ex;
      w = f.wcs[c];
      wc[c] = w;
    } else if (w < f.wcr[c]) {
      const double de = (f.wcr[c] - w) * volume;
      vloss[c] -= de;
      vl -= de;
      w = f.wcr[c];
      wc[c] = w;
    }
    vol += w * d.az * f.dz[c];
    const long long fz = fidx(d, j, i, k);
    const bool top = (k == 0) || !f.act[c - 1];
    if (top) inflow -= qzf[fz] * dtg;
    if (k == d.nz - 1) inflow += qzf[fz + 1] * dtg;
    if (i == 1) inflow -= qx[c - d.sx] * dtg;
    if (i == d.nx) inflow += qx[c] * dtg;
    if (j == 1) inflow -= qy[c - d.sy] * dtg;
    if (j == d.ny) inflow += qy[c] * dtg;
    if (!top) {
      const double qin = qx[c] / f.ax[c] + qy[c] / f.ay[c] + qzf[fz + 1] / d.az;
      const double qou = qx[c - d.sx] / f.ax[c] + qy[c - d.sy] / f.ay[c] + qzf[fz] / d.az;
      const double dq = fabs(qin - qou) * dtg / f.dz[c];
      if (dq > dqmax) dqmax = dq;
      if (w < f.wcs[c]) {
        const double dk = vg_dkdtheta(soil_at(f, c), w, f.ksz[c]);
        const double t = co_max * f.dz[c] / dk;
        if (t < dtco) dtco = t;
      }
    }
  }
  double s = block_reduce(vl, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPVloss * nblk + blockIdx.x] = s;
  s = block_reduce(inflow, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPInflow * nblk + blockIdx.x] = s;
  s = block_reduce(dqmax, MaxOp(), -DBL_MAX);
  if (threadIdx.x == 0) partial[kPDqmax * nblk + blockIdx.x] = s;
  s = block_reduce(dtco, MinOp(), DBL_MAX);
  if (threadIdx.x == 0) partial[kPDtco * nblk + blockIdx.x] = s;
  s = block_reduce(vol, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPVol * nblk + blockIdx.x] = s;
}

__global__ void k_volume(Dims d, Fields f, const double* __restrict__ wc, double* partial) {
  double vol = 0.0;
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    if (j < 1 || j > d.ny || i < 1 || i > d.nx || !f.act[c]) continue;
    vol += wc[c] * d.az * f.dz[c];
  }
  const double s = block_reduce(vol, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// applyInitialConditions (RichardsSolver.cpp:331-427) for every interior cell
// (active or not): moisture -> h from the retention curve (hydrostatic from
// the bed where saturated), head -> theta(h), water table -> hydrostatic head
// about the table (given in the unshifted datum) and theta(h).  `field` is
// per cell (moisture, head) or per column (water table) in the ABI's
// interior order, or null for the constant.
__global__ void k_init_state(Dims d, Fields f, int form, double constant,
                             const double* __restrict__ field, const double* __restrict__ bath,
                             double offset, double* h, double* wc) {
  for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    if (j < 1 || j > d.ny || i < 1 || i > d.nx) {
      h[c] = 0.0;
      wc[c] = 0.0;
      continue;
    }
    const long long col = static_cast<long long>(j - 1) * d.nx + (i - 1);
    double value = constant;
    if (field) value = (form == 2) ? field[col] : field[col * d.nz + k];
    const Soil so = soil_at(f, c);
    const double zc = f.bot[c] + 0.5 * f.dz[c];
    double hv, wv;
    if (form == 0) {
      wv = value;
      hv = (wv >= so.ts) ? (bath[col2(d, j, i)] - zc) : vg_head(so, wv);
    } else if (form == 1) {
      hv = value;
      wv = vg_theta(so, hv);
    } else {
      hv = (value + offset) - zc;
      wv = vg_theta(so, hv);
    }
    h[c] = hv;
    wc[c] = wv;
  }
}

template <class Op>
__device__ double reduce_slot(const double* p, int n, Op op, double identity) {
  double v = identity;
  for (int b = threadIdx.x; b < n; b += blockDim.x) v = op(v, p[b]);
  return block_reduce(v, op, identity);
}

// One block: combine the partials in block order into the step record and run
// the controller (adaptTimeStep, AdaptiveStep.cpp:100-117; grow 1.25, shrink
// 0.75, Courant cap, [dt_min, dt_max] clamp).
__global__ void k_step_info(const double* partial, int nblk, int off, double dtg, double dq_grow,
                            double dq_shrink, double dt_min, double dt_max, StepOut* out) {
  const double ss = reduce_slot(partial + kPSs * nblk, nblk, SumOp(), 0.0);
  const double adj = reduce_slot(partial + kPAdj * nblk, nblk, SumOp(), 0.0);
  const double drop = reduce_slot(partial + kPDrop * nblk, nblk, SumOp(), 0.0);
  const double lost = reduce_slot(partial + kPLost * nblk, nblk, SumOp(), 0.0);
  const double vl = reduce_slot(partial + kPVloss * nblk, nblk, SumOp(), 0.0);
  const double inflow = reduce_slot(partial + kPInflow * nblk, nblk, SumOp(), 0.0);
  const double dqmax = reduce_slot(partial + kPDqmax * nblk, nblk, MaxOp(), -DBL_MAX);
  const double dtco = reduce_slot(partial + kPDtco * nblk, nblk, MinOp(), DBL_MAX);
  const double vol = reduce_slot(partial + kPVol * nblk, nblk, SumOp(), 0.0);
  if (threadIdx.x == 0) {
    out->ss_storage = ss;
    out->realloc_adjust = off ? 0.0 : adj + lost;
    out->realloc_dropped = off ? 0.0 : drop - lost;
    out->vloss = vl;
    out->boundary_in = inflow;
    out->dqmax = dqmax;
    out->dtco = dtco;
    out->volume = vol;
    double next = dtg;
    if (dqmax > dq_shrink) next = dtg * 0.75;
    else if (dqmax < dq_grow) next = dtg * 1.25;
    if (next > dtco) next = dtco;
    if (next > dt_max) next = dt_max;
    if (next < dt_min) next = dt_min;
    out->next_dt = next;
  }
}

__global__ void k_volume_final(const double* partial, int nblk, StepOut* out) {
  const double vol = reduce_slot(partial, nblk, SumOp(), 0.0);
  if (threadIdx.x == 0) out->volume = vol;
}

}  // namespace

// ---------------------------------------------------------------- launchers
void launch_ghosts(const Device& D, double* h, double* wc) {
  const long long n = 2LL * (D.d.nx + D.d.ny) * D.d.nz;
  const int g = static_cast<int>(std::min<long long>((n + kBlock - 1) / kBlock, 4096));
  k_ghosts<<<g, kBlock, 0, D.stream>>>(D.d, D.f, h, wc);
  ++D.launches;
}

void launch_closure_pred(const Device& D, const double* h) {
  k_closure_pred<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, h, D.kcx, D.kcy, D.kcz,
                                                         D.ch);
  ++D.launches;
}

void launch_assemble(const Device& D, const double* hn, const double* wcn, double dtg) {
  PassK pk{D.kcx, D.kcy, D.kcz, wcn};
  k_assemble<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, pk, hn, wcn, D.ch, dtg, D.diag,
                                                     D.gxp, D.gyp, D.gzp, D.rhs);
  ++D.launches;
}

void launch_closure_corr(const Device& D, const double* hn) {
  k_closure_corr<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.x, hn, D.hp, D.kcx, D.kcy,
                                                         D.kcz);
  ++D.launches;
}

void launch_flux(const Device& D, const double* wcn, double dtg) {
  (void)dtg;
  PassK pk{D.kcx, D.kcy, D.kcz, wcn};
  k_flux<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, pk, D.hp, wcn, D.kx, D.ky, D.kzf, D.qx,
                                                 D.qy, D.qzf);
  ++D.launches;
}

void launch_update_wc(const Device& D, const double* hn, const double* wcn, double dtg) {
  k_update_wc<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.hp, hn, wcn, D.qx, D.qy, D.qzf,
                                                      dtg, D.wcu, D.satf, D.partial + kPSs * D.nblk);
  ++D.launches;
}

void launch_classify(const Device& D, double* wc_out, double* h_out) {
  cudaMemsetAsync(D.colflag, 0, sizeof(int) * D.d.ncol, D.stream);
  k_classify<<<cells_grid(D), kBlock, 0, D.stream>>>(
      D.d, D.f, D.kx, D.ky, D.kzf, D.wcu, D.hp, D.satf, wc_out, h_out, D.room, D.sup, D.sdn,
      D.colflag,
      D.partial + kPAdj * D.nblk, D.partial + kPDrop * D.nblk);
  ++D.launches;
}

// Columns deeper than the shared-memory staging allows take the per-thread walk.
constexpr size_t kWalkSmemMax = 48 * 1024;

void launch_walk(const Device& D, double* wc_out, double dtg) {
  const size_t smem = kWalkWarps * walk_warp_bytes(D.d.nz);
  if (smem <= kWalkSmemMax) {
    k_walk<<<cells_grid(D), kBlock, smem, D.stream>>>(D.d, D.f, wc_out, D.room, D.sup, D.sdn,
                                                      D.qzf, D.colflag, dtg,
                                                      D.partial + kPLost * D.nblk);
  } else {
    k_walk_thread<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, wc_out, D.room, D.sup, D.sdn,
                                                          D.qzf, D.colflag, dtg,
                                                          D.partial + kPLost * D.nblk);
  }
  ++D.launches;
}

void launch_finalize(const Device& D, double* wc_out, double dtg, double co_max) {
  k_finalize<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, wc_out, D.vloss, D.qx, D.qy,
                                                     D.qzf, dtg, co_max, D.partial, D.nblk);
  ++D.launches;
}

void launch_step_info(const Device& D, double dtg, double dq_grow, double dq_shrink,
                      double dt_min, double dt_max) {
  k_step_info<<<1, kBlock, 0, D.stream>>>(D.partial, D.nblk, D.d.off, dtg, dq_grow, dq_shrink,
                                          dt_min, dt_max, D.out);
  ++D.launches;
}

void launch_init_state(const Device& D, int form, double constant, const double* field,
                       const double* bath, double offset) {
  k_init_state<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, form, constant, field, bath,
                                                       offset, D.h[D.cur], D.wc[D.cur]);
  ++D.launches;
}

void launch_volume(const Device& D, const double* wc) {
  k_volume<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, wc, D.partial + kPVol * D.nblk);
  ++D.launches;
  k_volume_final<<<1, kBlock, 0, D.stream>>>(D.partial + kPVol * D.nblk, D.nblk, D.out);
  ++D.launches;
}

}  // namespace fgw
