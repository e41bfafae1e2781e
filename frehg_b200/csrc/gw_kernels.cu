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
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <map>
#include <mutex>

#include "gw_coop.cuh"
#include "gw_internal.h"
#include "gw_linefactor.cuh"

namespace fgw {

namespace {

__device__ inline double ghost_head(int code, double value, double interior, double zc,
                                    double r) {
  // enforceHeadBc / ghostHead, uncoupled (src/gw/Predictor.cpp:66-87); r =
  // the edge face's density ratio.
  if (code == kHead) return value;
  if (code == kHydro) return (value - zc) * r;
  return interior;
}

// ghostHead with the coupled rule (Predictor.cpp:80-83): a hydrostatic stage
// above the edge column's bed follows the live surface there, (bed - zc) r +
// depth (depth r on the plus sides).  cc = the edge column.
__device__ inline double ghost_head_at(const Dims& d, const Fields& f, int code, double value,
                                       double interior, double zc, long long cc, double r,
                                       bool plus) {
  if (code == kHydro && (f.cpl != nullptr)) {
    const double bed = f.cpl->bath[cc];
    if (value > bed) {
      const double hydro = (bed - zc) * r;
      return plus ? hydro + f.cpl->dept[cc] * r : hydro + f.cpl->dept[cc];
    }
  }
  return ghost_head(code, value, interior, zc, r);
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
__device__ __forceinline__ void ghosts_body(Dims d, Fields f, double* h, double* wc, const int bid, const int G) {
  const long long nxg = 2LL * d.ny * d.nz, nyg = 2LL * d.nx * d.nz;
  for (long long t = bid * static_cast<long long>(blockDim.x) + threadIdx.x; t < nxg + nyg;
       t += static_cast<long long>(G) * blockDim.x) {
    long long g, c, cc;
    int code;
    double val;
    bool plus, xs;
    if (t < nxg) {
      const int side = static_cast<int>(t / (static_cast<long long>(d.ny) * d.nz));
      const long long rem = t - static_cast<long long>(side) * d.ny * d.nz;
      const int j = static_cast<int>(rem / d.nz) + 1, k = static_cast<int>(rem % d.nz);
      const int ii = side == 0 ? 1 : d.nx;
      c = cidx(d, j, ii, k);
      g = side == 0 ? c - d.sx : c + d.sx;
      cc = col2(d, j, ii);
      code = side == 0 ? f.xmc[cc] : f.xpc[cc];
      val = side == 0 ? f.xmv[cc] : f.xpv[cc];
      plus = side != 0;
      xs = true;
    } else {
      const long long u = t - nxg;
      const int side = static_cast<int>(u / (static_cast<long long>(d.nx) * d.nz));
      const long long rem = u - static_cast<long long>(side) * d.nx * d.nz;
      const int i = static_cast<int>(rem / d.nz) + 1, k = static_cast<int>(rem % d.nz);
      const int jj = side == 0 ? 1 : d.ny;
      c = cidx(d, jj, i, k);
      g = side == 0 ? c - d.sy : c + d.sy;
      cc = col2(d, jj, i);
      code = side == 0 ? f.ymc[cc] : f.ypc[cc];
      val = side == 0 ? f.ymv[cc] : f.ypv[cc];
      plus = side != 0;
      xs = false;
    }
    // the edge face's density ratio: slot g on the minus sides, c on the plus
    const long long fs = plus ? c : g;
    const double r = (f.baro == nullptr) ? 1.0 : xs ? f.baro->rxp[fs] : f.baro->ryp[fs];
    if (h) h[g] = ghost_head_at(d, f, code, val, h[c], f.bot[c] + 0.5 * f.dz[c], cc, r, plus);
    if (wc) wc[g] = is_head(code) ? f.wcs[c] : wc[c];
  }
}

__global__ void k_ghosts(Dims d, Fields f, double* h, double* wc) {
  ghosts_body(d, f, h, wc, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- closures
// Per-cell directional conductivities K(h, Ksx|Ksy|Ksz) of the predictor pass
// from the step-start head (ghosts included; Predictor.cpp:127-232 evaluates
// them for both flanks of every face).
// The same pass also evaluates C(h^n), the capacity of the storage term
// (Predictor.cpp:445-452), from the same powers.
__device__ __forceinline__ void closure_pred_body(Dims d, Fields f,
                                                         const double* __restrict__ h,
                                                         double* __restrict__ kcx,
                                                         double* __restrict__ kcy,
                                                         double* __restrict__ kcz,
                                                         double* __restrict__ ch, const int bid, const int G) {
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    const double hc = h[c];
    const Soil so = soil_at(f, c);
    const double ksx = f.ksx[c], ksy = f.ksy[c], ksz = f.ksz[c];
    const VgParts v = vg_parts(so, hc);
    const KrParts p = vg_kr_from(v, hc);
    kcx[c] = vg_k_from(p, ksx);
    kcy[c] = vg_k_from(p, ksy);
    kcz[c] = vg_k_from(p, ksz);
    ch[c] = vg_capacity_from(so, v, hc);
  }
}

__global__ void __launch_bounds__(kBlock) k_closure_pred(Dims d, Fields f,
                                                         const double* __restrict__ h,
                                                         double* __restrict__ kcx,
                                                         double* __restrict__ kcy,
                                                         double* __restrict__ kcz,
                                                         double* __restrict__ ch) {
  closure_pred_body(d, f, h, kcx, kcy, kcz, ch, blockIdx.x, gridDim.x);
}

// The predicted head of cell c = (j, i, k): the solution of an active
// interior cell, h^n of an inactive one (fillAndSolve's gw_scatter_head,
// Predictor.cpp:745-754), the head BC's ghost of an edge ghost
// (enforceHeadBc, RichardsSolver.cpp:762), 0 in the four corner columns.
__device__ __forceinline__ double predicted_head(const Dims& d, const Fields& f,
                                                 const double* __restrict__ x,
                                                 const double* __restrict__ hn, long long c, int j,
                                                 int i) {
  const bool jin = j >= 1 && j <= d.ny, iin = i >= 1 && i <= d.nx;
  double hv = 0.0;
  if (jin && iin) {
    const int8_t ac = f.act[c];
    const double xc = x[c], hc = hn[c];
    hv = ac ? xc : hc;
  } else if (jin && (i == 0 || i == d.nx + 1)) {
    const long long ci = (i == 0) ? c + d.sx : c - d.sx;
    const long long cc = col2(d, j, i == 0 ? 1 : d.nx);
    const int8_t ai = f.act[ci];
    const double xi = x[ci], hi0 = hn[ci], zc = f.bot[ci] + 0.5 * f.dz[ci];
    const int code = i == 0 ? f.xmc[cc] : f.xpc[cc];
    const double val = i == 0 ? f.xmv[cc] : f.xpv[cc];
    // the edge face's density ratio: the ghost's slot west, the edge cell's east
    const double r = (f.baro == nullptr) ? 1.0 : f.baro->rxp[i == 0 ? c : ci];
    hv = ghost_head_at(d, f, code, val, ai ? xi : hi0, zc, cc, r, i != 0);
  } else if (iin && (j == 0 || j == d.ny + 1)) {
    const long long ci = (j == 0) ? c + d.sy : c - d.sy;
    const long long cc = col2(d, j == 0 ? 1 : d.ny, i);
    const int8_t ai = f.act[ci];
    const double xi = x[ci], hi0 = hn[ci], zc = f.bot[ci] + 0.5 * f.dz[ci];
    const int code = j == 0 ? f.ymc[cc] : f.ypc[cc];
    const double val = j == 0 ? f.ymv[cc] : f.ypv[cc];
    const double r = (f.baro == nullptr) ? 1.0 : f.baro->ryp[j == 0 ? c : ci];
    hv = ghost_head_at(d, f, code, val, ai ? xi : hi0, zc, cc, r, j != 0);
  }
  return hv;
}

// Corrector pass: scatter the solved heads (fillAndSolve's gw_scatter_head,
// Predictor.cpp:745-754), re-impose the ghost heads (enforceHeadBc after the
// solve, RichardsSolver.cpp:762) and evaluate the per-cell conductivities of
// the predicted head (the corrector's computeFaceConductivity, :768).
__device__ __forceinline__ void closure_corr_body(Dims d, Fields f,
                                                         const double* __restrict__ x,
                                                         const double* __restrict__ hn,
                                                         double* __restrict__ hp,
                                                         double* __restrict__ kcx,
                                                         double* __restrict__ kcy,
                                                         double* __restrict__ kcz, const int bid, const int G) {
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const Soil so = soil_at(f, c);
    const double ksx = f.ksx[c], ksy = f.ksy[c], ksz = f.ksz[c];
    const double hv = predicted_head(d, f, x, hn, c, j, i);
    const KrParts p = vg_kr_parts(so, hv);
    hp[c] = hv;
    kcx[c] = vg_k_from(p, ksx);
    kcy[c] = vg_k_from(p, ksy);
    kcz[c] = vg_k_from(p, ksz);
  }
}

__global__ void __launch_bounds__(kBlock) k_closure_corr(Dims d, Fields f,
                                                         const double* __restrict__ x,
                                                         const double* __restrict__ hn,
                                                         double* __restrict__ hp,
                                                         double* __restrict__ kcx,
                                                         double* __restrict__ kcy,
                                                         double* __restrict__ kcz) {
  closure_corr_body(d, f, x, hn, hp, kcx, kcy, kcz, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- assembly
// Everything the row of one active cell depends on, gathered before any
// arithmetic: the six face conductivities, activity of the upper neighbours
// and of the cells above and below, metrics, step-start state, BC data and
// (density) the ratios.  Shared by k_assemble and the fused predictor.
struct AsmIn {
  double kxp, kxm, kyp, kym, kzm, kzp;
  double dzc, dzu, dzl, wcnc, wcsc;
  double cosxc, cosxw, axc, axw, cosyc, cosys, ayc, ays;
  double chc, hnc, hne, hnw, hnn, hns;
  double vxp, vxm, vyp, vym, vbot, vtop;
  double botc_, bote, botw, botn, bots, sinxc, sinxw, sinyc, sinys;
  // density: r v of the lateral faces (bx*, by*), the z faces' r and v, the
  // lateral faces' r and the cell's r_rho; all 1 without density coupling
  double bxc, bxw, byc, bys, rzpf, rzmf, vzpf, vzmf, rxc, rxw, ryc, rys, rrc;
  // coupled top cell: exchange mode, surface depth, window budget, theta_r
  double dep, avl, wcrc;
  int cm;
  int cxp, cxm, cyp, cym, botc, topc;
  int8_t ae, an, au, al;
};

struct AsmOut {
  double diag, gxp, gyp, gzp, rhs;  // gxp, gyp, gzp: the stored upper legs
};

// The arithmetic of the row of active cell (j, i, k) from gathered values
// (assembleSystemImpl, Predictor.cpp:474-698).
template <bool CPL, bool BARO>
__device__ __forceinline__ AsmOut assemble_math(const Dims& d, const AsmIn& a, double dtg, int j,
                                                int i, int k) {
  const bool east = i == d.nx, west = i == 1, north = j == d.ny, south = j == 1;
  const bool top = (k == 0) || !a.au;
  const double volume = d.az * a.dzc;
  // The reference's legs K dt cos / dx^2 * (A dx) and K dt / (dz dzf) *
  // volume, and its RHS terms dt volume (...) / dz, with the lengths
  // cancelled: K dt cos A (1/dx), K dt az / dzf and dt az (...) (equal up
  // to rounding; three divisions per cell instead of nine).
  double gxp = -a.kxp * dtg * a.cosxc * (a.axc * d.idx);
  double gxm = -a.kxm * dtg * a.cosxw * (a.axw * d.idx);
  double gyp = -a.kyp * dtg * a.cosyc * (a.ayc * d.idy);
  double gym = -a.kym * dtg * a.cosys * (a.ays * d.idy);
  if (BARO) {
    gxp *= a.bxc;
    gxm *= a.bxw;
    gyp *= a.byc;
    gym *= a.bys;
  }
  if (east && is_head(a.cxp)) gxp *= 2.0;
  if (west && is_head(a.cxm)) gxm *= 2.0;
  if (north && is_head(a.cyp)) gyp *= 2.0;
  if (south && is_head(a.cym)) gym *= 2.0;
  const double kdt = dtg * d.az;  // dt * volume / dz
  // the z faces' K with their r v (and the gravity terms' r^2 v)
  const double kzpb = BARO ? a.kzp * a.rzpf * a.vzpf : a.kzp;
  const double kzmb = BARO ? a.kzm * a.rzmf * a.vzmf : a.kzm;
  double dzf = (k == d.nz - 1) ? 0.5 * a.dzc : 0.5 * (a.dzc + a.dzl);
  const double gzp = -kzpb * kdt / dzf;
  dzf = top ? 0.5 * a.dzc : 0.5 * (a.dzc + a.dzu);
  const double gzm = -kzmb * kdt / dzf;

  const double storage =
      BARO ? (a.chc + d.ss * a.wcnc / a.wcsc) * a.rrc : a.chc + d.ss * a.wcnc / a.wcsc;
  double gct = storage * volume - (gxp + gxm + gyp + gym);
  if (east && a.cxp == kFlux) gct += gxp;
  if (west && a.cxm == kFlux) gct += gxm;
  if (north && a.cyp == kFlux) gct += gyp;
  if (south && a.cym == kFlux) gct += gym;
  if (!(k == d.nz - 1 && a.botc != kHead)) gct -= gzp;
  // Coupled top (Predictor.cpp:527-547): the exchange mode decides the
  // Dirichlet leg, the surface depth and window budget feed the RHS.
  const int cm = (CPL && top) ? a.cm : 0;
  const bool dirichlet_top = CPL ? (cm == 1 || (d.pc && cm == 3)) : (a.topc == kHead);
  if (!top || dirichlet_top) gct -= gzm;

  double b = storage * a.hnc * volume;
  b -= kdt * (BARO ? kzpb * a.rzpf : a.kzp);
  b += kdt * (BARO ? kzmb * a.rzmf : a.kzm);
  if (d.terrain) {
    // along-layer gravity; the consistent form carries r^2 v of the face
    const bool rb = BARO && d.pc;
    double sg = (a.bote > a.botc_) ? 1.0 : -1.0;
    b += sg * dtg * a.axc * a.kxp * a.sinxc * (rb ? a.bxc * a.rxc : 1.0);
    sg = (a.botc_ > a.botw) ? -1.0 : 1.0;
    b += sg * dtg * a.axw * a.kxm * a.sinxw * (rb ? a.bxw * a.rxw : 1.0);
    sg = (a.botn > a.botc_) ? 1.0 : -1.0;
    b += sg * dtg * a.ayc * a.kyp * a.sinyc * (rb ? a.byc * a.ryc : 1.0);
    sg = (a.botc_ > a.bots) ? -1.0 : 1.0;
    b += sg * dtg * a.ays * a.kym * a.sinys * (rb ? a.bys * a.rys : 1.0);
  }
  if (east) {
    if (a.cxp == kFlux) b += a.axc * a.vxp * dtg * a.rxc;
    else b -= gxp * a.hne;
  }
  if (west) {
    if (a.cxm == kFlux) b += a.axw * a.vxm * dtg * a.rxw;
    else b -= gxm * a.hnw;
  }
  if (north) {
    if (a.cyp == kFlux) b += a.ayc * a.vyp * dtg * a.ryc;
    else b -= gyp * a.hnn;
  }
  if (south) {
    if (a.cym == kFlux) b += a.ays * a.vym * dtg * a.rys;
    else b -= gym * a.hns;
  }
  if (k == d.nz - 1) {
    if (a.botc == kFlux) b += kdt * a.rzpf * (a.vbot + kzpb);
    else if (a.botc == kHead) b -= gzp * a.vbot;
  }
  if (top && CPL) {  // Predictor.cpp:627-674
    if (cm == 1) {
      b -= gzm * a.dep;
    } else if (d.pc && cm == 3) {
      // the ghost head is 0: the leg sits in the diagonal only
    } else if (cm == 2) {
      const double roomTop = fmax(0.0, (0.9999 * a.wcsc - a.wcnc) * a.dzc);
      const double take = fmin(a.avl, roomTop);
      const double qsup = -take / dtg;
      b += -kdt * a.rzmf * (qsup + kzmb);
    } else {
      double qtop = 0.0;
      if (a.topc == kFlux &&
          ((a.vtop > 0.0 && a.wcnc < a.wcsc) || (a.vtop < 0.0 && a.wcnc > a.wcrc)))
        qtop = a.vtop;
      b += -kdt * a.rzmf * (qtop + kzmb);
    }
  } else if (top) {
    if (a.topc == kHead) b -= gzm * a.vtop;
    else if (a.topc == kFlux) b += -kdt * a.rzmf * (a.vtop + kzmb);
  }
  AsmOut o;
  o.diag = gct;
  o.gxp = (!east && a.ae) ? gxp : 0.0;
  o.gyp = (!north && a.an) ? gyp : 0.0;
  o.gzp = (k + 1 < d.nz && a.al) ? gzp : 0.0;
  o.rhs = b;
  return o;
}

// The per-cell data of the row other than the face conductivities (the
// caller fills kxp .. kzp): metrics, state, BC data, ratios.
template <bool CPL, bool BARO>
__device__ __forceinline__ void assemble_gather(const Dims& d, const Fields& f,
                                                const double* __restrict__ hn,
                                                const double* __restrict__ wcn, double chc,
                                                long long c, int j, int i, int k, AsmIn& a) {
  const long long cw = c - d.sx, ce = c + d.sx, cs = c - d.sy, cn = c + d.sy;
  const long long cu = (k >= 1) ? c - 1 : c, cl = (k + 1 < d.nz) ? c + 1 : c;
  const long long col = col2(d, j, i);
  a.ae = f.act[ce];
  a.an = f.act[cn];
  a.au = (k >= 1) ? f.act[cu] : int8_t(0);
  a.al = (k + 1 < d.nz) ? f.act[cl] : int8_t(0);
  a.dzc = f.dz[c];
  a.dzu = f.dz[cu];
  a.dzl = f.dz[cl];
  a.wcnc = wcn[c];
  a.wcsc = f.wcs[c];
  a.cosxc = f.cosx[c];
  a.cosxw = f.cosx[cw];
  a.axc = f.ax[c];
  a.axw = f.ax[cw];
  a.cosyc = f.cosy[c];
  a.cosys = f.cosy[cs];
  a.ayc = f.ay[c];
  a.ays = f.ay[cs];
  a.chc = chc;
  a.hnc = hn[c];
  a.hne = hn[ce];
  a.hnw = hn[cw];
  a.hnn = hn[cn];
  a.hns = hn[cs];
  a.cxp = f.xpc[col];
  a.cxm = f.xmc[col];
  a.cyp = f.ypc[col];
  a.cym = f.ymc[col];
  a.botc = f.botc[col];
  a.topc = f.topc[col];
  a.vxp = f.xpv[col];
  a.vxm = f.xmv[col];
  a.vyp = f.ypv[col];
  a.vym = f.ymv[col];
  a.vbot = f.botv[col];
  a.vtop = f.topv[col];
  a.botc_ = a.bote = a.botw = a.botn = a.bots = 0.0;
  a.sinxc = a.sinxw = a.sinyc = a.sinys = 0.0;
  if (d.terrain) {
    a.botc_ = f.bot[c];
    a.bote = f.bot[ce];
    a.botw = f.bot[cw];
    a.botn = f.bot[cn];
    a.bots = f.bot[cs];
    a.sinxc = f.sinx[c];
    a.sinxw = f.sinx[cw];
    a.sinyc = f.siny[c];
    a.sinys = f.siny[cs];
  }
  a.bxc = a.bxw = a.byc = a.bys = a.rzpf = a.rzmf = 1.0;
  a.vzpf = a.vzmf = a.rxc = a.rxw = a.ryc = a.rys = a.rrc = 1.0;
  if (BARO) {
    const long long fz = fidx(d, j, i, k);
    const BaroDev& B = *f.baro;
    a.rxc = B.rxp[c];
    a.rxw = B.rxp[cw];
    a.ryc = B.ryp[c];
    a.rys = B.ryp[cs];
    a.bxc = a.rxc * B.vxp[c];
    a.bxw = a.rxw * B.vxp[cw];
    a.byc = a.ryc * B.vyp[c];
    a.bys = a.rys * B.vyp[cs];
    a.rzmf = B.rzp[fz];
    a.rzpf = B.rzp[fz + 1];
    a.vzmf = B.vzp[fz];
    a.vzpf = B.vzp[fz + 1];
    a.rrc = B.rrho[c];
  }
  a.cm = 0;
  a.dep = a.avl = a.wcrc = 0.0;
  const bool top = (k == 0) || !a.au;
  if (CPL && top) {
    a.cm = f.cpl->cmode[col];
    a.dep = f.cpl->dept[col];
    a.avl = f.cpl->avail[col];
    a.wcrc = f.wcr[c];
  }
}

// The 7-point head system of one active cell (assembleSystemImpl,
// Predictor.cpp:400-698, uncoupled, density ratios 1): storage
// C(h^n) + Ss theta^n / theta_s, the six legs with the head-edge doubling,
// the flux-edge and Dirichlet-top diagonal rules, and the RHS with gravity,
// terrain and boundary terms.  The solver stores the diagonal and the three
// upper legs of each row; the lower legs are the neighbours' upper legs
// (the same expression on the same data, so the stored matrix is the
// reference's up to the rounding of its z legs).  Legs toward an inactive
// cell or out of the domain are stored as 0 (PETSc ignores column -1).
template <bool CPL, bool BARO>
__device__ __forceinline__ void assemble_body(
    Dims d, Fields f, const double* __restrict__ kxf, const double* __restrict__ kyf,
    const double* __restrict__ kzff, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ ch, const double* __restrict__ dtgp,
    double* __restrict__ diag, double* __restrict__ gxps, double* __restrict__ gyps,
    double* __restrict__ gzps, double* __restrict__ rhs, double* __restrict__ xw,
    const double* __restrict__ hprev, double ratio, const int bid, const int G) {
  const double dtg = *dtgp;
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    if (j < 1 || j > d.ny || i < 1 || i > d.nx) {
      if (xw) xw[c] = 0.0;
      continue;
    }
    // Gather: the six face conductivities (k_faces), the cell's metrics,
    // heads and BC data.
    const long long fz = fidx(d, j, i, k);
    AsmIn a;
    a.kxp = kxf[c];
    a.kxm = kxf[c - d.sx];
    a.kyp = kyf[c];
    a.kym = kyf[c - d.sy];
    a.kzm = kzff[fz];
    a.kzp = kzff[fz + 1];
    // h^(n-1) with the cell's other loads (behind the activity test it cost a
    // memory round trip of its own: 0.2 ms a 512x512x128 step).
    const double hpv = hprev ? hprev[c] : 0.0;
    const int8_t ac = f.act[c];
    assemble_gather<CPL, BARO>(d, f, hn, wcn, ch[c], c, j, i, k, a);
    // The mixed / FP64 line solves' starting iterate: h^n, or with hprev
    // (h^(n-1)) its linear extrapolation to the step's end,
    // h^n + (dt_n / dt_(n-1)) (h^n - h^(n-1)).
    if (xw) xw[c] = ac ? (hprev ? a.hnc + ratio * (a.hnc - hpv) : a.hnc) : 0.0;
    if (!ac) {
      diag[c] = 1.0;
      gxps[c] = 0.0;
      gyps[c] = 0.0;
      gzps[c] = 0.0;
      rhs[c] = 0.0;
      continue;
    }
    const AsmOut o = assemble_math<CPL, BARO>(d, a, dtg, j, i, k);
    diag[c] = o.diag;
    gxps[c] = o.gxp;
    gyps[c] = o.gyp;
    gzps[c] = o.gzp;
    rhs[c] = o.rhs;
  }
}

template <bool CPL, bool BARO>
__global__ void __launch_bounds__(kBlock, 2) k_assemble(
    Dims d, Fields f, const double* __restrict__ kxf, const double* __restrict__ kyf,
    const double* __restrict__ kzff, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ ch, const double* __restrict__ dtgp,
    double* __restrict__ diag, double* __restrict__ gxps, double* __restrict__ gyps,
    double* __restrict__ gzps, double* __restrict__ rhs, double* __restrict__ xw,
    const double* __restrict__ hprev, double ratio) {
  assemble_body<CPL, BARO>(d, f, kxf, kyf, kzff, hn, wcn, ch, dtgp, diag, gxps, gyps, gzps, rhs,
                           xw, hprev, ratio, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- predictor faces
// Face conductivities of the predictor pass (computeFaceConductivity from
// h^n, Predictor.cpp:105-386): thread c writes its cell's x+ and y+ faces
// (the domain's west and south boundary faces through the ghost cells i = 0,
// j = 0) and the z face above it (plus the bottom face for k = nz-1), into
// the face arrays the corrector's k_flux overwrites later in the step.  A
// separate pass keeps the assembly's loads to six face values.
template <bool CPL>
__device__ __forceinline__ void faces_body(Dims d, Fields f, PassK pk, double* __restrict__ kx,
                                           double* __restrict__ ky, double* __restrict__ kzf,
                                           const int bid, const int G) {
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const bool jin = j >= 1 && j <= d.ny, iin = i >= 1 && i <= d.nx;
    if (jin && i <= d.nx) {
      const long long e = c + d.sx;
      const Flank a{pk.kcx[c], f.ksx[c], pk.wc[c], f.wcs[c], f.act[c]};
      const Flank b{pk.kcx[e], f.ksx[e], pk.wc[e], f.wcs[e], f.act[e]};
      const int code = (i == 0) ? f.xmc[col2(d, j, 1)] : f.xpc[col2(d, j, d.nx)];
      kx[c] = face_lat(d, a, b, i == 0, i == d.nx, code);
    }
    if (iin && j <= d.ny) {
      const long long n = c + d.sy;
      const Flank a{pk.kcy[c], f.ksy[c], pk.wc[c], f.wcs[c], f.act[c]};
      const Flank b{pk.kcy[n], f.ksy[n], pk.wc[n], f.wcs[n], f.act[n]};
      const int code = (j == 0) ? f.ymc[col2(d, 1, i)] : f.ypc[col2(d, d.ny, i)];
      ky[c] = face_lat(d, a, b, j == 0, j == d.ny, code);
    }
    if (jin && iin) {
      const long long col = col2(d, j, i), fz = fidx(d, j, i, k);
      const long long cu = (k >= 1) ? c - 1 : c;
      const ZFlank zu{pk.kcz[cu], f.ksz[cu], f.dz[cu], (k >= 1) ? f.act[cu] : int8_t(0)};
      const ZFlank zc{pk.kcz[c], f.ksz[c], f.dz[c], f.act[c]};
      const int topc = f.topc[col], botc = f.botc[col];
      const double dep = (CPL && k == 0) ? f.cpl->dept[col] : 0.0;
      kzf[fz] = face_z<CPL>(d, zu, zc, k, topc, botc, dep);
      if (k == d.nz - 1) {
        const ZFlank none{0.0, 0.0, 0.0, 0};
        kzf[fz + 1] = face_z<CPL>(d, zc, none, d.nz, topc, botc, 0.0);
      }
    }
  }
}

template <bool CPL>
__global__ void __launch_bounds__(kBlock, 4) k_faces(Dims d, Fields f, PassK pk, double* kx,
                                                     double* ky, double* kzf) {
  faces_body<CPL>(d, f, pk, kx, ky, kzf, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- fused predictor
// The whole predictor of a groundwater-only domain (no coupled top, no
// density coupling; nz <= 32 E) in one pass: the closures of h^n, the face
// conductivities, the row assembly and, for the mixed form, the FP32 casts
// and the column LDL^T factors -- the work of k_closure_pred, k_faces,
// k_assemble and k_line_factor_warp without their intermediate arrays (per
// cell K x3 and C, the three face arrays, the FP64 re-read by the factor).
//
// A block owns a strip of kPredCols interior columns along i plus one halo
// column on each side, one warp per column, lane l holding the E consecutive
// cells k = l E + e of it, and marches j over kPredRows rows.  At row j it
// evaluates the closures of row j + 1 (K along x for the strip and its
// halo, K along y for the strip into shared memory; K along z and C(h^n)
// stay in registers for the next row), then every interior warp takes its
// cell's six faces -- x from the shared row, y from the shared rows j - 1,
// j, j + 1, z by shuffles along its own column -- and the row.  K along x
// lives in three row slots and K along y in four, so a slot is rewritten
// only after every warp has passed the barrier that follows its last
// reader: one __syncthreads per row.  Halo columns cost 2 / kPredCols more
// closures and each segment one more row; the closures are cheap against
// the memory traffic.  The values are those of the separate passes: the
// same closure, face-rule and row functions on the same inputs.
constexpr int kPredWarps = 8;
constexpr int kPredCols = kPredWarps - 2;
constexpr int kPredRows = 16;

// Shared memory of one block: K along x in three row slots for every warp,
// K along y in four row slots and K along z and C(h^n) in two row slots for
// the interior warps.
__host__ __device__ inline size_t pred_smem_bytes(int E) {
  return static_cast<size_t>(3 * kPredWarps + 4 * kPredCols + 4 * kPredCols) * 32 * E *
         sizeof(double);
}

// Closures of row jj for warp w's column i (Predictor.cpp:127-232,
// 445-452): K along x into its slot; with `ky` K along y, with `full` K
// along z and C(h^n) into the interior column iw's slots.
template <int E>
__device__ __forceinline__ void pred_closures(const Dims& d, const Fields& f,
                                              const double* __restrict__ hn, double* psm, int w,
                                              int iw, int i, int jj, bool ky, bool full) {
  constexpr int NZP = 32 * E;
  double* kxs = psm + ((jj % 3) * kPredWarps + w) * NZP;
  double* kys = psm + 3 * kPredWarps * NZP + ((jj & 3) * kPredCols + iw) * NZP;
  double* kzs = psm + (3 * kPredWarps + 4 * kPredCols) * NZP + ((jj & 1) * kPredCols + iw) * NZP;
  double* chs = psm + (3 * kPredWarps + 6 * kPredCols) * NZP + ((jj & 1) * kPredCols + iw) * NZP;
  const int k0 = (threadIdx.x & 31) * E, nz = d.nz;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    if (k < nz) {
      const long long c = cidx(d, jj, i, k);
      const double hc = hn[c];
      const Soil so = soil_at(f, c);
      const double ksx = f.ksx[c], ksy = f.ksy[c], ksz = f.ksz[c];
      const VgParts v = vg_parts(so, hc);
      const KrParts p = vg_kr_from(v, hc);
      kxs[k] = vg_k_from(p, ksx);
      if (ky) kys[k] = vg_k_from(p, ksy);
      if (full) {
        kzs[k] = vg_k_from(p, ksz);
        chs[k] = vg_capacity_from(so, v, hc);
      }
    }
  }
}

// Two blocks per SM up to 128 cells a column; deeper columns need 147 KB of
// shared memory a block, one block per SM, with the registers that frees.
// The kernel body takes the domain's Dims and Fields by value, as the other
// cell kernels' bodies do.
template <int E, bool MIXED>
__device__ __forceinline__ void predict_body(
    Dims d, Fields f, const double* __restrict__ hn, const double* __restrict__ wcn,
    const double* __restrict__ dtgp, double* __restrict__ diag, double* __restrict__ gxps,
    double* __restrict__ gyps, double* __restrict__ gzps, double* __restrict__ rhs,
    double* __restrict__ xw, float* __restrict__ diag32, float* __restrict__ gxp32,
    float* __restrict__ gyp32, float* __restrict__ gzp32, float* __restrict__ dinv32,
    float* __restrict__ l32) {
  extern __shared__ __align__(16) double psm[];
  constexpr int NZP = 32 * E;
  double* skx = psm;                                // [3][kPredWarps][NZP]
  double* sky = skx + 3 * kPredWarps * NZP;         // [4][kPredCols][NZP]
  double* skz = sky + 4 * kPredCols * NZP;          // [2][kPredCols][NZP]
  double* sch = skz + 2 * kPredCols * NZP;          // [2][kPredCols][NZP]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, k0 = lane * E;
  const int i = blockIdx.x * kPredCols + w;  // this warp's column (warp 0: the west halo)
  const bool has_col = i <= d.nx + 1;
  const bool inner = w >= 1 && w <= kPredCols && i <= d.nx;
  const int iw = w - 1;  // index among the interior columns
  const int jb = 1 + blockIdx.y * kPredRows;
  const int je = min(d.ny, jb + kPredRows - 1);
  const int nz = d.nz;
  const double dtg = *dtgp;

  if (has_col) {
    if (inner) pred_closures<E>(d, f, hn, psm, w, iw, i, jb - 1, true, false);  // K along y
    pred_closures<E>(d, f, hn, psm, w, iw, i, jb, inner, inner);
  }
  for (int j = jb; j <= je; ++j) {
    if (has_col) pred_closures<E>(d, f, hn, psm, w, iw, i, j + 1, inner, inner);
    __syncthreads();
    if (inner) {
      const double* kx0 = skx + ((j % 3) * kPredWarps) * NZP;
      const double* kyS = sky + (((j - 1) & 3) * kPredCols + iw) * NZP;
      const double* kyC = sky + ((j & 3) * kPredCols + iw) * NZP;
      const double* kyN = sky + (((j + 1) & 3) * kPredCols + iw) * NZP;
      const double* kzC = skz + ((j & 1) * kPredCols + iw) * NZP;
      const double* chC = sch + ((j & 1) * kPredCols + iw) * NZP;
      const long long col = col2(d, j, i), cb = cidx(d, j, i, 0);
      const int topc = f.topc[col], botc = f.botc[col];
      const int xcode_m = (i == 1) ? f.xmc[col2(d, j, 1)] : f.xpc[col2(d, j, d.nx)];
      const int xcode_p = f.xpc[col2(d, j, d.nx)];
      const int ycode_m = (j == 1) ? f.ymc[col2(d, 1, i)] : f.ypc[col2(d, d.ny, i)];
      const int ycode_p = f.ypc[col2(d, d.ny, i)];
      double av[E], ev[E], xv[E], yv[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = k0 + e;
        av[e] = 1.0;
        ev[e] = xv[e] = yv[e] = 0.0;
        if (k < nz) {
          const long long c = cb + k;
          const long long ce = c + d.sx, cw = c - d.sx, cn = c + d.sy, cs = c - d.sy;
          const long long cu = (k >= 1) ? c - 1 : c, cl = (k + 1 < nz) ? c + 1 : c;
          const double wcc = wcn[c], wsc = f.wcs[c];
          const int8_t ac = f.act[c];
          const Flank fc_x{kx0[w * NZP + k], f.ksx[c], wcc, wsc, ac};
          const Flank fe_x{kx0[(w + 1) * NZP + k], f.ksx[ce], wcn[ce], f.wcs[ce], f.act[ce]};
          const Flank fw_x{kx0[(w - 1) * NZP + k], f.ksx[cw], wcn[cw], f.wcs[cw], f.act[cw]};
          const Flank fc_y{kyC[k], f.ksy[c], wcc, wsc, ac};
          const Flank fn_y{kyN[k], f.ksy[cn], wcn[cn], f.wcs[cn], f.act[cn]};
          const Flank fs_y{kyS[k], f.ksy[cs], wcn[cs], f.wcs[cs], f.act[cs]};
          const ZFlank zu{(k >= 1) ? kzC[k - 1] : kzC[k], f.ksz[cu], f.dz[cu],
                          (k >= 1) ? f.act[cu] : int8_t(0)};
          const ZFlank zc{kzC[k], f.ksz[c], f.dz[c], ac};
          const ZFlank zl{(k + 1 < nz) ? kzC[k + 1] : 0.0, f.ksz[cl], f.dz[cl],
                          (k + 1 < nz) ? f.act[cl] : int8_t(0)};
          AsmIn a;
          a.kxp = face_lat(d, fc_x, fe_x, false, i == d.nx, xcode_p);
          a.kxm = face_lat(d, fw_x, fc_x, i == 1, false, xcode_m);
          a.kyp = face_lat(d, fc_y, fn_y, false, j == d.ny, ycode_p);
          a.kym = face_lat(d, fs_y, fc_y, j == 1, false, ycode_m);
          a.kzm = face_z<false>(d, zu, zc, k, topc, botc, 0.0);
          if (k + 1 < nz) {
            a.kzp = face_z<false>(d, zc, zl, k + 1, topc, botc, 0.0);
          } else {
            const ZFlank none{0.0, 0.0, 0.0, 0};
            a.kzp = face_z<false>(d, zc, none, nz, topc, botc, 0.0);
          }
          assemble_gather<false, false>(d, f, hn, wcn, chC[k], c, j, i, k, a);
          if (MIXED) xw[c] = ac ? a.hnc : 0.0;  // the mixed solve's starting iterate
          double rv = 0.0;
          if (ac) {
            const AsmOut o = assemble_math<false, false>(d, a, dtg, j, i, k);
            av[e] = o.diag;
            xv[e] = o.gxp;
            yv[e] = o.gyp;
            ev[e] = o.gzp;
            rv = o.rhs;
          }
          diag[c] = av[e];
          gxps[c] = xv[e];
          gyps[c] = yv[e];
          gzps[c] = ev[e];
          rhs[c] = rv;
        }
      }
      if (MIXED) factor_column<E>(nz, cb, av, ev, xv, yv, diag32, gxp32, gyp32, gzp32, dinv32, l32);
    }
    // The next row's closures rewrite this warp's K along z and C slots
    // that other lanes of the warp have just read.
    __syncwarp();
  }
}

// ---------------------------------------------------------------- fluxes
// Corrector faces and Darcy fluxes (computeFaceConductivity from the predicted
// head, Predictor.cpp:105-386, and computeFluxesImpl<PC, HARM>,
// Corrector.cpp:135-527, uncoupled).  Thread c owns the x+ and y+ faces of
// its cell and the z face above it (plus the bottom face for k = nz-1).
// Darcy flux of a lateral face from loaded values (computeFluxesImpl's x / y
// branches): a = the face's lower-index flank, b = its upper one; lo_edge /
// hi_edge mark the domain's boundary faces, whose BC code and value apply.
// ih = 1 / dx (1 / dy): the head difference over the spacing (half of it at
// the domain's edges) is a product with the reciprocal, equal up to rounding.
// rf, vf: the face's density and viscosity ratios (1 without density
// coupling): v on the pressure term, r v on the consistent form's gravity.
struct LatFlux {
  double kca, kcb, ksa, ksb, hpa, hpb, wa, wb, wsa, wsb, bota, botb;
  double area, cosv, sinv;
  int8_t acta, actb;
};

__device__ inline double flux_lat(const Dims& d, const Fields& f, const LatFlux& v, double ih,
                                  bool lo_edge, bool hi_edge, int code, double value, long long b,
                                  double rf, double vf) {
  double q;
  if (lo_edge) {
    q = v.area * v.kcb * vf * v.cosv * (v.hpb - v.hpa) * (2.0 * ih);
    if (code == kNoFlux) q = 0.0;
    else if (code == kFlux) q = -value * v.area;
    return q;
  }
  double kf, idelta = ih;
  const double sg = (v.botb > v.bota) ? 1.0 : -1.0;
  if (hi_edge) {
    kf = v.kca;
    idelta = 2.0 * ih;
  } else {
    if (d.pc) {
      kf = d.harm ? face_harm(v.kca, v.ksa, 1.0, v.kcb, v.ksb, 1.0) : 0.5 * (v.kca + v.kcb);
    } else {
      kf = 0.5 * (v.kca + vg_k(soil_at(f, b), v.hpb, v.ksa));
    }
    if (!v.acta || !v.actb) kf = 0.0;
  }
  q = v.area * (kf * vf * v.cosv * (v.hpb - v.hpa) * idelta +
                sg * kf * (d.pc ? rf * vf : 1.0) * v.sinv);
  if (!d.full3d && ((v.acta && v.wa < v.wsa) || (v.actb && v.wb < v.wsb))) q = 0.0;
  if (hi_edge) {
    if (code == kNoFlux) q = 0.0;
    else if (code == kFlux) q = value * v.area;
  }
  return q;
}

// Darcy flux of z-face plane k from loaded values (computeFluxesImpl's z
// branch): u = cell k-1, l = cell k; rz, vz = the face's density and
// viscosity ratios (1 without density coupling), gravity r and the
// conductance's v.
__device__ inline double flux_zv(const Dims& d, const Fields& f, const ZFlank& u, const ZFlank& l,
                                 double hpu, double hpl, int k, int topc, double topv, int botc,
                                 double botv, long long cu, double rz, double vz) {
  const bool below = (k < d.nz) && l.act;
  const bool above = (k >= 1) && u.act;
  if (below && !above) {  // face above a column's top cell
    if (topc == kFlux) return topv * d.az;
    if (topc == kHead) {
      const double delta = 0.5 * l.dz;
      return d.az * l.ks * vz * ((hpl - topv) / delta - rz);
    }
    return 0.0;
  }
  if (k == d.nz && above) {  // bottom boundary face
    const double kf = u.kc;
    if (botc == kFlux) return botv * d.az;
    if (botc == kGravity) return -kf * vz * rz * d.az;
    if (botc == kHead) {
      const double delta = 0.5 * u.dz;
      return d.az * kf * vz * ((botv - hpu) / delta - rz);
    }
    return 0.0;
  }
  if (above && below) {
    double kf;
    if (d.pc) {
      kf = d.harm ? face_harm(u.kc, u.ks, u.dz, l.kc, l.ks, l.dz) : 0.5 * (u.kc + l.kc);
    } else {
      kf = 0.5 * (vg_k(soil_at(f, cu), hpu, l.ks) + l.kc);
    }
    const double delta = 0.5 * (u.dz + l.dz);
    return d.az * kf * vz * ((hpl - hpu) / delta - rz);
  }
  return 0.0;
}

// The coupled exchange face above top cell c of column col
// (Corrector.cpp:388-465, density ratios 1): by exchange mode, the supply-
// limited take of the remaining surface water, the saturated Darcy flux
// capped by the window's budget, the pressurized seepage face (upward only;
// the clamped volume is booked by k_cpl_book), or the dry seepage face with
// the guarded top flux.  Debits the column's budget; hc = predicted head,
// wcc = theta of the cell.
__device__ inline double flux_top_coupled(const Dims& d, const Fields& f, long long col,
                                          long long c, double hc, double wcc, double dtg,
                                          double rz, double vz) {
  const double ks = f.ksz[c], dzc = f.dz[c], dep = f.cpl->dept[col];
  const int m = f.cpl->cmode[col];
  const double delta = 0.5 * dzc;
  double q;
  if (m == 2) {
    const double roomTop = fmax(0.0, (0.9999 * f.wcs[c] - wcc) * dzc);
    const double take = fmin(f.cpl->avail[col], roomTop);
    q = -take * d.az / dtg;
    f.cpl->avail[col] -= take;
  } else if (m == 1) {
    q = d.az * ks * vz * ((hc - dep) / delta - rz);
    if (q < 0.0) {
      const double need = -q * dtg / d.az;
      const double av = f.cpl->avail[col];
      if (need > av) {
        q = -av * d.az / dtg;
        f.cpl->avail[col] = 0.0;
      } else {
        f.cpl->avail[col] = av - need;
      }
    }
  } else if (d.pc && m == 3) {
    q = d.az * ks * vz * ((hc - dep) / delta - rz);
    if (q <= 0.0) q = 0.0;
  } else {
    const Soil so = soil_at(f, c);
    const double kface = 0.5 * (vg_k(so, dep, ks) + vg_k(so, hc, ks));
    q = d.az * kface * vz * ((hc - dep) / delta - rz);
    if (q <= 0.0) q = 0.0;
    if (f.topc[col] == kFlux) {
      const double v = f.topv[col];
      if ((v > 0.0 && wcc > f.wcr[c]) || v < 0.0) q += v * d.az;
    }
  }
  return q;
}

// Thread c owns the x+ and y+ faces of its cell (the domain's west and south
// boundary faces through the ghost cells i = 0, j = 0) and the z face above
// it (plus the bottom face for k = nz-1).  Each face's loads are issued
// before its rules run.
template <bool CPL, bool BARO>
__device__ __forceinline__ void flux_body(Dims d, Fields f, PassK pk,
                                                    const double* __restrict__ hp,
                                                    const double* __restrict__ wcn,
                                                    double* __restrict__ kx,
                                                    double* __restrict__ ky,
                                                    double* __restrict__ kzf,
                                                    double* __restrict__ qx,
                                                    double* __restrict__ qy,
                                                    double* __restrict__ qzf,
                                                    const double* __restrict__ dtgp,
                                                    const int bid, const int G) {
  const double dtg = CPL ? *dtgp : 0.0;
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    const bool jin = j >= 1 && j <= d.ny, iin = i >= 1 && i <= d.nx;
    const bool doX = jin && i <= d.nx, doY = iin && j <= d.ny, doZ = jin && iin;
    LatFlux vx{}, vy{};
    int codex = 0, codey = 0;
    double valx = 0.0, valy = 0.0;
    const long long e = c + d.sx, n = c + d.sy;
    if (doX) {
      const long long ec = col2(d, j, i == 0 ? 1 : d.nx);
      vx = LatFlux{pk.kcx[c], pk.kcx[e], f.ksx[c], f.ksx[e], hp[c], hp[e], wcn[c], wcn[e],
                   f.wcs[c], f.wcs[e], f.bot[c], f.bot[e], f.ax[c], f.cosx[c], f.sinx[c],
                   f.act[c], f.act[e]};
      codex = (i == 0) ? f.xmc[ec] : f.xpc[ec];
      valx = (i == 0) ? f.xmv[ec] : f.xpv[ec];
    }
    if (doY) {
      const long long ec = col2(d, j == 0 ? 1 : d.ny, i);
      vy = LatFlux{pk.kcy[c], pk.kcy[n], f.ksy[c], f.ksy[n], hp[c], hp[n], wcn[c], wcn[n],
                   f.wcs[c], f.wcs[n], f.bot[c], f.bot[n], f.ay[c], f.cosy[c], f.siny[c],
                   f.act[c], f.act[n]};
      codey = (j == 0) ? f.ymc[ec] : f.ypc[ec];
      valy = (j == 0) ? f.ymv[ec] : f.ypv[ec];
    }
    ZFlank zu{}, zc{};
    double hpu = 0.0, hpc = 0.0, topv = 0.0, botv = 0.0;
    int topc = 0, botc = 0;
    const long long cu = (k >= 1) ? c - 1 : c;
    if (doZ) {
      const long long col = col2(d, j, i);
      zu = ZFlank{pk.kcz[cu], f.ksz[cu], f.dz[cu], (k >= 1) ? f.act[cu] : int8_t(0)};
      zc = ZFlank{pk.kcz[c], f.ksz[c], f.dz[c], f.act[c]};
      hpu = hp[cu];
      hpc = hp[c];
      topc = f.topc[col];
      botc = f.botc[col];
      topv = f.topv[col];
      botv = f.botv[col];
    }
    if (doX) {
      const Flank a{vx.kca, vx.ksa, vx.wa, vx.wsa, vx.acta};
      const Flank b{vx.kcb, vx.ksb, vx.wb, vx.wsb, vx.actb};
      kx[c] = face_lat(d, a, b, i == 0, i == d.nx, codex);
      qx[c] = flux_lat(d, f, vx, d.idx, i == 0, i == d.nx, codex, valx, e,
                       BARO ? f.baro->rxp[c] : 1.0, BARO ? f.baro->vxp[c] : 1.0);
    }
    if (doY) {
      const Flank a{vy.kca, vy.ksa, vy.wa, vy.wsa, vy.acta};
      const Flank b{vy.kcb, vy.ksb, vy.wb, vy.wsb, vy.actb};
      ky[c] = face_lat(d, a, b, j == 0, j == d.ny, codey);
      qy[c] = flux_lat(d, f, vy, d.idy, j == 0, j == d.ny, codey, valy, n,
                       BARO ? f.baro->ryp[c] : 1.0, BARO ? f.baro->vyp[c] : 1.0);
    }
    if (doZ) {
      const long long fz = fidx(d, j, i, k), col = col2(d, j, i);
      const double dep = (CPL && k == 0) ? f.cpl->dept[col] : 0.0;
      const double rz = BARO ? f.baro->rzp[fz] : 1.0, vz = BARO ? f.baro->vzp[fz] : 1.0;
      kzf[fz] = face_z<CPL>(d, zu, zc, k, topc, botc, dep);
      if (CPL && zc.act && !(k >= 1 && zu.act))
        qzf[fz] = flux_top_coupled(d, f, col, c, hpc, wcn[c], dtg, rz, vz);
      else
        qzf[fz] = flux_zv(d, f, zu, zc, hpu, hpc, k, topc, topv, botc, botv, cu, rz, vz);
      if (k == d.nz - 1) {
        const ZFlank none{0.0, 0.0, 0.0, 0};
        kzf[fz + 1] = face_z<CPL>(d, zc, none, d.nz, topc, botc, 0.0);
        qzf[fz + 1] = flux_zv(d, f, zc, none, hpc, 0.0, d.nz, topc, topv, botc, botv, c,
                              BARO ? f.baro->rzp[fz + 1] : 1.0,
                              BARO ? f.baro->vzp[fz + 1] : 1.0);
      }
    }
  }
}

template <bool CPL, bool BARO>
__global__ void __launch_bounds__(kBlock, 2) k_flux(Dims d, Fields f, PassK pk,
                                                    const double* __restrict__ hp,
                                                    const double* __restrict__ wcn,
                                                    double* __restrict__ kx,
                                                    double* __restrict__ ky,
                                                    double* __restrict__ kzf,
                                                    double* __restrict__ qx,
                                                    double* __restrict__ qy,
                                                    double* __restrict__ qzf,
                                                    const double* __restrict__ dtgp) {
  flux_body<CPL, BARO>(d, f, pk, hp, wcn, kx, ky, kzf, qx, qy, qzf, dtgp, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- theta update
// theta from the flux divergence with the Ss factor, and the Ss audit term
// (updateWaterContent, Corrector.cpp:629-672).  Cells outside the update keep
// theta^n, so the output buffer is a full copy.
//
// The same pass writes the saturation flag of every cell (theta >= theta_s or
// h > h_ae on the corrected theta and predicted head, ghosts included) that
// the post-allocation classification tests on the six neighbours of a cell,
// and clears the column flags the classification then sets.
// All loads of a cell are issued before its first store and before any
// branch on loaded data, so one memory round trip serves the cell.
// BARO: density coupling (updateWaterContent with its ratios): the storage
// weighs by the cell's r_rho, each face flux by its face's r.
// theta of an active cell from its six face fluxes (density ratios 1);
// adds the cell's Ss storage term to acc.
__device__ __forceinline__ double theta_update(const Dims& d, double dtg, double w0, double hpc,
                                               double hnc, double dzc, double ts, double qxp,
                                               double qxm, double qyp, double qym, double qzt,
                                               double qzb, double& acc) {
  const double volume = d.az * dzc;
  const double dh = hpc - hnc;
  const double coeff = volume * (1.0 + d.ss * dh / ts);
  const double dqx = dtg * (qxp - qxm);
  const double dqy = dtg * (qyp - qym);
  const double dqz = dtg * (qzb - qzt);
  const double upd = (w0 * volume + dqx + dqy + dqz) / coeff;
  acc += upd * volume * d.ss * dh / ts;
  return upd;
}

template <bool BARO>
__device__ __forceinline__ void update_wc_body(
    Dims d, Fields f, const double* __restrict__ hp, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ qx, const double* __restrict__ qy,
    const double* __restrict__ qzf, const double* __restrict__ dtgp, double* __restrict__ wcu,
    uint8_t* __restrict__ satf, int* __restrict__ colflag, double* partial, const int bid,
    const int G) {
  const double dtg = *dtgp;
  double acc = 0.0;
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
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
      if (ac && BARO) {
        const BaroDev& B = *f.baro;
        const double r = B.rrho[c];
        const double volume = d.az * dzc;
        const double dh = hpc - hnc;
        const double coeff = volume * (r + r * d.ss * dh / ts);
        const double dqx = dtg * (qxp * B.rxp[c] - qxm * B.rxp[c - d.sx]);
        const double dqy = dtg * (qyp * B.ryp[c] - qym * B.ryp[c - d.sy]);
        const double dqz = dtg * (qzb * B.rzp[fz + 1] - qzt * B.rzp[fz]);
        upd = (w0 * r * volume + dqx + dqy + dqz) / coeff;
        acc += upd * volume * r * d.ss * dh / ts;
      } else if (ac) {
        upd = theta_update(d, dtg, w0, hpc, hnc, dzc, ts, qxp, qxm, qyp, qym, qzt, qzb, acc);
      }
    }
    wcu[c] = upd;
    satf[c] = (upd >= ts || hpc > aev) ? 1 : 0;
    if (k == 0) colflag[col2(d, j, i)] = 0;  // the walk's column flags start clear
  }
  const double s = block_reduce(acc, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[bid] = s;
}

template <bool BARO>
__global__ void __launch_bounds__(kBlock, 4) k_update_wc(
    Dims d, Fields f, const double* __restrict__ hp, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ qx, const double* __restrict__ qy,
    const double* __restrict__ qzf, const double* __restrict__ dtgp, double* __restrict__ wcu,
    uint8_t* __restrict__ satf, int* __restrict__ colflag, double* partial) {
  update_wc_body<BARO>(d, f, hp, hn, wcn, qx, qy, qzf, dtgp, wcu, satf, colflag, partial,
                       blockIdx.x, gridDim.x);
}

template <int E, bool MIXED>
__global__ void __launch_bounds__(kPredWarps * 32, (E >= 8) ? 1 : 2) k_predict(
    Dims d, Fields f, const double* __restrict__ hn, const double* __restrict__ wcn,
    const double* __restrict__ dtgp, double* __restrict__ diag, double* __restrict__ gxps,
    double* __restrict__ gyps, double* __restrict__ gzps, double* __restrict__ rhs,
    double* __restrict__ xw, float* __restrict__ diag32, float* __restrict__ gxp32,
    float* __restrict__ gyp32, float* __restrict__ gzp32, float* __restrict__ dinv32,
    float* __restrict__ l32) {
  predict_body<E, MIXED>(d, f, hn, wcn, dtgp, diag, gxps, gyps, gzps, rhs, xw, diag32, gxp32,
                         gyp32, gzp32, dinv32, l32);
}

// ---------------------------------------------------------------- fused corrector
// The corrector of a groundwater-only domain (no coupled top, no density
// coupling; nz <= 32 E) in one pass: the head scatter with its ghosts and
// the closures of the predicted head (k_closure_corr), the corrector's face
// conductivities and Darcy fluxes (k_flux) and the theta update with the
// saturation flags and the Ss audit partials (k_update_wc), without the
// per-cell K arrays between them.  The same strip and row march as
// k_predict: at row j the closures of row j + 1 fill the shared rows (the
// predicted head and K along x for the strip and its halo, K along y for
// the strip, K along z per warp), then every interior warp takes its cell's
// six fluxes -- the x- and y- ones evaluated again from the same inputs as
// the neighbour that owns and stores them -- and theta.  Ghost cells'
// outputs (predicted head, theta, flags) are stored by the block that owns
// the strip and rows they border, once.  The grid is the domain's reducing
// grid (D.nblk blocks) walking the (strip, segment) items, so each block
// leaves one Ss partial.
constexpr int kCorrWarps = 8;
constexpr int kCorrCols = kCorrWarps - 2;
constexpr int kCorrRows = 16;

__host__ __device__ inline size_t corr_smem_bytes(int E) {
  // K along x [3][warps], head [4][warps], K along y [4][cols], K along z [2][cols]
  return static_cast<size_t>(3 * kCorrWarps + 4 * kCorrWarps + 4 * kCorrCols + 2 * kCorrCols) *
         32 * E * sizeof(double);
}

// The ghost cells an item of k_correct stores: its columns [.., ..] (own_i
// for this warp's column) and rows [jlo, jhi].
struct CorrOwn {
  bool own_i;
  int jlo, jhi;
};

// Closures of row jj for warp w's column i of k_correct: the predicted head
// and K along x into their slots; with `ky` K along y, with `full` K along z
// (interior column iw).  Ghost cells the item owns get their outputs (head,
// theta^n as theta, the saturation flag, a cleared column flag).
template <int E>
__device__ __forceinline__ void corr_closures(const Dims& d, const Fields& f,
                                              const double* __restrict__ x,
                                              const double* __restrict__ hn,
                                              const double* __restrict__ wcn, double* csm, int w,
                                              int iw, int i, int jj, bool ky, bool full,
                                              CorrOwn own, double* __restrict__ hp,
                                              double* __restrict__ wcu, uint8_t* __restrict__ satf,
                                              int* __restrict__ colflag) {
  constexpr int NZP = 32 * E;
  double* kxs = csm + ((jj % 3) * kCorrWarps + w) * NZP;
  double* hps = csm + 3 * kCorrWarps * NZP + ((jj & 3) * kCorrWarps + w) * NZP;
  double* kys = csm + 7 * kCorrWarps * NZP + ((jj & 3) * kCorrCols + iw) * NZP;
  double* kzs = csm + (7 * kCorrWarps + 4 * kCorrCols) * NZP + ((jj & 1) * kCorrCols + iw) * NZP;
  const bool ghost = jj == 0 || jj == d.ny + 1 || i == 0 || i == d.nx + 1;
  const bool store = ghost && own.own_i && jj >= own.jlo && jj <= own.jhi;
  const int k0 = (threadIdx.x & 31) * E, nz = d.nz;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    if (k < nz) {
      const long long c = cidx(d, jj, i, k);
      const Soil so = soil_at(f, c);
      const double ksx = f.ksx[c], ksy = f.ksy[c], ksz = f.ksz[c];
      const double hv = predicted_head(d, f, x, hn, c, jj, i);
      const KrParts p = vg_kr_parts(so, hv);
      hps[k] = hv;
      kxs[k] = vg_k_from(p, ksx);
      if (ky) kys[k] = vg_k_from(p, ksy);
      if (full) kzs[k] = vg_k_from(p, ksz);
      if (store) {
        const double w0 = wcn[c];
        hp[c] = hv;
        wcu[c] = w0;
        satf[c] = (w0 >= so.ts || hv > so.aev) ? 1 : 0;
        if (k == 0) colflag[col2(d, jj, i)] = 0;
      }
    }
  }
}

template <int E>
__device__ __forceinline__ void correct_body(
    Dims d, Fields f, const double* __restrict__ x, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ dtgp, double* __restrict__ hp,
    double* __restrict__ kx, double* __restrict__ ky, double* __restrict__ kzf,
    double* __restrict__ qx, double* __restrict__ qy, double* __restrict__ qzf,
    double* __restrict__ wcu, uint8_t* __restrict__ satf, int* __restrict__ colflag,
    double* __restrict__ partial) {
  extern __shared__ __align__(16) double csm[];
  constexpr int NZP = 32 * E;
  double* skx = csm;                               // [3][kCorrWarps][NZP]
  double* shp = skx + 3 * kCorrWarps * NZP;        // [4][kCorrWarps][NZP]
  double* sky = shp + 4 * kCorrWarps * NZP;        // [4][kCorrCols][NZP]
  double* skz = sky + 4 * kCorrCols * NZP;         // [2][kCorrCols][NZP]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, k0 = lane * E;
  const int iw = w - 1;
  const int nz = d.nz;
  const double dtg = *dtgp;
  const int nstrips = (d.nx + kCorrCols - 1) / kCorrCols;
  const int nitems = nstrips * ((d.ny + kCorrRows - 1) / kCorrRows);
  double acc = 0.0;

  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int strip = item % nstrips, seg = item / nstrips;
    const int i0 = 1 + strip * kCorrCols;
    const int i = i0 - 1 + w;
    const bool has_col = i <= d.nx + 1;
    const bool inner = w >= 1 && w <= kCorrCols && i <= d.nx;
    const int jb = 1 + seg * kCorrRows;
    const int je = min(d.ny, jb + kCorrRows - 1);
    // the columns and rows whose ghost cells this item stores
    const int ilo = (strip == 0) ? 0 : i0, ihi = min(d.nx, i0 + kCorrCols - 1);
    const int ihi_g = (ihi == d.nx) ? d.nx + 1 : ihi;
    const int jlo_g = (jb == 1) ? 0 : jb, jhi_g = (je == d.ny) ? d.ny + 1 : je;
    const bool own_i = i >= ilo && i <= ihi_g;

    __syncthreads();  // the previous item's last row is read before the slots are rewritten
    const CorrOwn own{own_i, jlo_g, jhi_g};
    if (has_col) {
      corr_closures<E>(d, f, x, hn, wcn, csm, w, iw, i, jb - 1, inner, false, own, hp, wcu, satf,
                       colflag);
      corr_closures<E>(d, f, x, hn, wcn, csm, w, iw, i, jb, inner, inner, own, hp, wcu, satf,
                       colflag);
    }
    for (int j = jb; j <= je; ++j) {
      if (has_col)
        corr_closures<E>(d, f, x, hn, wcn, csm, w, iw, i, j + 1, inner, inner, own, hp, wcu,
                         satf, colflag);
      __syncthreads();
      if (inner) {
        const double* kx0 = skx + ((j % 3) * kCorrWarps) * NZP;
        const double* hp0 = shp + ((j & 3) * kCorrWarps) * NZP;
        const double* hpS = shp + (((j - 1) & 3) * kCorrWarps + w) * NZP;
        const double* hpN = shp + (((j + 1) & 3) * kCorrWarps + w) * NZP;
        const double* kyS = sky + (((j - 1) & 3) * kCorrCols + iw) * NZP;
        const double* kyC = sky + ((j & 3) * kCorrCols + iw) * NZP;
        const double* kyN = sky + (((j + 1) & 3) * kCorrCols + iw) * NZP;
        const double* kzC = skz + ((j & 1) * kCorrCols + iw) * NZP;
        const long long col = col2(d, j, i), cb = cidx(d, j, i, 0), fb = fidx(d, j, i, 0);
        const int topc = f.topc[col], botc = f.botc[col];
        const double topv = f.topv[col], botv = f.botv[col];
        const long long exm = col2(d, j, 1), exp_ = col2(d, j, d.nx);
        const long long eym = col2(d, 1, i), eyp = col2(d, d.ny, i);
        const int cxm = (i == 1) ? f.xmc[exm] : f.xpc[exp_], cxp = f.xpc[exp_];
        const double vxm = (i == 1) ? f.xmv[exm] : f.xpv[exp_], vxp = f.xpv[exp_];
        const int cym = (j == 1) ? f.ymc[eym] : f.ypc[eyp], cyp = f.ypc[eyp];
        const double vym = (j == 1) ? f.ymv[eym] : f.ypv[eyp], vyp = f.ypv[eyp];
        // one cell at a time: a cell's loads fill the registers
#pragma unroll 1
        for (int e = 0; e < E; ++e) {
          const int k = k0 + e;
          if (k >= nz) break;
          const long long c = cb + k, fz = fb + k;
          const long long ce = c + d.sx, cw = c - d.sx, cn = c + d.sy, cs = c - d.sy;
          const long long cu = (k >= 1) ? c - 1 : c, cl = (k + 1 < nz) ? c + 1 : c;
          const double hpc = hp0[w * NZP + k];
          const double w0 = wcn[c], ts = f.wcs[c];
          const int8_t ac = f.act[c];
          const double botc_ = f.bot[c];
          // lateral faces: c with its east / north neighbour (stored here),
          // west / south neighbour with c (evaluated again)
          const LatFlux vxe{kx0[w * NZP + k], kx0[(w + 1) * NZP + k], f.ksx[c], f.ksx[ce], hpc,
                            hp0[(w + 1) * NZP + k], w0, wcn[ce], ts, f.wcs[ce], botc_, f.bot[ce],
                            f.ax[c], f.cosx[c], f.sinx[c], ac, f.act[ce]};
          const LatFlux vxw{kx0[(w - 1) * NZP + k], kx0[w * NZP + k], f.ksx[cw], f.ksx[c],
                            hp0[(w - 1) * NZP + k], hpc, wcn[cw], w0, f.wcs[cw], ts, f.bot[cw],
                            botc_, f.ax[cw], f.cosx[cw], f.sinx[cw], f.act[cw], ac};
          const LatFlux vyn{kyC[k], kyN[k], f.ksy[c], f.ksy[cn], hpc, hpN[k], w0, wcn[cn], ts,
                            f.wcs[cn], botc_, f.bot[cn], f.ay[c], f.cosy[c], f.siny[c], ac,
                            f.act[cn]};
          const LatFlux vys{kyS[k], kyC[k], f.ksy[cs], f.ksy[c], hpS[k], hpc, wcn[cs], w0,
                            f.wcs[cs], ts, f.bot[cs], botc_, f.ay[cs], f.cosy[cs], f.siny[cs],
                            f.act[cs], ac};
          const double qxp = flux_lat(d, f, vxe, d.idx, false, i == d.nx, cxp, vxp, ce, 1.0, 1.0);
          const double qxm = flux_lat(d, f, vxw, d.idx, i == 1, false, cxm, vxm, c, 1.0, 1.0);
          const double qyp = flux_lat(d, f, vyn, d.idy, false, j == d.ny, cyp, vyp, cn, 1.0, 1.0);
          const double qym = flux_lat(d, f, vys, d.idy, j == 1, false, cym, vym, c, 1.0, 1.0);
          kx[c] = face_lat(d, Flank{vxe.kca, vxe.ksa, vxe.wa, vxe.wsa, vxe.acta},
                           Flank{vxe.kcb, vxe.ksb, vxe.wb, vxe.wsb, vxe.actb}, false, i == d.nx,
                           cxp);
          qx[c] = qxp;
          ky[c] = face_lat(d, Flank{vyn.kca, vyn.ksa, vyn.wa, vyn.wsa, vyn.acta},
                           Flank{vyn.kcb, vyn.ksb, vyn.wb, vyn.wsb, vyn.actb}, false, j == d.ny,
                           cyp);
          qy[c] = qyp;
          if (i == 1) {  // the west boundary face, in the ghost column's slot
            kx[cw] = face_lat(d, Flank{vxw.kca, vxw.ksa, vxw.wa, vxw.wsa, vxw.acta},
                              Flank{vxw.kcb, vxw.ksb, vxw.wb, vxw.wsb, vxw.actb}, true, false,
                              cxm);
            qx[cw] = qxm;
          }
          if (j == 1) {  // the south boundary face, in the ghost row's slot
            ky[cs] = face_lat(d, Flank{vys.kca, vys.ksa, vys.wa, vys.wsa, vys.acta},
                              Flank{vys.kcb, vys.ksb, vys.wb, vys.wsb, vys.actb}, true, false,
                              cym);
            qy[cs] = qym;
          }
          // z faces: above c (stored here) and below c (stored by the cell
          // below, or here for the bottom face)
          const double hpu = (k >= 1) ? hp0[w * NZP + k - 1] : hpc;
          const ZFlank zu{(k >= 1) ? kzC[k - 1] : kzC[k], f.ksz[cu], f.dz[cu],
                          (k >= 1) ? f.act[cu] : int8_t(0)};
          const ZFlank zc{kzC[k], f.ksz[c], f.dz[c], ac};
          kzf[fz] = face_z<false>(d, zu, zc, k, topc, botc, 0.0);
          const double qzt = flux_zv(d, f, zu, zc, hpu, hpc, k, topc, topv, botc, botv, cu, 1.0, 1.0);
          qzf[fz] = qzt;
          double qzb;
          if (k + 1 < nz) {
            const ZFlank zl{kzC[k + 1], f.ksz[cl], f.dz[cl], f.act[cl]};
            qzb = flux_zv(d, f, zc, zl, hpc, hp0[w * NZP + k + 1], k + 1, topc, topv, botc, botv,
                          c, 1.0, 1.0);
          } else {
            const ZFlank none{0.0, 0.0, 0.0, 0};
            kzf[fz + 1] = face_z<false>(d, zc, none, nz, topc, botc, 0.0);
            qzb = flux_zv(d, f, zc, none, hpc, 0.0, nz, topc, topv, botc, botv, c, 1.0, 1.0);
            qzf[fz + 1] = qzb;
          }
          double upd = w0;
          if (ac)
            upd = theta_update(d, dtg, w0, hpc, hn[c], zc.dz, ts, qxp, qxm, qyp, qym, qzt, qzb,
                               acc);
          hp[c] = hpc;
          wcu[c] = upd;
          satf[c] = (upd >= ts || hpc > f.aev[c]) ? 1 : 0;
          if (k == 0) colflag[col] = 0;  // the walk's column flags start clear
        }
      }
      // The next row's closures rewrite this warp's K along z slot, which
      // other lanes of the warp have just read.
      __syncwarp();
    }
  }
  const double s = block_reduce(acc, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <int E>
__global__ void __launch_bounds__(kCorrWarps * 32, (E >= 8) ? 1 : 2) k_correct(
    Dims d, Fields f, const double* __restrict__ x, const double* __restrict__ hn,
    const double* __restrict__ wcn, const double* __restrict__ dtgp, double* __restrict__ hp,
    double* __restrict__ kx, double* __restrict__ ky, double* __restrict__ kzf,
    double* __restrict__ qx, double* __restrict__ qy, double* __restrict__ qzf,
    double* __restrict__ wcu, uint8_t* __restrict__ satf, int* __restrict__ colflag,
    double* __restrict__ partial) {
  correct_body<E>(d, f, x, hn, wcn, dtgp, hp, kx, ky, kzf, qx, qy, qzf, wcu, satf, colflag,
                  partial);
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
  double gzb, gzt;  // gravity of the lower / upper z face: 1, or its r_rho (density gradient)
  int8_t axp, axm, ayp, aym, azp, azm;
};

__device__ inline Split gradient_split(const Dims& d, const SplitIn& n, int k) {
  double dh0 = 0.0, dh1 = 0.0, dh2 = 0.0, dh3 = 0.0, dh4 = 0.0, dh5 = 0.0;
  if (d.full3d) {
    const double idx = d.idx, idy = d.idy;
    if (n.axp && n.kxp > 0.0) dh0 = (n.hxp - n.hc) * idx;
    if (n.axm && n.kxm > 0.0) dh1 = (n.hc - n.hxm) * idx;
    if (n.ayp && n.kyp > 0.0) dh2 = (n.hyp - n.hc) * idy;
    if (n.aym && n.kym > 0.0) dh3 = (n.hc - n.hym) * idy;
  }
  if (k + 1 < d.nz && n.azp && n.kzb > 0.0) {
    const double dzp = 0.5 * (n.dzc + n.dzp);
    dh4 = (n.hzp - n.hc) / dzp - n.gzb;
  }
  if (k >= 1 && n.azm && n.kzt > 0.0) {
    const double dzm = 0.5 * (n.dzc + n.dzm);
    dh5 = (n.hc - n.hzm) / dzm - n.gzt;
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
// Classification of interior cell c (Reallocate.cpp:181-391) from the
// pre-sweep snapshot wcR, hR: the restored theta and head, the fresh room
// and the surplus sent up and down; accumulates the audit terms.
struct CellPost {
  double wout, hout, rm, up, dn;
};

template <bool BARO>
__device__ __forceinline__ CellPost classify_cell(
    const Dims& d, const Fields& f, const double* __restrict__ kx, const double* __restrict__ ky,
    const double* __restrict__ kzf, const double* __restrict__ wcR,
    const double* __restrict__ hR, const uint8_t* __restrict__ satf, long long c, int j, int i,
    int k, double& adj, double& drop) {
  const double before = wcR[c];
  double wout = before, hout = hR[c], rm = 0.0, up = 0.0, dn = 0.0;
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
  n.gzb = 1.0;
  n.gzt = 1.0;
  if (BARO && f.baro->dgrad) {  // densityReallocationGradient (Reallocate.cpp:223-233)
    n.gzb = f.baro->rzp[fz + 1];
    n.gzt = f.baro->rzp[fz];
  }
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
        // A cell exactly at theta_s (the whole saturated zone) has no excess:
        // its split would send 0 each way, so it is not computed.
        const double excess = (before - so.ts) * volume;
        if (excess > 0.0) {
          const Split sp = gradient_split(d, n, k);
          up = excess * sp.up;
          dn = excess * sp.down;
          adj -= excess - up - dn;
          drop += excess - up - dn;
        }
        wout = so.ts;
      }
    } else {
      rm = (so.ts - before) * volume;
      const bool top = (k == 0) || !n.azm;
      const bool adjsat = (n.azp && szp) || (n.kxp != 0.0 && sxp) ||
                          (n.kxm != 0.0 && sxm) || (n.kyp != 0.0 && syp) ||
                          (n.kym != 0.0 && sym) ||
                          (top ? (f.cpl ? f.cpl->dept[col] > 0.0  // coupled: a wet surface
                                        : (topc == kHead && topv >= 0.0))
                               : (szm != 0));
      if (!adjsat) {
        if (before < 0.9999 * so.ts) hout = vg_head_fast(so, before);
      } else if (!d.off) {
        const double after = vg_theta_fast(so, hout);
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
  }
  return CellPost{wout, hout, rm, up, dn};
}

template <bool BARO>
__device__ __forceinline__ void classify_body(
    Dims d, Fields f, const double* __restrict__ kx, const double* __restrict__ ky,
    const double* __restrict__ kzf, const double* __restrict__ wcR,
    const double* __restrict__ hR, const uint8_t* __restrict__ satf, double* __restrict__ wc_out,
    double* __restrict__ h_out, double* __restrict__ room, double* __restrict__ sup,
    double* __restrict__ sdn, int* colflag, double* part_adj, double* part_drop, const int bid,
    const int G) {
  double adj = 0.0, drop = 0.0;
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    CellPost r{wcR[c], hR[c], 0.0, 0.0, 0.0};
    if (j >= 1 && j <= d.ny && i >= 1 && i <= d.nx) {
      r = classify_cell<BARO>(d, f, kx, ky, kzf, wcR, hR, satf, c, j, i, k, adj, drop);
      if (r.up > 0.0 || r.dn > 0.0) colflag[col2(d, j, i)] = 1;
    }
    wc_out[c] = r.wout;
    h_out[c] = r.hout;
    room[c] = r.rm;
    sup[c] = r.up;
    sdn[c] = r.dn;
  }
  const double s1 = block_reduce(adj, SumOp(), 0.0);
  if (threadIdx.x == 0) part_adj[bid] = s1;
  const double s2 = block_reduce(drop, SumOp(), 0.0);
  if (threadIdx.x == 0) part_drop[bid] = s2;
}

template <bool BARO>
__global__ void __launch_bounds__(kBlock, 3) k_classify(
    Dims d, Fields f, const double* __restrict__ kx, const double* __restrict__ ky,
    const double* __restrict__ kzf, const double* __restrict__ wcR,
    const double* __restrict__ hR, const uint8_t* __restrict__ satf, double* __restrict__ wc_out,
    double* __restrict__ h_out, double* __restrict__ room, double* __restrict__ sup,
    double* __restrict__ sdn, int* colflag, double* part_adj, double* part_drop) {
  classify_body<BARO>(d, f, kx, ky, kzf, wcR, hR, satf, wc_out, h_out, room, sup, sdn, colflag,
                      part_adj, part_drop, blockIdx.x, gridDim.x);
}

// A coupled column's surface during its send walks: the vent deposits
// (Reallocate.cpp:463-490) land in these copies, written back after the
// column, and in the vent books.
struct VentState {
  double eta, dept, avail, gain;
  double vent, thin;
  double min_depth;
  int vent_all;
  double wv;  // this column's vented volume (transport window)
};

// What the upward walk could not place, dv > 0, leaves through the top of
// column face `ll` of a coupled column: onto the surface when it is wet, the
// amount exceeds min_depth or every vent deposits; else it is lost.
__device__ inline bool vent_top(const Dims& d, double dv, double idtg, double& qface,
                                VentState& v, double& lost) {
  const double dd = dv / d.az;
  if (v.vent_all || v.dept > 0.0 || dd > v.min_depth) {
    if (!(v.dept > 0.0 || dd > v.min_depth)) v.thin += dv;
    v.eta += dd;
    v.dept += dd;
    v.avail += dd;
    v.gain += dd;
    qface += __dmul_rn(dv, idtg);
    v.vent += dv;
    v.wv += dv;
    return true;
  }
  lost -= dv;
  return false;
}

// The transport window's record of one transfer of `rate` from cell `from`
// to cell `to` of a column (to = the cell above the column's top for a
// release through it), mirrored by the legacy rule on face `face` with
// `sign` (Reallocate.cpp:418-446): the column's path corrections pc (faces
// 0..nz) move the rate from the mirrored face onto every face crossed.
__device__ inline void path_record(double* pc, int from, int to, double rate, int face,
                                   double sign) {
  pc[face] -= sign * rate;
  if (to < from) {
    for (int f = to + 1; f <= from; ++f) pc[f] += rate;
  } else {
    for (int f = from + 1; f <= to; ++f) pc[f] -= rate;
  }
}

__device__ inline void vent_load(const Fields& f, long long col, VentState& v) {
  v.eta = f.cpl->eta[col];
  v.dept = f.cpl->dept[col];
  v.avail = f.cpl->avail[col];
  v.gain = f.cpl->gain[col];
  v.min_depth = f.cpl->min_depth;
  v.vent_all = f.cpl->vent_all;
  v.wv = 0.0;
}

__device__ inline void vent_store(const Fields& f, long long col, const VentState& v) {
  f.cpl->eta[col] = v.eta;
  f.cpl->dept[col] = v.dept;
  f.cpl->avail[col] = v.avail;
  f.cpl->gain[col] = v.gain;
}

// Block sums of the walk's books: the overflow into slot kPLost and, in
// coupled runs, the vents into kPVent / kPThin.
template <bool CPL>
__device__ inline void walk_books(const Dims& d, double lost, const VentState& v, double* partial,
                                  int nblk, int bid) {
  const double s = block_reduce(lost, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPLost * nblk + bid] = s;
  if (CPL) {
    const double sv = block_reduce(v.vent, SumOp(), 0.0);
    if (threadIdx.x == 0) partial[kPVent * nblk + bid] = sv;
    const double st = block_reduce(v.thin, SumOp(), 0.0);
    if (threadIdx.x == 0) partial[kPThin * nblk + bid] = st;
  }
}

// Phase 2: the vertical send walks, one thread per flagged column, k
// ascending (Reallocate.cpp:410-540, no transport window).
template <bool CPL>
__device__ __forceinline__ void walk_thread_body(Dims d, Fields f, double* wc, double* room, const double* __restrict__ sup,
                       const double* __restrict__ sdn, double* qzf, const int* __restrict__ colflag,
                       const double* __restrict__ dtgp, double* partial, int nblk,
                       double* pcorr, double* wvent, const int bid, const int G) {
  const double dtg = *dtgp;
  double lost = 0.0;
  VentState v{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0.0};
  const long long ncolint = static_cast<long long>(d.nx) * d.ny;
  for (long long t = bid * static_cast<long long>(blockDim.x) + threadIdx.x; t < ncolint;
       t += static_cast<long long>(G) * blockDim.x) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    if (!colflag[col]) continue;
    const long long base = cidx(d, j, i, 0), fb = fidx(d, j, i, 0);
    const bool topHead = f.topc[col] == kHead;
    if (CPL) vent_load(f, col, v);
    double* pc = pcorr ? pcorr + fb : nullptr;  // transport window: this column's path records
    if (pc)
      for (int q = 0; q <= d.nz; ++q) pc[q] = 0.0;
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
            if (pc) path_record(pc, k, ll, take / dtg, ll + 1, 1.0);
            dv -= take;
          }
        }
        if (dv > 0.0) {
          if (CPL) {
            if (vent_top(d, dv, 1.0 / dtg, qzf[fb + ll], v, lost) && pc)
              path_record(pc, k, ll - 1, dv / dtg, ll, 1.0);
          } else if (topHead) {
            qzf[fb + ll] += dv / dtg;
            if (pc) path_record(pc, k, ll - 1, dv / dtg, ll, 1.0);
          } else {
            while (ll + 1 < d.nz && dv > 0.0) {
              ++ll;
              const long long c = base + ll;
              if (room[c] > 0.0) {
                const double take = (room[c] > dv) ? dv : room[c];
                wc[c] += take / (d.az * f.dz[c]);
                room[c] -= take;
                qzf[fb + ll] -= take / dtg;
                if (pc) path_record(pc, k, ll, take / dtg, ll, -1.0);
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
            if (pc) path_record(pc, k, ll, take / dtg, ll, -1.0);
            dv -= take;
          }
        }
        lost -= dv;
      }
    }
    if (CPL) {
      vent_store(f, col, v);
      if (wvent) wvent[col] += v.wv;
    }
  }
  walk_books<CPL>(d, lost, v, partial, nblk, bid);
}

template <bool CPL>
__global__ void k_walk_thread(Dims d, Fields f, double* wc, double* room, const double* __restrict__ sup,
                       const double* __restrict__ sdn, double* qzf, const int* __restrict__ colflag,
                       const double* __restrict__ dtgp, double* partial, int nblk,
                       double* pcorr, double* wvent) {
  walk_thread_body<CPL>(d, f, wc, room, sup, sdn, qzf, colflag, dtgp, partial, nblk, pcorr, wvent,
                        blockIdx.x, gridDim.x);
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
// The divisions by the cell volume and by dtg are multiplications by their
// reciprocals (ivs staged per column, idtg once per kernel): a walk runs on
// one lane, and FP64 divisions were most of its issue slots.
__device__ inline void walk_take(double& dv, int m, double* rs, double* ws, const double* ivs,
                                 double* qs, unsigned* rbits, int face, bool plus, double idtg,
                                 double* pc, int from) {
  const double take = (rs[m] > dv) ? dv : rs[m];
  ws[m] = __fma_rn(take, ivs[m], ws[m]);
  rs[m] -= take;
  // The rate is rounded on its own (no fused multiply-add), so every kernel
  // that inlines this walk -- with or without the path record that reuses
  // the rate -- adds the same value.
  const double rate = __dmul_rn(take, idtg);
  if (plus) {
    qs[face] += rate;
  } else {
    qs[face] -= rate;
  }
  if (pc) path_record(pc, from, m, rate, face, plus ? 1.0 : -1.0);
  dv -= take;
  if (!(rs[m] > 0.0)) rbits[m >> 5] &= ~(1u << (m & 31));
}

// Lane 0's send walks of surplus cell kk (sent up upv, sent down dnv) on a
// staged column (Reallocate.cpp:410-540): upward through the cells with room
// up to the first inactive cell above or the surface, then out through a
// head top or back down; downward to the bottom; what finds no room is lost.
template <bool CPL>
__device__ inline void walk_cell(const Dims& d, int kk, double upv, double dnv, int nz, bool topHead,
                                 double* rs, double* ws, const double* ivs, double* qs,
                                 unsigned* rbits, const unsigned* ibits, double idtg, double& lost,
                                 VentState& v, double* pc) {
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
      walk_take(dv, m, rs, ws, ivs, qs, rbits, m + 1, true, idtg, pc, kk);
      ll = m;
    }
    if (dv > 0.0) {
      if (CPL) {
        if (vent_top(d, dv, idtg, qs[ll], v, lost) && pc)
          path_record(pc, kk, ll - 1, __dmul_rn(dv, idtg), ll, 1.0);
      } else if (topHead) {
        const double rate = __dmul_rn(dv, idtg);
        qs[ll] += rate;
        if (pc) path_record(pc, kk, ll - 1, rate, ll, 1.0);
      } else {
        while (dv > 0.0) {
          const int m = bits_lowest(rbits, ll + 1, nz - 1);
          if (m < 0) break;
          walk_take(dv, m, rs, ws, ivs, qs, rbits, m, false, idtg, pc, kk);
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
      walk_take(dv, m, rs, ws, ivs, qs, rbits, m, false, idtg, pc, kk);
      ll = m;
    }
    lost -= dv;
  }
}

// Stages flagged column `base` for the walk: room, theta and the face fluxes
// into shared memory and the room bits; with `all` also the reciprocal cell
// volumes and the inactive bits (a restage keeps those).
__device__ inline void walk_stage(const Dims& d, const Fields& f, long long base, long long fb,
                                  int nz, int lane, const double* __restrict__ room,
                                  const double* wc, const double* qzf, double* rs, double* ws,
                                  double* ivs, double* qs, unsigned* rbits, unsigned* ibits,
                                  bool all) {
  for (int k0 = 0; k0 < nz; k0 += 32) {
    const int k = k0 + lane;
    double r = 0.0;
    bool inact = false;
    if (k < nz) {
      r = room[base + k];
      rs[k] = r;
      ws[k] = wc[base + k];
      if (all) ivs[k] = 1.0 / (d.az * f.dz[base + k]);
      inact = !f.act[base + k];
    }
    const unsigned rb = __ballot_sync(0xffffffffu, r > 0.0);
    const unsigned ib = __ballot_sync(0xffffffffu, inact);
    if (lane == 0) {
      rbits[k0 >> 5] = rb;
      if (all) ibits[k0 >> 5] = ib;
    }
  }
  for (int k = lane; k <= nz; k += 32) qs[k] = qzf[fb + k];
  __syncwarp();
}

// The walk of a staged column in the common case, where no deposit changes
// where a later one goes: every surplus cell's upward send finds a cell with
// room between it and the first inactive cell above it, and every deposit
// leaves its cell some room (rs > dv before the deposit), so the room bits
// never change.  Each lane resolves the targets of its own cells from the
// bits (the nearest cell with room above within the active run; the nearest
// below, or none: lost), and lane 0 applies the deposits in the general
// walk's order -- cells ascending, each one's upward send before its
// downward one -- with walk_take's arithmetic, so the result is the general
// walk's bit for bit.  Returns 0 when the column is walked; 2 when a send
// fell outside the case (no target above, or a deposit that would use up
// its cell's room): the shared column is then partly updated and `lost` is
// restored, the caller restages the column and runs the general walk.
__device__ inline int walk_fast(const Fields& f, long long base, int nz, int lane, double* rs,
                                double* ws, const double* ivs, double* qs, const unsigned* rbits,
                                const unsigned* ibits, const double* __restrict__ sup,
                                const double* __restrict__ sdn, double idtg, double& lost) {
  const double lost0 = lost;
  for (int k0 = 0; k0 < nz; k0 += 32) {
    const int k = k0 + lane;
    double su = 0.0, sd = 0.0;
    int mu = -1, md = -1;
    bool any = false, bad = false;
    if (k < nz && f.act[base + k]) {
      su = sup[base + k];
      sd = sdn[base + k];
      any = su > 0.0 || sd > 0.0;
      if (su > 0.0) {
        mu = bits_highest(rbits, bits_highest(ibits, 0, k - 1) + 1, k - 1);
        bad = mu < 0;
      }
      if (sd > 0.0) md = bits_lowest(rbits, k + 1, nz - 1);
    }
    if (__any_sync(0xffffffffu, bad)) {
      lost = lost0;
      __syncwarp();
      return 2;
    }
    unsigned mask = __ballot_sync(0xffffffffu, any);
    int fail = 0;
    while (mask) {
      const int b = __ffs(mask) - 1;
      mask &= mask - 1;
      const double upv = __shfl_sync(0xffffffffu, su, b);
      const double dnv = __shfl_sync(0xffffffffu, sd, b);
      const int tu = __shfl_sync(0xffffffffu, mu, b);
      const int td = __shfl_sync(0xffffffffu, md, b);
      if (lane == 0 && !fail) {
        if (upv > 0.0) {
          if (rs[tu] > upv) {
            ws[tu] = __fma_rn(upv, ivs[tu], ws[tu]);
            rs[tu] -= upv;
            qs[tu + 1] += __dmul_rn(upv, idtg);
          } else {
            fail = 1;
          }
        }
        if (!fail && dnv > 0.0) {
          if (td < 0) {
            lost -= dnv;
          } else if (rs[td] > dnv) {
            ws[td] = __fma_rn(dnv, ivs[td], ws[td]);
            rs[td] -= dnv;
            qs[td] -= __dmul_rn(dnv, idtg);
          } else {
            fail = 1;
          }
        }
      }
    }
    if (__shfl_sync(0xffffffffu, fail, 0)) {
      lost = lost0;
      __syncwarp();
      return 2;
    }
    __syncwarp();
  }
  return 0;
}

template <bool CPL>
__device__ __forceinline__ void walk_body(Dims d, Fields f, double* wc,
                                                 const double* __restrict__ room,
                                                 const double* __restrict__ sup,
                                                 const double* __restrict__ sdn, double* qzf,
                                                 const int* __restrict__ colflag,
                                                 const double* __restrict__ dtgp,
                                                 double* partial, int nblk, double* pcorr,
                                                 double* wvent, const int bid, const int G) {
  extern __shared__ __align__(16) unsigned char walk_smem[];
  const double idtg = 1.0 / *dtgp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nz = d.nz, nw = walk_words(nz);
  double* rs = reinterpret_cast<double*>(walk_smem + warp * walk_warp_bytes(nz));
  double* ws = rs + nz;
  double* ivs = ws + nz;  // 1 / cell volume
  double* qs = ivs + nz;  // nz + 1 faces
  unsigned* rbits = reinterpret_cast<unsigned*>(qs + nz + 1);
  unsigned* ibits = rbits + nw;  // inactive cells
  double lost = 0.0;
  VentState v{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0.0};
  const long long ncolint = static_cast<long long>(d.nx) * d.ny;
  const long long nwarps = static_cast<long long>(G) * kWalkWarps;
  for (long long t = bid * static_cast<long long>(kWalkWarps) + warp; t < ncolint;
       t += nwarps) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    if (!colflag[col]) continue;
    const long long base = cidx(d, j, i, 0), fb = fidx(d, j, i, 0);
    const bool topHead = f.topc[col] == kHead;
    if (CPL && lane == 0) vent_load(f, col, v);
    double* pc = pcorr ? pcorr + fb : nullptr;  // transport window: this column's path records
    if (pc)
      for (int q = lane; q <= nz; q += 32) pc[q] = 0.0;
    walk_stage(d, f, base, fb, nz, lane, room, wc, qzf, rs, ws, ivs, qs, rbits, ibits, true);
    int how = 1;
    if (!CPL && !pc)
      how = walk_fast(f, base, nz, lane, rs, ws, ivs, qs, rbits, ibits, sup, sdn, idtg, lost);
    if (how == 0) {
      for (int k = lane; k < nz; k += 32) wc[base + k] = ws[k];
      for (int k = lane; k <= nz; k += 32) qzf[fb + k] = qs[k];
      __syncwarp();
      continue;
    }
    if (how == 2) walk_stage(d, f, base, fb, nz, lane, room, wc, qzf, rs, ws, ivs, qs, rbits, ibits,
                             false);
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
        if (lane == 0)
          walk_cell<CPL>(d, k0 + b, upv, dnv, nz, topHead, rs, ws, ivs, qs, rbits, ibits, idtg, lost,
                         v, pc);
        __syncwarp();
      }
    }
    for (int k = lane; k < nz; k += 32) wc[base + k] = ws[k];
    for (int k = lane; k <= nz; k += 32) qzf[fb + k] = qs[k];
    if (CPL && lane == 0) {
      vent_store(f, col, v);
      if (wvent) wvent[col] += v.wv;
    }
    __syncwarp();
  }
  walk_books<CPL>(d, lost, v, partial, nblk, bid);
}

// Four blocks per SM (three for the coupled form's vent state): without a
// minimum ptxas settled on 64 / 80 registers with spills.
template <bool CPL>
__global__ void __launch_bounds__(kBlock, CPL ? 3 : 4) k_walk(Dims d, Fields f, double* wc,
                                                 const double* __restrict__ room,
                                                 const double* __restrict__ sup,
                                                 const double* __restrict__ sdn, double* qzf,
                                                 const int* __restrict__ colflag,
                                                 const double* __restrict__ dtgp,
                                                 double* partial, int nblk, double* pcorr,
                                                 double* wvent) {
  walk_body<CPL>(d, f, wc, room, sup, sdn, qzf, colflag, dtgp, partial, nblk, pcorr, wvent,
                 blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------- coupled top
// First active cell of column (j, i), or -1.
__device__ inline int first_active(const Dims& d, const Fields& f, int j, int i) {
  const long long base = cidx(d, j, i, 0);
  for (int k = 0; k < d.nz; ++k)
    if (f.act[base + k]) return k;
  return -1;
}

// classifyCoupledTopImpl<PC> (Corrector.cpp:55-115), one thread per column:
// 1 = a wet surface whose saturated demand the window's water funds, 2 = a
// wet surface it cannot fund, 3 = (consistent form) a dry surface over a
// top cell pressurized past dz/2, 0 = dry.
__global__ void k_cpl_mode(Dims d, Fields f, const double* __restrict__ h,
                           const double* __restrict__ dtgp) {
  const double dtg = *dtgp;
  const long long ncol = static_cast<long long>(d.nx) * d.ny;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < ncol;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    const int kt = first_active(d, f, j, i);
    const double dep = f.cpl->dept[col];
    int8_t m = 0;
    if (kt < 0 || dep <= 0.0) {
      if (d.pc && kt >= 0) {
        // pressurized past r dz / 2 (r = the top face's density ratio)
        const long long c = cidx(d, j, i, kt);
        const double r = (f.baro == nullptr) ? 1.0 : f.baro->rzp[fidx(d, j, i, kt)];
        if (h[c] > r * 0.5 * f.dz[c]) m = 3;
      }
    } else {
      const long long c = cidx(d, j, i, kt);
      const double ks = f.ksz[c];
      const double qest = 2.0 * ks * (h[c] - dep) / f.dz[c] - ks;
      m = (qest < 0.0 && -qest * dtg > f.cpl->avail[col]) ? 2 : 1;
    }
    f.cpl->cmode[col] = m;
  }
}

// applyCoupledTopBookkeeping (Corrector.cpp:539-627, no ET), one thread per
// column after the corrector's fluxes: the exchanged volume, the bounce-back
// of infiltration a full top cell cannot take under a dry surface, the
// seepage accumulator and the evaporation correction; also books the
// consistent form's mode-3 upward-only clamp from the flux pass's inputs
// (Corrector.cpp:431-445).  wcn = theta of the step start (the corrector's
// theta until the update), hp = predicted head.  nblk blocks, one partial
// per block in each book.
__global__ void k_cpl_book(Dims d, Fields f, const double* __restrict__ hp,
                           const double* __restrict__ wcn, const double* __restrict__ qzf,
                           const double* __restrict__ dtgp, double* partial, int nblk) {
  const double dtg = *dtgp;
  double se = 0.0, sb = 0.0, sv = 0.0, sc = 0.0;
  const long long ncol = static_cast<long long>(d.nx) * d.ny;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < ncol;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    const int kt = first_active(d, f, j, i);
    if (kt < 0) continue;
    const long long c = cidx(d, j, i, kt);
    const double q = qzf[fidx(d, j, i, kt)];
    double dep = f.cpl->dept[col];
    se += q * dtg;
    if (d.pc && f.cpl->cmode[col] == 3) {
      const long long fz = fidx(d, j, i, kt);
      const double rz = (f.baro == nullptr) ? 1.0 : f.baro->rzp[fz];
      const double vz = (f.baro == nullptr) ? 1.0 : f.baro->vzp[fz];
      const double qr = d.az * f.ksz[c] * vz * ((hp[c] - dep) / (0.5 * f.dz[c]) - rz);
      if (qr <= 0.0) sc += -qr * dtg;
    }
    if (q < 0.0 && dep <= f.cpl->min_depth) {
      const double volume = d.az * f.dz[c];
      if ((f.wcs[c] - wcn[c]) < -q * dtg / volume) {
        const double dd = -q * dtg / d.az;
        f.cpl->eta[col] += dd;
        dep += dd;
        f.cpl->dept[col] = dep;
        f.cpl->avail[col] += dd;
        f.cpl->gain[col] += dd;
        if (f.cpl->book_bounce) f.cpl->bounce[col] += dd;
        sb += dd * d.az;
      }
    }
    double acc = f.cpl->seep[col] + q * dtg / d.az;
    const double tv = f.topv[col];
    if (f.topc[col] == kFlux && tv > 0.0 && wcn[c] > f.wcr[c] && dep <= f.cpl->min_depth) {
      acc -= tv * dtg;
      sv += tv * dtg * d.az;
    }
    f.cpl->seep[col] = acc;
  }
  const double r0 = block_reduce(se, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPExch * nblk + blockIdx.x] = r0;
  const double r1 = block_reduce(sb, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPBounce * nblk + blockIdx.x] = r1;
  const double r2 = block_reduce(sv, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPEvap * nblk + blockIdx.x] = r2;
  const double r3 = block_reduce(sc, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPClamp * nblk + blockIdx.x] = r3;
}

// Coupler::beginWindow (Exchange.cpp:21-52): the window's infiltration
// budget from the refreshed depth, the deposit tally cleared.
__global__ void k_cpl_begin_window(Dims d, Fields f) {
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < d.ncol;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(t / d.nx2), i = static_cast<int>(t % d.nx2);
    if (j >= 1 && j <= d.ny && i >= 1 && i <= d.nx) {
      f.cpl->avail[t] = f.cpl->dept[t];
      f.cpl->gain[t] = 0.0;
    }
    if (f.cpl->book_bounce) f.cpl->bounce[t] = 0.0;
  }
}

// Coupler::applySeepage (Exchange.cpp:54-107) and reduceAudit (:109-127):
// infiltration applied in full down to the bed, seepage applied onto a wet
// surface or once it exceeds min_depth, else held; qss = the window's rate.
// Books per block: applied, clamp remainder, gain and held seepage.
__global__ void k_cpl_seepage(Dims d, Fields f, double* __restrict__ qss,
                              const double* __restrict__ bottom, double dt, double* partial,
                              int nblk) {
  double sa = 0.0, sd = 0.0, sg = 0.0, sh = 0.0;
  const long long ncol = static_cast<long long>(d.nx) * d.ny;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < ncol;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(t / d.nx) + 1, i = static_cast<int>(t % d.nx) + 1;
    const long long col = col2(d, j, i);
    const double a = f.cpl->seep[col];
    double gain = f.cpl->gain[col], held = a;
    qss[col] = a / dt;
    if (a < 0.0) {
      const double before = f.cpl->eta[col];
      double e = before + a;
      if (e < bottom[col]) e = bottom[col];
      f.cpl->eta[col] = e;
      const double change = e - before;
      gain += change;
      sa += change;
      sd += change - a;
      held = 0.0;
    } else if (f.cpl->dept[col] > f.cpl->min_depth || a > f.cpl->min_depth) {
      f.cpl->eta[col] += a;
      gain += a;
      sa += a;
      held = 0.0;
    }
    f.cpl->gain[col] = gain;
    f.cpl->seep[col] = held;
    sg += gain;
    sh += held;
  }
  const double r0 = block_reduce(sa, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[0 * nblk + blockIdx.x] = r0;
  const double r1 = block_reduce(sd, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[1 * nblk + blockIdx.x] = r1;
  const double r2 = block_reduce(sg, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[2 * nblk + blockIdx.x] = r2;
  const double r3 = block_reduce(sh, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[3 * nblk + blockIdx.x] = r3;
}

// ---------------------------------------------------------------- clamp, audit, controller
// finalizeWaterContent (Corrector.cpp:758-792), accumulateBoundaryFlux
// (RichardsSolver.cpp:961-1006), the adaptTimeStep inputs (AdaptiveStep.cpp:
// 58-98) and the owned volume (RichardsSolver.cpp:892-912), in one sweep.
// Clamp, clamp loss, boundary inflow and controller inputs of active interior
// cell c (finalizeWaterContent, Corrector.cpp:758-792; accumulateBoundaryFlux,
// RichardsSolver.cpp:961-1006; adaptTimeStep's dq and Courant terms,
// AdaptiveStep.cpp:58-98; ownedVolume) from its values loaded by the caller;
// returns the clamped moisture.
struct FinIn {
  double w0, dzc, ts, tr, qxp, qxm, qyp, qym, qzt, qzb, axc, ayc, vga, vgn, ksz;
  bool top;
};

struct FinAcc {
  double vl = 0.0, inflow = 0.0, dqmax = -DBL_MAX, dtco = DBL_MAX, vol = 0.0;
};

__device__ __forceinline__ double finalize_cell(const Dims& d, const FinIn& v, long long c, int j,
                                                int i, int k, double dtg, double co_max,
                                                double* __restrict__ vloss, FinAcc& acc) {
  const double volume = d.az * v.dzc;
  double w = v.w0;
  if (w > v.ts) {
    const double ex = (w - v.ts) * volume;
    vloss[c] += ex;
    acc.vl += ex;
    w = v.ts;
  } else if (w < v.tr) {
    const double de = (v.tr - w) * volume;
    vloss[c] -= de;
    acc.vl -= de;
    w = v.tr;
  }
  acc.vol += w * d.az * v.dzc;
  if (v.top) acc.inflow -= v.qzt * dtg;
  if (k == d.nz - 1) acc.inflow += v.qzb * dtg;
  if (i == 1) acc.inflow -= v.qxm * dtg;
  if (i == d.nx) acc.inflow += v.qxp * dtg;
  if (j == 1) acc.inflow -= v.qym * dtg;
  if (j == d.ny) acc.inflow += v.qyp * dtg;
  if (!v.top) {
    // |q_in - q_out| per unit area, grouped by direction (three divisions
    // instead of the reference's six; equal up to rounding).
    const double dq =
        fabs((v.qxp - v.qxm) / v.axc + (v.qyp - v.qym) / v.ayc + (v.qzb - v.qzt) / d.az) * dtg /
        v.dzc;
    if (dq > acc.dqmax) acc.dqmax = dq;
    if (w < v.ts) {
      const Soil so{v.vga, v.vgn, v.ts, v.tr, 0.0};
      const double dk = vg_dkdtheta(so, w, v.ksz);
      const double t = co_max * v.dzc / dk;
      if (t < acc.dtco) acc.dtco = t;
    }
  }
  return w;
}

// The finalize reductions of a block into the partial slots.
__device__ __forceinline__ void finalize_reduce(const FinAcc& acc, double* partial, int nblk,
                                                int bid) {
  double s = block_reduce(acc.vl, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPVloss * nblk + bid] = s;
  s = block_reduce(acc.inflow, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPInflow * nblk + bid] = s;
  s = block_reduce(acc.dqmax, MaxOp(), -DBL_MAX);
  if (threadIdx.x == 0) partial[kPDqmax * nblk + bid] = s;
  s = block_reduce(acc.dtco, MinOp(), DBL_MAX);
  if (threadIdx.x == 0) partial[kPDtco * nblk + bid] = s;
  s = block_reduce(acc.vol, SumOp(), 0.0);
  if (threadIdx.x == 0) partial[kPVol * nblk + bid] = s;
}

__device__ __forceinline__ void finalize_body(Dims d, Fields f, double* __restrict__ wc,
                                              double* __restrict__ vloss,
                                              const double* __restrict__ qx,
                                              const double* __restrict__ qy,
                                              const double* __restrict__ qzf,
                                              const double* __restrict__ dtgp, double co_max,
                                              double* partial, int nblk, const int bid,
                                              const int G) {
  const double dtg = *dtgp;
  FinAcc acc;
  for (long long c = bid * static_cast<long long>(blockDim.x) + threadIdx.x; c < d.ncell;
       c += static_cast<long long>(G) * blockDim.x) {
    int j, i, k;
    unflatten(d, c, j, i, k);
    if (j < 1 || j > d.ny || i < 1 || i > d.nx) continue;
    const long long fz = fidx(d, j, i, k);
    const long long cu = (k >= 1) ? c - 1 : c;
    const int8_t ac = f.act[c];
    const int8_t au = (k >= 1) ? f.act[cu] : int8_t(0);
    FinIn v;
    v.w0 = wc[c];
    v.dzc = f.dz[c];
    v.ts = f.wcs[c];
    v.tr = f.wcr[c];
    v.qxp = qx[c];
    v.qxm = qx[c - d.sx];
    v.qyp = qy[c];
    v.qym = qy[c - d.sy];
    v.qzt = qzf[fz];
    v.qzb = qzf[fz + 1];
    v.axc = f.ax[c];
    v.ayc = f.ay[c];
    v.vga = f.vga[c];
    v.vgn = f.vgn[c];
    v.ksz = f.ksz[c];
    v.top = (k == 0) || !au;
    if (!ac) continue;
    const double w = finalize_cell(d, v, c, j, i, k, dtg, co_max, vloss, acc);
    if (w != v.w0) wc[c] = w;
  }
  finalize_reduce(acc, partial, nblk, bid);
}

__global__ void __launch_bounds__(kBlock, 4) k_finalize(Dims d, Fields f, double* __restrict__ wc,
                                                        double* __restrict__ vloss,
                                                        const double* __restrict__ qx,
                                                        const double* __restrict__ qy,
                                                        const double* __restrict__ qzf,
                                                        const double* __restrict__ dtgp,
                                                        double co_max, double* partial, int nblk) {
  finalize_body(d, f, wc, vloss, qx, qy, qzf, dtgp, co_max, partial, nblk, blockIdx.x, gridDim.x);
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
// The step's dtg is read from out->next_dt, where the step found it, and the
// controller's next dt replaces it there.
__device__ __forceinline__ void step_info_body(const double* partial, int nblk, int off, int cpl,
                                               double dq_grow, double dq_shrink, double dt_min,
                                               double dt_max, double dtg, StepOut* out) {
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
  if (cpl) {
    // exchanged, bounce, vent, vent_thin, evap, mode-3 clamp (frehg_gw_coupled_audit order);
    // the reallocation's vent books are zero when it is disabled
    const int slot[6] = {kPExch, kPBounce, kPVent, kPThin, kPEvap, kPClamp};
    for (int s = 0; s < 6; ++s) {
      double v = reduce_slot(partial + slot[s] * nblk, nblk, SumOp(), 0.0);
      if (off && (slot[s] == kPVent || slot[s] == kPThin)) v = 0.0;
      if (threadIdx.x == 0) out->cpl[s] = v;
    }
  }
}

__global__ void k_step_info(const double* partial, int nblk, int off, int cpl, double dq_grow,
                            double dq_shrink, double dt_min, double dt_max, StepOut* out) {
  const double dtg = out->next_dt;  // read by every thread before thread 0 replaces it
  step_info_body(partial, nblk, off, cpl, dq_grow, dq_shrink, dt_min, dt_max, dtg, out);
}

__global__ void k_volume_final(const double* partial, int nblk, StepOut* out) {
  const double vol = reduce_slot(partial, nblk, SumOp(), 0.0);
  if (threadIdx.x == 0) out->volume = vol;
}

// The coupler window's four books (k_cpl_seepage) in a fixed order.
__global__ void k_cpl_window_final(const double* partial, int nblk, StepOut* out) {
  for (int s = 0; s < 4; ++s) {
    const double v = reduce_slot(partial + s * nblk, nblk, SumOp(), 0.0);
    if (threadIdx.x == 0) out->win[s] = v;
  }
}

// ---------------------------------------------------------------- batched phases
// One launch runs a phase for every member of a batch: block b belongs to the
// member whose range [first[i], first[i+1]) holds it, loads that member's
// record into shared memory and runs the phase's body on its own blocks.

__device__ inline void load_member(const StepArgs* tab, const int* first, int n, StepArgs& sa,
                                   int& bid, int& G) {
  __shared__ int si;
  if (threadIdx.x == 0) si = coop::instance_of(first, n, blockIdx.x);
  __syncthreads();
  const int i = si;
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(tab + i);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sa);
  for (int w = threadIdx.x; w < static_cast<int>(sizeof(StepArgs) / 8); w += blockDim.x)
    dst[w] = src[w];
  bid = blockIdx.x - first[i];
  G = first[i + 1] - first[i];
  __syncthreads();
}

static_assert(sizeof(StepArgs) % 8 == 0, "StepArgs is copied in 8-byte words");

__global__ void k_ghosts_batch(const StepArgs* tab, const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  ghosts_body(sa.d, sa.f, sa.hn, sa.wcn, bid, G);
}

__global__ void __launch_bounds__(kBlock) k_closure_pred_batch(const StepArgs* tab,
                                                               const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  closure_pred_body(sa.d, sa.f, sa.hn, sa.kcx, sa.kcy, sa.kcz, sa.ch, bid, G);
}

__global__ void __launch_bounds__(kBlock, 2) k_assemble_batch(const StepArgs* tab,
                                                              const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  assemble_body<false, false>(sa.d, sa.f, sa.kx, sa.ky, sa.kzf, sa.hn, sa.wcn, sa.ch, &sa.dtg, sa.diag, sa.gxp,
                sa.gyp, sa.gzp, sa.rhs, sa.mixed ? sa.x : nullptr, nullptr, 0.0, bid, G);
}

__global__ void __launch_bounds__(kBlock, 4) k_faces_batch(const StepArgs* tab, const int* first,
                                                           int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  const PassK pk{sa.kcx, sa.kcy, sa.kcz, sa.wcn};
  faces_body<false>(sa.d, sa.f, pk, sa.kx, sa.ky, sa.kzf, bid, G);
}

__global__ void __launch_bounds__(kBlock) k_closure_corr_batch(const StepArgs* tab,
                                                               const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  closure_corr_body(sa.d, sa.f, sa.x, sa.hn, sa.hp, sa.kcx, sa.kcy, sa.kcz, bid, G);
}

__global__ void __launch_bounds__(kBlock, 2) k_flux_batch(const StepArgs* tab, const int* first,
                                                          int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  const PassK pk{sa.kcx, sa.kcy, sa.kcz, sa.wcn};
  flux_body<false, false>(sa.d, sa.f, pk, sa.hp, sa.wcn, sa.kx, sa.ky, sa.kzf, sa.qx, sa.qy, sa.qzf, &sa.dtg, bid,
            G);
}

__global__ void __launch_bounds__(kBlock, 4) k_update_wc_batch(const StepArgs* tab,
                                                               const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  update_wc_body<false>(sa.d, sa.f, sa.hp, sa.hn, sa.wcn, sa.qx, sa.qy, sa.qzf, &sa.dtg, sa.wcu, sa.satf,
                 sa.colflag, sa.partial + kPSs * sa.nblk, bid, G);
}

__global__ void __launch_bounds__(kBlock, 3) k_classify_batch(const StepArgs* tab,
                                                              const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  classify_body<false>(sa.d, sa.f, sa.kx, sa.ky, sa.kzf, sa.wcu, sa.hp, sa.satf, sa.wc_out, sa.h_out,
                sa.room, sa.sup, sa.sdn, sa.colflag, sa.partial + kPAdj * sa.nblk,
                sa.partial + kPDrop * sa.nblk, bid, G);
}

__global__ void __launch_bounds__(kBlock) k_walk_batch(const StepArgs* tab, const int* first,
                                                       int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  if (sa.warp_walk) {
    walk_body<false>(sa.d, sa.f, sa.wc_out, sa.room, sa.sup, sa.sdn, sa.qzf, sa.colflag, &sa.dtg,
              sa.partial, sa.nblk, nullptr, nullptr, bid, G);
  } else {
    walk_thread_body<false>(sa.d, sa.f, sa.wc_out, sa.room, sa.sup, sa.sdn, sa.qzf, sa.colflag, &sa.dtg,
                     sa.partial, sa.nblk, nullptr, nullptr, bid, G);
  }
}

__global__ void __launch_bounds__(kBlock, 4) k_finalize_batch(const StepArgs* tab,
                                                              const int* first, int n) {
  __shared__ StepArgs sa;
  int bid, G;
  load_member(tab, first, n, sa, bid, G);
  finalize_body(sa.d, sa.f, sa.wc_out, sa.vloss, sa.qx, sa.qy, sa.qzf, &sa.dtg, sa.co_max,
                sa.partial, sa.nblk, bid, G);
}

// One block per member.
__global__ void k_step_info_batch(const StepArgs* tab) {
  __shared__ StepArgs sa;
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(tab + blockIdx.x);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sa);
  for (int w = threadIdx.x; w < static_cast<int>(sizeof(StepArgs) / 8); w += blockDim.x)
    dst[w] = src[w];
  __syncthreads();
  step_info_body(sa.partial, sa.nblk, sa.d.off, (sa.f.cpl != nullptr), sa.dq_grow, sa.dq_shrink, sa.dt_min,
                 sa.dt_max, sa.dtg, sa.out);
}

// The members' step records into one array, for a single read-back.
__global__ void k_gather_outs(const StepArgs* tab, StepOut* outs, int n) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const unsigned* src = reinterpret_cast<const unsigned*>(tab[i].out);
    unsigned* dst = reinterpret_cast<unsigned*>(outs + i);
    for (int w = threadIdx.x; w < static_cast<int>(sizeof(StepOut) / 4); w += blockDim.x)
      dst[w] = src[w];
  }
}

}  // namespace

// ---------------------------------------------------------------- launchers
cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<const void*, size_t> limit;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limit[kernel];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(bytes));
  if (e == cudaSuccess) cur = bytes;
  return e;
}

// Kernels that need the step's dtg read it on the device from the step record
// (see k_step_info), so a captured step replays with the dt the previous step
// chose.
inline const double* dtg_slot(const Device& D) { return &D.out->next_dt; }

int ghost_blocks(const Device& D) {
  const long long n = 2LL * (D.d.nx + D.d.ny) * D.d.nz;
  return static_cast<int>(std::min<long long>((n + kBlock - 1) / kBlock, 4096));
}

void launch_ghosts(const Device& D, double* h, double* wc) {
  k_ghosts<<<ghost_blocks(D), kBlock, 0, D.stream>>>(D.d, D.f, h, wc);
  ++D.launches;
}

void launch_closure_pred(const Device& D, const double* h) {
  k_closure_pred<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, h, D.kcx, D.kcy, D.kcz,
                                                         D.ch);
  ++D.launches;
}

// The predictor's faces go through D.kx, D.ky, D.kzf (free until k_flux).
void launch_assemble(const Device& D, const double* hn, const double* wcn, bool warm,
                     const double* hprev, double ratio) {
  const PassK pk{D.kcx, D.kcy, D.kcz, wcn};
  const auto faces = (D.f.cpl != nullptr) ? k_faces<true> : k_faces<false>;
  const bool cpl = D.f.cpl != nullptr, baro = D.f.baro != nullptr;
  const auto assemble = cpl ? (baro ? k_assemble<true, true> : k_assemble<true, false>)
                            : (baro ? k_assemble<false, true> : k_assemble<false, false>);
  faces<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, pk, D.kx, D.ky, D.kzf);
  assemble<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.kx, D.ky, D.kzf, hn, wcn, D.ch,
                                                     dtg_slot(D), D.diag, D.gxp, D.gyp, D.gzp,
                                                     D.rhs, warm ? D.x : nullptr,
                                                     warm ? hprev : nullptr, ratio);
  D.launches += 2;
}

// The fused predictor where it applies (groundwater-only domain, nz <= 256);
// false: the caller launches the separate passes.
bool launch_predict(const Device& D, const double* hn, const double* wcn, bool mixed) {
  if (D.f.cpl != nullptr || D.f.baro != nullptr || D.d.nz > 256) return false;
  const int E = D.d.nz <= 32 ? 1 : D.d.nz <= 64 ? 2 : D.d.nz <= 128 ? 4 : 8;
  using Kern = void (*)(Dims, Fields, const double*, const double*, const double*, double*,
                        double*, double*, double*, double*, double*, float*, float*, float*,
                        float*, float*, float*);
  Kern k;
  if (mixed) k = E == 1 ? k_predict<1, true> : E == 2 ? k_predict<2, true>
               : E == 4 ? k_predict<4, true> : k_predict<8, true>;
  else k = E == 1 ? k_predict<1, false> : E == 2 ? k_predict<2, false>
         : E == 4 ? k_predict<4, false> : k_predict<8, false>;
  const size_t smem = pred_smem_bytes(E);
  if (raise_smem_limit(reinterpret_cast<const void*>(k), smem) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const dim3 grid((D.d.nx + kPredCols - 1) / kPredCols, (D.d.ny + kPredRows - 1) / kPredRows);
  k<<<grid, kPredWarps * 32, smem, D.stream>>>(D.d, D.f, hn, wcn, dtg_slot(D), D.diag, D.gxp,
                                                D.gyp, D.gzp, D.rhs, mixed ? D.x : nullptr,
                                                D.diag32, D.gxp32, D.gyp32, D.gzp32, D.dinv32,
                                                D.l32);
  ++D.launches;
  return true;
}

// The fused corrector where it applies (groundwater-only domain, nz <= 256);
// false: the caller launches the separate passes.
bool launch_correct(const Device& D, const double* hn, const double* wcn) {
  if (D.f.cpl != nullptr || D.f.baro != nullptr || D.d.nz > 256) return false;
  const int E = D.d.nz <= 32 ? 1 : D.d.nz <= 64 ? 2 : D.d.nz <= 128 ? 4 : 8;
  const auto k = E == 1 ? k_correct<1> : E == 2 ? k_correct<2> : E == 4 ? k_correct<4>
                                                                  : k_correct<8>;
  const size_t smem = corr_smem_bytes(E);
  if (raise_smem_limit(reinterpret_cast<const void*>(k), smem) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  k<<<cells_grid(D), kCorrWarps * 32, smem, D.stream>>>(
      D.d, D.f, D.x, hn, wcn, dtg_slot(D), D.hp, D.kx, D.ky, D.kzf, D.qx, D.qy, D.qzf, D.wcu,
      D.satf, D.colflag, D.partial + kPSs * D.nblk);
  ++D.launches;
  return true;
}

void launch_closure_corr(const Device& D, const double* hn) {
  k_closure_corr<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.x, hn, D.hp, D.kcx, D.kcy,
                                                         D.kcz);
  ++D.launches;
}

void launch_flux(const Device& D, const double* wcn) {
  PassK pk{D.kcx, D.kcy, D.kcz, wcn};
  const bool cpl = D.f.cpl != nullptr, baro = D.f.baro != nullptr;
  const auto flux = cpl ? (baro ? k_flux<true, true> : k_flux<true, false>)
                        : (baro ? k_flux<false, true> : k_flux<false, false>);
  flux<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, pk, D.hp, wcn, D.kx, D.ky, D.kzf, D.qx,
                                                 D.qy, D.qzf, dtg_slot(D));
  ++D.launches;
}

void launch_update_wc(const Device& D, const double* hn, const double* wcn) {
  const auto update = (D.f.baro != nullptr) ? k_update_wc<true> : k_update_wc<false>;
  update<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.hp, hn, wcn, D.qx, D.qy, D.qzf,
                                                      dtg_slot(D), D.wcu, D.satf, D.colflag,
                                                      D.partial + kPSs * D.nblk);
  ++D.launches;
}

void launch_classify(const Device& D, double* wc_out, double* h_out) {
  const auto classify = (D.f.baro != nullptr) ? k_classify<true> : k_classify<false>;
  classify<<<cells_grid(D), kBlock, 0, D.stream>>>(
      D.d, D.f, D.kx, D.ky, D.kzf, D.wcu, D.hp, D.satf, wc_out, h_out, D.room, D.sup, D.sdn,
      D.colflag,
      D.partial + kPAdj * D.nblk, D.partial + kPDrop * D.nblk);
  ++D.launches;
}

// Columns up to kWalkMaxNz cells take the warp walk (dynamic shared memory
// opted in up to kWalkSmemMax); deeper columns take the per-thread walk.
constexpr int kWalkMaxNz = 256;
constexpr size_t kWalkSmemMax = 96 * 1024;

void launch_walk(const Device& D, double* wc_out) {
  const size_t smem = kWalkWarps * walk_warp_bytes(D.d.nz);
  if (D.d.nz <= kWalkMaxNz && smem <= kWalkSmemMax &&
      raise_smem_limit(reinterpret_cast<const void*>((D.f.cpl != nullptr) ? k_walk<true> : k_walk<false>),
                       smem) == cudaSuccess) {
    const auto walk = (D.f.cpl != nullptr) ? k_walk<true> : k_walk<false>;
    walk<<<cells_grid(D), kBlock, smem, D.stream>>>(D.d, D.f, wc_out, D.room, D.sup, D.sdn,
                                                      D.qzf, D.colflag, dtg_slot(D), D.partial,
                                                      D.nblk, D.pcorr, D.win_vent);
  } else {
    const auto walk = (D.f.cpl != nullptr) ? k_walk_thread<true> : k_walk_thread<false>;
    walk<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, wc_out, D.room, D.sup, D.sdn,
                                                          D.qzf, D.colflag, dtg_slot(D),
                                                          D.partial, D.nblk, D.pcorr, D.win_vent);
  }
  ++D.launches;
}

// accumulateTransportWindow (RichardsSolver.cpp:826-847): q dtg of every x, y
// and z face slot into the window, the z faces with the walks' path records
// (written this step in the flagged columns only; the others have none).
__global__ void k_window_accum(Dims d, const double* __restrict__ qx,
                               const double* __restrict__ qy, const double* __restrict__ qzf,
                               const double* __restrict__ pcorr, const int* __restrict__ colflag,
                               const double* __restrict__ dtgp, double* __restrict__ wx,
                               double* __restrict__ wy, double* __restrict__ wz) {
  const double dtg = *dtgp;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long t0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  for (long long c = t0; c < d.ncell; c += stride) {
    wx[c] += qx[c] * dtg;
    wy[c] += qy[c] * dtg;
  }
  const long long nf = d.ncol * (d.nz + 1);
  for (long long q = t0; q < nf; q += stride) {
    const long long col = q / (d.nz + 1);
    const double corr = colflag[col] ? pcorr[q] : 0.0;
    wz[q] += (qzf[q] + corr) * dtg;
  }
}

void launch_window_accum(const Device& D) {
  k_window_accum<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.qx, D.qy, D.qzf, D.pcorr,
                                                         D.colflag, dtg_slot(D), D.win_x,
                                                         D.win_y, D.win_z);
  ++D.launches;
}

void launch_finalize(const Device& D, double* wc_out, double co_max) {
  k_finalize<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, wc_out, D.vloss, D.qx, D.qy,
                                                     D.qzf, dtg_slot(D), co_max, D.partial, D.nblk);
  ++D.launches;
}

void launch_step_info(const Device& D, double dq_grow, double dq_shrink,
                      double dt_min, double dt_max) {
  k_step_info<<<1, kBlock, 0, D.stream>>>(D.partial, D.nblk, D.d.off, (D.f.cpl != nullptr), dq_grow,
                                          dq_shrink, dt_min, dt_max, D.out);
  ++D.launches;
}

int column_blocks(const Device& D) {
  const long long n = static_cast<long long>(D.d.nx) * D.d.ny;
  return static_cast<int>(std::min<long long>((n + kBlock - 1) / kBlock, 4096));
}

void launch_cpl_mode(const Device& D, const double* hn) {
  k_cpl_mode<<<column_blocks(D), kBlock, 0, D.stream>>>(D.d, D.f, hn, dtg_slot(D));
  ++D.launches;
}

void launch_cpl_book(const Device& D, const double* wcn) {
  k_cpl_book<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.hp, wcn, D.qzf, dtg_slot(D),
                                                     D.partial, D.nblk);
  ++D.launches;
}

void launch_cpl_begin_window(const Device& D) {
  const int nb = static_cast<int>(std::min<long long>((D.d.ncol + kBlock - 1) / kBlock, 4096));
  k_cpl_begin_window<<<nb, kBlock, 0, D.stream>>>(D.d, D.f);
  ++D.launches;
}

// The window's books use the first four partial slots (free once the step
// record is out).
void launch_cpl_seepage(const Device& D, double dt) {
  k_cpl_seepage<<<cells_grid(D), kBlock, 0, D.stream>>>(D.d, D.f, D.surf[6], D.surf[7], dt,
                                                        D.partial, D.nblk);
  k_cpl_window_final<<<1, kBlock, 0, D.stream>>>(D.partial, D.nblk, D.out);
  D.launches += 2;
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

// ---------------------------------------------------------------- batched phases (host)
// Blocks of a member in the batched cell passes: a block per 8 cells a thread
// (at most the member's own single-domain count).  Many members share each
// launch, so the single-domain count (up to 8 blocks per SM for every
// member, one or two cells a thread on small members) only added blocks and
// their reductions; the member's arithmetic per cell does not depend on it,
// its partial sums' order does (on its own size only).
constexpr int kBatchCellsPerThread = 8;
int batch_cell_blocks(const Device& D) {
  const long long per = static_cast<long long>(kBlock) * kBatchCellsPerThread;
  const long long want = (D.d.ncell + per - 1) / per;
  return static_cast<int>(std::max(1LL, std::min<long long>(want, D.nblk)));
}

void fill_step_args(const Device& D, bool mixed, double dtg, double co_max, double dq_grow,
                    double dq_shrink, double dt_min, double dt_max, StepArgs& a) {
  std::memset(&a, 0, sizeof(a));
  const int cur = D.cur, nxt = 1 - D.cur;
  a.d = D.d;
  a.f = D.f;
  a.hn = D.h[cur];
  a.wcn = D.wc[cur];
  a.h_out = D.h[nxt];
  a.wc_out = D.wc[nxt];
  a.hp = D.hp;
  a.wcu = D.wcu;
  a.ch = D.ch;
  a.kcx = D.kcx;
  a.kcy = D.kcy;
  a.kcz = D.kcz;
  a.kx = D.kx;
  a.ky = D.ky;
  a.kzf = D.kzf;
  a.qx = D.qx;
  a.qy = D.qy;
  a.qzf = D.qzf;
  a.vloss = D.vloss;
  a.room = D.room;
  a.sup = D.sup;
  a.sdn = D.sdn;
  a.diag = D.diag;
  a.gxp = D.gxp;
  a.gyp = D.gyp;
  a.gzp = D.gzp;
  a.rhs = D.rhs;
  a.x = D.x;
  a.diag32 = D.diag32;
  a.gxp32 = D.gxp32;
  a.gyp32 = D.gyp32;
  a.gzp32 = D.gzp32;
  a.dinv32 = D.dinv32;
  a.l32 = D.l32;
  a.satf = D.satf;
  a.colflag = D.colflag;
  a.partial = D.partial;
  a.out = D.out;
  a.dtg = dtg;
  a.co_max = co_max;
  a.dq_grow = dq_grow;
  a.dq_shrink = dq_shrink;
  a.dt_min = dt_min;
  a.dt_max = dt_max;
  a.nblk = batch_cell_blocks(D);
  a.tc = line_tile_cols(D.d.nz);
  a.mixed = mixed ? 1 : 0;
  const size_t smem = kWalkWarps * walk_warp_bytes(D.d.nz);
  a.warp_walk = (D.d.nz <= kWalkMaxNz && smem <= kWalkSmemMax) ? 1 : 0;
}

cudaError_t phase_tables_build(PhaseTables& t, const std::vector<const Device*>& ds,
                               const std::vector<int>& mixed) {
  t.n = static_cast<int>(ds.size());
  cudaError_t e = cudaSuccess;
  if (t.n > t.cap) {
    // Grow (sizes first: freeing resets the record).
    const int n = t.n, cap = std::max(t.n, 2 * t.cap);
    phase_tables_free(t);
    t.n = n;
    t.cap = cap;
    e = cudaMalloc(&t.tab, sizeof(StepArgs) * cap);
    if (e == cudaSuccess) e = cudaMallocHost(&t.tab_host, sizeof(StepArgs) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&t.first_cells, sizeof(int) * (cap + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t.first_ghost, sizeof(int) * (cap + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t.first_factor, sizeof(int) * (cap + 1));
    if (e == cudaSuccess) e = cudaMalloc(&t.outs, sizeof(StepOut) * cap);
    if (e == cudaSuccess) e = cudaMallocHost(&t.outs_host, sizeof(StepOut) * cap);
  }
  std::vector<int> fc(t.n + 1, 0), fg(t.n + 1, 0), ff(t.n + 1, 0);
  t.walk_smem = 0;
  t.factor_smem = 0;
  for (int i = 0; i < t.n; ++i) {
    const Device& D = *ds[i];
    fc[i + 1] = fc[i] + batch_cell_blocks(D);
    fg[i + 1] = fg[i] + ghost_blocks(D);
    ff[i + 1] = ff[i] + (mixed[i] ? line_factor_blocks(D) : 0);
    const size_t ws = kWalkWarps * walk_warp_bytes(D.d.nz);
    if (D.d.nz <= kWalkMaxNz && ws <= kWalkSmemMax) t.walk_smem = std::max(t.walk_smem, ws);
    if (mixed[i]) t.factor_smem = std::max(t.factor_smem, line_factor_smem(D.d.nz));
  }
  t.grid_cells = fc.back();
  t.grid_ghost = fg.back();
  t.grid_factor = ff.back();
  if (e == cudaSuccess)
    e = cudaMemcpy(t.first_cells, fc.data(), sizeof(int) * fc.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(t.first_ghost, fg.data(), sizeof(int) * fg.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(t.first_factor, ff.data(), sizeof(int) * ff.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && t.walk_smem > 0)
    e = raise_smem_limit(reinterpret_cast<const void*>(k_walk_batch), t.walk_smem);
  return e;
}

void phase_tables_free(PhaseTables& t) {
  if (t.tab) cudaFree(t.tab);
  if (t.tab_host) cudaFreeHost(t.tab_host);
  if (t.first_cells) cudaFree(t.first_cells);
  if (t.first_ghost) cudaFree(t.first_ghost);
  if (t.first_factor) cudaFree(t.first_factor);
  if (t.outs) cudaFree(t.outs);
  if (t.outs_host) cudaFreeHost(t.outs_host);
  t = PhaseTables{};
}

cudaError_t batch_predictor(const PhaseTables& t, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(t.tab, t.tab_host, sizeof(StepArgs) * t.n,
                                  cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  k_ghosts_batch<<<t.grid_ghost, kBlock, 0, s>>>(t.tab, t.first_ghost, t.n);
  k_closure_pred_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_faces_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_assemble_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  if (t.grid_factor > 0) {
    e = launch_line_factor_batch(t, s);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

cudaError_t batch_corrector(const PhaseTables& t, cudaStream_t s) {
  k_closure_corr_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_flux_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_update_wc_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_classify_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_walk_batch<<<t.grid_cells, kBlock, t.walk_smem, s>>>(t.tab, t.first_cells, t.n);
  k_finalize_batch<<<t.grid_cells, kBlock, 0, s>>>(t.tab, t.first_cells, t.n);
  k_step_info_batch<<<t.n, kBlock, 0, s>>>(t.tab);
  k_gather_outs<<<std::min(t.n, 1024), 32, 0, s>>>(t.tab, t.outs, t.n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(t.outs_host, t.outs, sizeof(StepOut) * t.n, cudaMemcpyDeviceToHost, s);
}

}  // namespace fgw
