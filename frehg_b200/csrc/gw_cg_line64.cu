// The FP64 line form of the predictor solve: the mixed form's algorithm with
// every vector and coefficient in FP64 -- CG preconditioned by the exact
// solve of each column's vertical tridiagonal block, inside defect
// correction on the true residual, started from h^n, with the mixed form's
// stopping rules (||b - A x|| <= outer_rtol ||b|| after at least one
// correction; inner solves to a reduction of 1e-4, the last only as far as
// the outer target needs).  It exists to measure what FP32 buys the mixed
// form: the two differ only in the inner precision, so their ratio is the
// precision's share and the ratio of this form to the Jacobi FP64 form
// (PETSc's x0 = 0, point Jacobi) the algorithm's.
//
// Columns of nz <= 256 cells (one warp per column, E consecutive cells a
// lane, as in the mixed form's column path); the stencil pass is cell
// parallel with one cell a thread.  FP64 traffic per cell and inner
// iteration: stencil pass 10 words (z, p_old, d, diag, gxp, gyp, gzp in; p,
// w, d out), update + line solve 6 words (r, w, dinv, l in; r, z out) --
// 128 B, the FP64 Jacobi iteration's 16 words.
#include "gw_coop.cuh"
#include "gw_internal.h"
#include "gw_linefactor.cuh"
#include "gw_linesolve.cuh"

namespace fgw {

using namespace coop;

namespace {

struct Line64Args {
  Dims d;
  const double *diag, *gxp, *gyp, *gzp, *b;
  double *x0, *x1;              // iterate ping-pong (x0 holds h^n at entry)
  const double *dinv, *l;       // column LDL^T factors
  double *r, *z, *p0, *p1, *w, *dd;
  double* part;                 // 4 x G
  CgState* st;
  double outer_rtol, inner_rtol, atol;
  int max_inner, max_outer, max_total;
};

// x + d with the inner solve's last update pal * pend still pending.
__device__ inline double x64_at(const Line64Args& a, const double* __restrict__ xo,
                                const double* __restrict__ pend, double pal, long long c) {
  double v = a.dd[c];
  if (pal != 0.0) v += pal * pend[c];
  return xo[c] + v;
}

__device__ inline double outer64_ax(const Line64Args& a, const double* __restrict__ xo,
                                    const double* __restrict__ pend, double pal, long long c,
                                    long long sx, long long sy) {
  double ax = a.gyp[c - sy] * x64_at(a, xo, pend, pal, c - sy);
  ax += a.gxp[c - sx] * x64_at(a, xo, pend, pal, c - sx);
  ax += a.gzp[c - 1] * x64_at(a, xo, pend, pal, c - 1);
  ax += a.diag[c] * x64_at(a, xo, pend, pal, c);
  ax += a.gzp[c] * x64_at(a, xo, pend, pal, c + 1);
  ax += a.gxp[c] * x64_at(a, xo, pend, pal, c + sx);
  ax += a.gyp[c] * x64_at(a, xo, pend, pal, c + sy);
  return ax;
}

// Stencil pass: p = z + bc p_old at the seven points, w = A p, and (after
// the first iteration of an inner solve) d += pal p_old; returns p'w.
template <bool FIRST>
__device__ inline double line64_phase_a(const Line64Args& a, double bc,
                                        const double* __restrict__ pold,
                                        double* __restrict__ pnew, double pal, long long t0,
                                        long long stride) {
  const long long N = a.d.ncell, sx = a.d.sx, sy = a.d.sy;
  auto pv = [&](long long m) { return FIRST ? a.z[m] : a.z[m] + bc * pold[m]; };
  double pw = 0.0;
  for (long long c = t0; c < N; c += stride) {
    const double po = FIRST ? 0.0 : pold[c];
    const double dv = FIRST ? 0.0 : a.dd[c];
    const double pc = pv(c);
    double wv = a.gyp[c - sy] * pv(c - sy);
    wv += a.gxp[c - sx] * pv(c - sx);
    wv += a.gzp[c - 1] * pv(c - 1);
    wv += a.diag[c] * pc;
    wv += a.gzp[c] * pv(c + 1);
    wv += a.gxp[c] * pv(c + sx);
    wv += a.gyp[c] * pv(c + sy);
    pnew[c] = pc;
    a.w[c] = wv;
    if (!FIRST) a.dd[c] = dv + pal * po;
    pw += pc * wv;
  }
  return pw;
}

template <int E>
__device__ __forceinline__ void line64_body(const Line64Args& a, const int bid, const int G) {
  const Dims& d = a.d;
  const int nz = d.nz;
  const long long N = d.ncell, sx = d.sx, sy = d.sy;
  const long long stride = static_cast<long long>(G) * blockDim.x;
  const long long t0 = bid * static_cast<long long>(blockDim.x) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool vec = (nz % E == 0);
  const long long gwarp = bid * static_cast<long long>(kCgBlock / 32) + (threadIdx.x >> 5);
  const long long nwarp = static_cast<long long>(G) * (kCgBlock / 32);
  double* const q0 = a.part;
  double* const q1 = a.part + G;
  double* const q2 = a.part + 2 * G;
  double* const q3 = a.part + 3 * G;

  // ||b|| (the first residual is b - A h^n, not b) and d = 0.
  double bb = 0.0;
  for (long long c = t0; c < N; c += stride) {
    const double bv = a.b[c];
    bb += bv * bv;
    a.dd[c] = 0.0;
  }
  double s0 = block_sum_all(bb);
  if (threadIdx.x == 0) q3[bid] = s0;
  if (!grid_sync(a.st, G)) return;

  double bnorm = 0.0, rnorm = 0.0;
  int total = 0, outer = 0, reason = 0, final_buf = 0;
  // The last inner iteration's update d += s_pal p_(s_pbuf), applied by the
  // next stencil pass or outer pass (s_pal = 0: none); thread 0 writes them
  // after a grid sync that follows every read of the old values.
  __shared__ double s_pal;
  __shared__ int s_pbuf;
  if (threadIdx.x == 0) {
    s_pal = 0.0;
    s_pbuf = 0;
  }
  __syncthreads();
  for (int o = 0;; ++o) {
    const double pal = s_pal;
    const double* __restrict__ pend = s_pbuf ? a.p1 : a.p0;
    const double* __restrict__ xo = (o & 1) ? a.x1 : a.x0;
    double* __restrict__ xn = (o & 1) ? a.x0 : a.x1;
    // Outer pass: x_new = x + d, r = b - A x_new, z = T^-1 r.
    double rn2 = 0.0, zz = 0.0, zr = 0.0;
    for (long long col = gwarp; col < d.ncol; col += nwarp) {
      const long long cb = col * nz;
      const int k0 = lane * E;
      double rv[E], zv[E], lk[E], di[E], xv[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        rv[e] = 0.0;
        xv[e] = 0.0;
        if (k0 + e < nz) {
          const long long c = cb + k0 + e;
          const double rr = a.b[c] - outer64_ax(a, xo, pend, pal, c, sx, sy);
          xv[e] = x64_at(a, xo, pend, pal, c);
          rn2 += rr * rr;
          rv[e] = rr;
        }
      }
      ld_col<E>(a.l, cb, lane, nz, vec, lk);
      ld_col<E>(a.dinv, cb, lane, nz, vec, di);
      warp_column_solve<E>(lk, di, lane, nz, rv, zv);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        if (k0 + e < nz) {
          xn[cb + k0 + e] = xv[e];
          zz += zv[e] * zv[e];
          zr += zv[e] * rv[e];
        }
      }
      st_col<E>(a.r, cb, lane, nz, vec, rv);
      st_col<E>(a.z, cb, lane, nz, vec, zv);
    }
    double s = block_sum_all(rn2);
    if (threadIdx.x == 0) q0[bid] = s;
    s = block_sum_all(zz);
    if (threadIdx.x == 0) q1[bid] = s;
    s = block_sum_all(zr);
    if (threadIdx.x == 0) q2[bid] = s;
    if (!grid_sync(a.st, G)) return;
    rnorm = sqrt(reduce_partials(q0, G));
    const double zn0 = sqrt(reduce_partials(q1, G));
    double beta = reduce_partials(q2, G);
    final_buf = (o & 1) ? 0 : 1;
    if (o == 0) bnorm = sqrt(reduce_partials(q3, G));
    if (!isfinite(rnorm)) {
      reason = -9;
      break;
    }
    // The warm start always takes one correction (h^n itself is not returned).
    if (o > 0 && rnorm <= fmax(a.outer_rtol * bnorm, a.atol)) {
      reason = (rnorm < a.atol) ? 3 : 2;
      break;
    }
    if (outer >= a.max_outer || total >= a.max_total) {
      reason = -3;
      break;
    }
    ++outer;
    if (threadIdx.x == 0) s_pal = 0.0;  // the outer pass applied it
    for (long long c = t0; c < N; c += stride) a.dd[c] = 0.0;
    const double need = (rnorm > 0.0) ? 0.5 * a.outer_rtol * bnorm / rnorm : a.inner_rtol;
    const double itol = fmax(a.inner_rtol, need) * zn0;
    double betaold = 1.0;
    for (int i = 0; i < a.max_inner && total < a.max_total; ++i) {
      if (beta == 0.0 || (i > 0 && beta * betaold <= 0.0)) break;
      const double bc = (i == 0) ? 0.0 : beta / betaold;
      const double* __restrict__ pold = (i & 1) ? a.p1 : a.p0;
      double* __restrict__ pnew = (i & 1) ? a.p0 : a.p1;
      const double pw = (i == 0) ? line64_phase_a<true>(a, bc, pold, pnew, 0.0, t0, stride)
                                 : line64_phase_a<false>(a, bc, pold, pnew, s_pal, t0, stride);
      s = block_sum_all(pw);
      if (threadIdx.x == 0) q0[bid] = s;
      if (!grid_sync(a.st, G)) return;
      const double dpi = reduce_partials(q0, G);
      if (!(dpi > 0.0)) break;  // breakdown: keep d, the outer sweep decides
      const double al = beta / dpi;
      betaold = beta;
      ++total;
      if (threadIdx.x == 0) {
        s_pal = al;
        s_pbuf = (i & 1) ? 0 : 1;
      }
      zz = 0.0;
      zr = 0.0;
      for (long long col = gwarp; col < d.ncol; col += nwarp) {
        const long long cb = col * nz;
        const int k0 = lane * E;
        double wv[E], rv[E], lk[E], di[E], zv[E];
        ld_col<E>(a.w, cb, lane, nz, vec, wv);
        ld_col<E>(a.r, cb, lane, nz, vec, rv);
        ld_col<E>(a.l, cb, lane, nz, vec, lk);
        ld_col<E>(a.dinv, cb, lane, nz, vec, di);
#pragma unroll
        for (int e = 0; e < E; ++e) rv[e] -= al * wv[e];
        warp_column_solve<E>(lk, di, lane, nz, rv, zv);
        st_col<E>(a.r, cb, lane, nz, vec, rv);
        st_col<E>(a.z, cb, lane, nz, vec, zv);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          if (k0 + e < nz) {
            zz += zv[e] * zv[e];
            zr += zv[e] * rv[e];
          }
        }
      }
      s = block_sum_all(zz);
      if (threadIdx.x == 0) q1[bid] = s;
      s = block_sum_all(zr);
      if (threadIdx.x == 0) q2[bid] = s;
      if (!grid_sync(a.st, G)) return;
      const double zn = sqrt(reduce_partials(q1, G));
      if (zn <= itol) break;
      beta = reduce_partials(q2, G);
    }
  }
  // The solution of the last outer pass lives in x1 after even passes.
  if (final_buf == 1) {
    for (long long c = t0; c < N; c += stride) a.x0[c] = a.x1[c];
  }
  if (bid == 0 && threadIdx.x == 0) {
    a.st->dp = rnorm;
    a.st->rnorm0 = bnorm;
    a.st->its = total;
    a.st->reason = reason;
    a.st->outer = outer;
  }
}

template <int E>
__global__ void __launch_bounds__(kCgBlock, 2) k_cg_line64(Line64Args a) {
  line64_body<E>(a, blockIdx.x, gridDim.x);
}

// FP64 column factors: the warp scan of gw_linefactor.cuh over every column.
template <int E>
__global__ void __launch_bounds__(256) k_line_factor64(Dims d, const double* __restrict__ diag,
                                                       const double* __restrict__ gzp,
                                                       double* __restrict__ dinv,
                                                       double* __restrict__ l) {
  const int lane = threadIdx.x & 31, nz = d.nz, k0 = lane * E;
  const long long nw = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
  for (long long col = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
       col < d.ncol; col += nw) {
    const long long cb = col * nz;
    double av[E], ev[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = k0 + e;
      av[e] = 1.0;
      ev[e] = 0.0;
      if (k < nz) {
        av[e] = diag[cb + k];
        ev[e] = gzp[cb + k];
      }
    }
    factor_column64<E>(nz, cb, av, ev, dinv, l);
  }
}

int line64_cells(int nz) { return nz <= 32 ? 1 : nz <= 64 ? 2 : nz <= 128 ? 4 : nz <= 256 ? 8 : 0; }

}  // namespace

cudaError_t launch_line_factor64(Device& D) {
  const int E = line64_cells(D.d.nz);
  if (!E) return cudaErrorInvalidValue;
  const long long per = 256 / 32;
  const int grid = static_cast<int>(std::min<long long>((D.d.ncol + per - 1) / per,
                                                        16LL * D.sm_count));
  auto k = E == 1 ? k_line_factor64<1> : E == 2 ? k_line_factor64<2>
         : E == 4 ? k_line_factor64<4> : k_line_factor64<8>;
  k<<<grid, 256, 0, D.stream>>>(D.d, D.diag, D.gzp, D.dinv64, D.l64);
  ++D.launches;
  return cudaGetLastError();
}

cudaError_t launch_cg_line64(Device& D, double atol, int maxit, double outer_rtol,
                             int max_outer) {
  const int E = line64_cells(D.d.nz);
  if (!E) return cudaErrorInvalidValue;
  using Kern = void (*)(Line64Args);
  const Kern k = E == 1 ? k_cg_line64<1> : E == 2 ? k_cg_line64<2>
               : E == 4 ? k_cg_line64<4> : k_cg_line64<8>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(k),
                                                kCgBlock, 0);
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  // 4 x g reduction partials fit the 4 x (4 sm_count) doubles allocated at create.
  if (per_sm > 4) per_sm = 4;
  const long long g = static_cast<long long>(per_sm) * D.sm_count;
  cudaMemsetAsync(&D.out->cg, 0, sizeof(CgState), D.stream);
  Line64Args a;
  a.d = D.d;
  a.diag = D.diag;
  a.gxp = D.gxp;
  a.gyp = D.gyp;
  a.gzp = D.gzp;
  a.b = D.rhs;
  a.x0 = D.x;
  a.x1 = D.xalt;
  a.dinv = D.dinv64;
  a.l = D.l64;
  a.r = D.r;
  a.z = D.z;
  a.p0 = D.p0;
  a.p1 = D.p1;
  a.w = D.w;
  a.dd = D.d64;
  a.part = D.cgpart;
  a.st = &D.out->cg;
  a.outer_rtol = outer_rtol;
  a.inner_rtol = 1.0e-4;  // the mixed form's inner reduction
  a.atol = atol;
  a.max_inner = maxit;
  a.max_outer = max_outer;
  a.max_total = maxit;
  void* args[] = {&a};
  ++D.launches;
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k), dim3(g), dim3(kCgBlock),
                                     args, 0, D.stream);
}

}  // namespace fgw
