// Mixed-precision predictor solve: FP32 inner preconditioned CG inside FP64
// defect correction on the true residual.
//
//   x = h^n (the step-start head, written by the assembly; PETSc's x = 0
//            stays with the FP64 form, whose iteration counts are the
//            reference's)
//   repeat (outer sweep o = 0, 1, ...):
//     x <- x + d;  r = b - A x  in FP64 with the FP64 coefficients
//     stop when ||r||_2 <= outer_rtol ||b||_2 (after at least one
//     correction: h^n passing the test is not accurate enough)
//     solve A d = r approximately in FP32: CG preconditioned by the exact
//     solve of each column's vertical tridiagonal block (line Jacobi along
//     k), stopped at inner_rtol of the initial preconditioned norm
//
// The line preconditioner follows the thin-layer anisotropy of the head
// system (dz << dx makes the vertical legs 10^2-10^3 times the lateral ones):
// it solves the dominant couplings exactly and cuts the inner iteration count
// by an order of magnitude against point Jacobi.  Every iterate that leaves
// the solve is an FP64 vector whose FP64 residual met outer_rtol, so the
// solution's accuracy is set by the FP64 sweep, not by the FP32 arithmetic.
//
// Layout.  The tridiagonal solve needs whole columns.  For nz <= 256 phase B
// and the outer residual pass give each warp whole columns: row e of a column
// holds cells k = 32 e + lane (coalesced loads and stores), and the two
// bidiagonal sweeps of the LDL^T solve run as warp scans of affine maps, so
// every thread works and no block barrier is needed.  Deeper columns walk the
// domain in tiles of `tc` consecutive columns (one contiguous run of tc*nz
// cells in the halo layout), stage the tile in shared memory (row pitch nz+1
// so the per-column sweeps are bank-conflict free), let one thread per column
// run the LDL^T sweeps, and write back coalesced.
// Phase A (direction update + stencil product) is cell-parallel as in the
// FP64 kernel.  The correction update d += alpha p of an iteration is applied
// by the next iteration's phase A, which reads that p as p_old anyway (the
// last one of an inner solve by the outer pass).  FP32 inner traffic per cell
// and iteration: phase A 10 words (z, p_old, d, diag, gxp, gyp, gzp in;
// p_new, w, d out), phase B 6 words (r, w, dinv, l in; r, z out) -> 64 B.
#include <cfloat>
#include <cstring>

#include "gw_coop.cuh"
#include "gw_internal.h"
#include "gw_linefactor.cuh"
#include "gw_linesolve.cuh"

namespace fgw {

using namespace coop;

namespace {

constexpr int kFactorBlock = 256;
constexpr int kTileCells = 4096;  // tc * nz <= kTileCells (2 x 16 KB of FP32 staging)

// Deep columns (nz > 256; shallower ones take line_factor_warp_body below):
// cast the FP64 coefficients to FP32 and factor every column's tridiagonal
// block T = LDL^T (pivots in FP64, stored as FP32 1/d_k and l_k).
__device__ __forceinline__ void line_factor_body(Dims d, const double* __restrict__ diag,
                                                              const double* __restrict__ gxp,
                                                              const double* __restrict__ gyp,
                                                              const double* __restrict__ gzp,
                                                              float* diag32, float* gxp32,
                                                              float* gyp32, float* gzp32,
                                                              float* dinv32, float* l32, int tc, const int bid, const int G) {
  extern __shared__ double fsm[];
  const int nz = d.nz, nzp = nz + 1;
  double* s_a = fsm;
  double* s_e = fsm + static_cast<long long>(tc) * nzp;
  const long long ntiles = (d.ncol + tc - 1) / tc;
  for (long long t = bid; t < ntiles; t += G) {
    const long long base = t * tc * nz;
    const int ncols = static_cast<int>((d.ncol - t * tc) < tc ? (d.ncol - t * tc) : tc);
    const int ncells = ncols * nz;
    for (int f = threadIdx.x; f < ncells; f += blockDim.x) {
      const long long c = base + f;
      const int col = f / nz, k = f - col * nz;
      s_a[col * nzp + k] = diag[c];
      s_e[col * nzp + k] = gzp[c];
      diag32[c] = static_cast<float>(diag[c]);
      gxp32[c] = static_cast<float>(gxp[c]);
      gyp32[c] = static_cast<float>(gyp[c]);
      gzp32[c] = static_cast<float>(gzp[c]);
    }
    __syncthreads();
    if (threadIdx.x < ncols) {
      double* a = s_a + threadIdx.x * nzp;
      double* e = s_e + threadIdx.x * nzp;
      double dprev = a[0];
      a[0] = dprev;
      for (int k = 1; k < nz; ++k) {
        const double l = e[k - 1] / dprev;
        const double dk = a[k] - l * e[k - 1];
        e[k - 1] = l;
        a[k] = dk;
        dprev = dk;
      }
      e[nz - 1] = 0.0;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < ncells; f += blockDim.x) {
      const long long c = base + f;
      const int col = f / nz, k = f - col * nz;
      const double dk = s_a[col * nzp + k];
      dinv32[c] = (dk > 0.0 && isfinite(dk)) ? static_cast<float>(1.0 / dk)
                                             : static_cast<float>(1.0 / diag[c]);
      l32[c] = static_cast<float>(s_e[col * nzp + k]);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kFactorBlock) k_line_factor(Dims d, const double* __restrict__ diag,
                                                              const double* __restrict__ gxp,
                                                              const double* __restrict__ gyp,
                                                              const double* __restrict__ gzp,
                                                              float* diag32, float* gxp32,
                                                              float* gyp32, float* gzp32,
                                                              float* dinv32, float* l32, int tc) {
  line_factor_body(d, diag, gxp, gyp, gzp, diag32, gxp32, gyp32, gzp32, dinv32, l32, tc, blockIdx.x, gridDim.x);
}

// The same factorization with one warp per column (nz <= 256), by the warp
// scan of gw_linefactor.cuh.
template <int E>
__device__ __forceinline__ void line_factor_warp_body(
    Dims d, const double* __restrict__ diag, const double* __restrict__ gxp,
    const double* __restrict__ gyp, const double* __restrict__ gzp, float* __restrict__ diag32,
    float* __restrict__ gxp32, float* __restrict__ gyp32, float* __restrict__ gzp32,
    float* __restrict__ dinv32, float* __restrict__ l32, const int bid, const int G) {
  const int lane = threadIdx.x & 31, nz = d.nz, k0 = lane * E;
  const long long nw = static_cast<long long>(G) * (blockDim.x >> 5);
  for (long long col = static_cast<long long>(bid) * (blockDim.x >> 5) + (threadIdx.x >> 5);
       col < d.ncol; col += nw) {
    const long long cb = col * nz;
    double av[E], ev[E], xv[E], yv[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = k0 + e;
      av[e] = 1.0;
      ev[e] = xv[e] = yv[e] = 0.0;
      if (k < nz) {
        av[e] = diag[cb + k];
        ev[e] = gzp[cb + k];
        xv[e] = gxp[cb + k];
        yv[e] = gyp[cb + k];
      }
    }
    factor_column<E>(nz, cb, av, ev, xv, yv, diag32, gxp32, gyp32, gzp32, dinv32, l32);
  }
}

template <int E>
__global__ void __launch_bounds__(kFactorBlock) k_line_factor_warp(
    Dims d, const double* __restrict__ diag, const double* __restrict__ gxp,
    const double* __restrict__ gyp, const double* __restrict__ gzp, float* diag32, float* gxp32,
    float* gyp32, float* gzp32, float* dinv32, float* l32) {
  line_factor_warp_body<E>(d, diag, gxp, gyp, gzp, diag32, gxp32, gyp32, gzp32, dinv32, l32,
                           blockIdx.x, gridDim.x);
}

// Cells per lane of the warp factorization (0: the tiled path, nz > 256).
__host__ __device__ inline int factor_lane_cells(int nz) {
  return nz <= 32 ? 1 : nz <= 64 ? 2 : nz <= 128 ? 4 : nz <= 256 ? 8 : 0;
}

struct MixedArgs {
  Dims d;
  const double *diag, *gxp, *gyp, *gzp, *b;
  double *x0, *x1;
  const float *diag32, *gxp32, *gyp32, *gzp32, *dinv32, *l32;
  float *r32, *z32, *p0, *p1, *w32, *d32;
  double* part;  // 4 x G
  CgState* st;
  double outer_rtol, inner_rtol, atol;
  int max_inner, max_outer, max_total;
  int tc;
  int warm;     // x0 holds the starting iterate (h^n, written by the assembly)
  int variant;  // batched solves: 16 V + E (mixed_variant)
};

// Forward/backward LDL^T sweeps of one column: z = T^-1 r.  r and z live in
// the staged shared-memory tile; the factors are read straight from global
// memory (one thread walks its own contiguous column, so every 32-byte sector
// it touches serves 8 consecutive steps from L1).
__device__ inline void column_solve(const float* r, const float* __restrict__ dinv,
                                    const float* __restrict__ l, float* z, int nz) {
  float y = r[0];
  z[0] = y;
  for (int k = 1; k < nz; ++k) {
    y = r[k] - __ldg(l + k - 1) * y;
    z[k] = y;
  }
  float zk = z[nz - 1] * __ldg(dinv + nz - 1);
  z[nz - 1] = zk;
  for (int k = nz - 2; k >= 0; --k) {
    zk = z[k] * __ldg(dinv + k) - __ldg(l + k) * zk;
    z[k] = zk;
  }
}

__device__ inline float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ inline void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

// Phase A for V consecutive k-cells per thread (V = 4: 16-byte loads; the
// lower/upper z legs of the group come from gzp[c-1] and the group's own).
// (A (x + d))_c in FP64 with the FP64 coefficients, in the SpMV's fixed
// summation order (ym, xm, zm, diag, zp, xp, yp).
// The correction of cell c with the inner solve's last update pal * pend
// still pending (pal = 0: none, pend not read).
__device__ inline float corr_at(const MixedArgs& a, const float* __restrict__ pend, float pal,
                                long long c) {
  float v = a.d32[c];
  if (pal != 0.0f) v += pal * pend[c];
  return v;
}
__device__ inline double x_at(const MixedArgs& a, const double* __restrict__ xo,
                              const float* __restrict__ pend, float pal, long long c) {
  return xo[c] + static_cast<double>(corr_at(a, pend, pal, c));
}
__device__ inline double outer_ax(const MixedArgs& a, const double* __restrict__ xo,
                                  const float* __restrict__ pend, float pal, long long c,
                                  long long sx, long long sy) {
  const double xc = x_at(a, xo, pend, pal, c);
  double ax = a.gyp[c - sy] * x_at(a, xo, pend, pal, c - sy);
  ax += a.gxp[c - sx] * x_at(a, xo, pend, pal, c - sx);
  ax += a.gzp[c - 1] * x_at(a, xo, pend, pal, c - 1);
  ax += a.diag[c] * xc;
  ax += a.gzp[c] * x_at(a, xo, pend, pal, c + 1);
  ax += a.gxp[c] * x_at(a, xo, pend, pal, c + sx);
  ax += a.gyp[c] * x_at(a, xo, pend, pal, c + sy);
  return ax;
}

// FIRST (the first iteration of an inner solve): p = z, and p_old is not
// read.  Otherwise p = z + bc p_old and d += pal p_old (the previous
// iteration's update).
template <int V, bool FIRST>
__device__ inline double phase_a(const MixedArgs& a, float bc, const float* __restrict__ pold,
                                 float* __restrict__ pnew, float pal, long long t0,
                                 long long stride) {
  const long long N = a.d.ncell, sx = a.d.sx, sy = a.d.sy;
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  double pw = 0.0;
  if constexpr (V == 4) {
    for (long long q = t0; q < N / 4; q += stride) {
      const long long c = 4 * q;
      const float4 z = ld4(a.z32 + c), p = FIRST ? zero4 : ld4(pold + c);
      const float4 zxm = ld4(a.z32 + c - sx), pxm = FIRST ? zero4 : ld4(pold + c - sx);
      const float4 zxp = ld4(a.z32 + c + sx), pxp = FIRST ? zero4 : ld4(pold + c + sx);
      const float4 zym = ld4(a.z32 + c - sy), pym = FIRST ? zero4 : ld4(pold + c - sy);
      const float4 zyp = ld4(a.z32 + c + sy), pyp = FIRST ? zero4 : ld4(pold + c + sy);
      const float pkm = FIRST ? a.z32[c - 1] : a.z32[c - 1] + bc * pold[c - 1];
      const float pkp = FIRST ? a.z32[c + 4] : a.z32[c + 4] + bc * pold[c + 4];
      float4 dd = FIRST ? zero4 : ld4(a.d32 + c);
      const float4 dg = ld4(a.diag32 + c);
      const float4 gx = ld4(a.gxp32 + c), gxm = ld4(a.gxp32 + c - sx);
      const float4 gy = ld4(a.gyp32 + c), gym = ld4(a.gyp32 + c - sy);
      const float4 gz = ld4(a.gzp32 + c);
      const float gzm = a.gzp32[c - 1];
      float4 P, W;
      P.x = z.x + bc * p.x;
      P.y = z.y + bc * p.y;
      P.z = z.z + bc * p.z;
      P.w = z.w + bc * p.w;
      W.x = gym.x * (zym.x + bc * pym.x) + gxm.x * (zxm.x + bc * pxm.x) + gzm * pkm +
            dg.x * P.x + gz.x * P.y + gx.x * (zxp.x + bc * pxp.x) + gy.x * (zyp.x + bc * pyp.x);
      W.y = gym.y * (zym.y + bc * pym.y) + gxm.y * (zxm.y + bc * pxm.y) + gz.x * P.x +
            dg.y * P.y + gz.y * P.z + gx.y * (zxp.y + bc * pxp.y) + gy.y * (zyp.y + bc * pyp.y);
      W.z = gym.z * (zym.z + bc * pym.z) + gxm.z * (zxm.z + bc * pxm.z) + gz.y * P.y +
            dg.z * P.z + gz.z * P.w + gx.z * (zxp.z + bc * pxp.z) + gy.z * (zyp.z + bc * pyp.z);
      W.w = gym.w * (zym.w + bc * pym.w) + gxm.w * (zxm.w + bc * pxm.w) + gz.z * P.z +
            dg.w * P.w + gz.w * pkp + gx.w * (zxp.w + bc * pxp.w) + gy.w * (zyp.w + bc * pyp.w);
      st4(pnew + c, P);
      st4(a.w32 + c, W);
      if (!FIRST) {
        dd.x += pal * p.x;
        dd.y += pal * p.y;
        dd.z += pal * p.z;
        dd.w += pal * p.w;
        st4(a.d32 + c, dd);
      }
      pw += static_cast<double>(P.x) * W.x;
      pw += static_cast<double>(P.y) * W.y;
      pw += static_cast<double>(P.z) * W.z;
      pw += static_cast<double>(P.w) * W.w;
    }
  } else {
    auto pv = [&](long long m) { return FIRST ? a.z32[m] : a.z32[m] + bc * pold[m]; };
    for (long long c = t0; c < N; c += stride) {
      const float po = FIRST ? 0.0f : pold[c];
      const float dv = FIRST ? 0.0f : a.d32[c];
      const float pc = pv(c);
      float wv = a.gyp32[c - sy] * pv(c - sy);
      wv += a.gxp32[c - sx] * pv(c - sx);
      wv += a.gzp32[c - 1] * pv(c - 1);
      wv += a.diag32[c] * pc;
      wv += a.gzp32[c] * pv(c + 1);
      wv += a.gxp32[c] * pv(c + sx);
      wv += a.gyp32[c] * pv(c + sy);
      pnew[c] = pc;
      a.w32[c] = wv;
      if (!FIRST) a.d32[c] = dv + pal * po;
      pw += static_cast<double>(pc) * wv;
    }
  }
  return pw;
}

// E = 0: shared-memory tiled line solve; E > 0: warp-per-column solve with E
// cells per lane.
template <int V, int E>
__device__ __forceinline__ void cg_mixed_body(const MixedArgs& a, const int bid, const int G) {
  extern __shared__ float msm[];
  const Dims& d = a.d;
  const int nz = d.nz, nzp = nz + 1, tc = a.tc;
  float* s_r = msm;
  float* s_z = msm + tc * nzp;
  const long long N = d.ncell, sx = d.sx, sy = d.sy;
  const long long stride = static_cast<long long>(G) * blockDim.x;
  const long long t0 = bid * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long ntiles = (d.ncol + tc - 1) / tc;
  const int lane = threadIdx.x & 31;
  const bool vec = (E > 0) && (nz % (E > 0 ? E : 1) == 0);
  const long long gwarp = bid * static_cast<long long>(kCgBlock / 32) + (threadIdx.x >> 5);
  const long long nwarp = static_cast<long long>(G) * (kCgBlock / 32);
  double* const q0 = a.part;
  double* const q1 = a.part + G;
  double* const q2 = a.part + 2 * G;
  double* const q3 = a.part + 3 * G;

  // A warm start begins from the assembly's x0 = h^n; the outer test is
  // relative to ||b||, reduced here since the first residual is no longer b.
  double bb = 0.0;
  for (long long c = t0; c < N; c += stride) {
    if (a.warm) {
      const double bv = a.b[c];
      bb += bv * bv;
    } else {
      a.x0[c] = 0.0;
    }
    a.d32[c] = 0.0f;
  }
  if (a.warm) {
    const double s0 = block_sum_all(bb);
    if (threadIdx.x == 0) q3[bid] = s0;
  }
  if (!grid_sync(a.st, G)) return;

  double bnorm = 0.0, rnorm = 0.0;
  int total = 0, outer = 0, reason = 0, final_buf = 0;
  // The last inner iteration's update d += s_pal * p_(s_pbuf), applied by
  // the next phase A or outer pass (s_pal = 0: none).  Shared rather than
  // loop-carried registers: those spilled the 80-register budget of three
  // blocks per SM.  Thread 0 writes them only after a grid sync that follows
  // every read of the old values; the next reads follow another grid sync.
  __shared__ float s_pal;
  __shared__ int s_pbuf;
  if (threadIdx.x == 0) {
    s_pal = 0.0f;
    s_pbuf = 0;
  }
  __syncthreads();
  for (int o = 0;; ++o) {
    const float pal = s_pal;
    const float* __restrict__ pend = s_pbuf ? a.p1 : a.p0;
    const double* __restrict__ xo = (o & 1) ? a.x1 : a.x0;
    double* __restrict__ xn = (o & 1) ? a.x0 : a.x1;
    // Outer pass: x_new = x + d (with the pending update), r = b - A x_new
    // (FP64), r32, z = T^-1 r32.
    double rn2 = 0.0, zz = 0.0, zr = 0.0;
    if constexpr (E > 0) {
      for (long long col = gwarp; col < d.ncol; col += nwarp) {
        const long long cb = col * nz;
        const int k0 = lane * E;
        float rv[E], zv[E], lk[E], di[E];
        double xv[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          rv[e] = 0.0f;
          xv[e] = 0.0;
          if (k0 + e < nz) {
            const long long c = cb + k0 + e;
            const double rr = a.b[c] - outer_ax(a, xo, pend, pal, c, sx, sy);
            xv[e] = x_at(a, xo, pend, pal, c);
            rn2 += rr * rr;
            rv[e] = static_cast<float>(rr);
          }
        }
        ld_col<E>(a.l32, cb, lane, nz, vec, lk);
        ld_col<E>(a.dinv32, cb, lane, nz, vec, di);
        warp_column_solve<E>(lk, di, lane, nz, rv, zv);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          if (k0 + e < nz) {
            xn[cb + k0 + e] = xv[e];
            zz += static_cast<double>(zv[e]) * zv[e];
            zr += static_cast<double>(zv[e]) * rv[e];
          }
        }
        st_col<E>(a.r32, cb, lane, nz, vec, rv);
        st_col<E>(a.z32, cb, lane, nz, vec, zv);
      }
    } else {
    for (long long t = bid; t < ntiles; t += G) {
      const long long base = t * tc * nz;
      const int ncols = static_cast<int>((d.ncol - t * tc) < tc ? (d.ncol - t * tc) : tc);
      const int ncells = ncols * nz;
      for (int f = threadIdx.x; f < ncells; f += blockDim.x) {
        const long long c = base + f;
        const int col = f / nz, k = f - col * nz;
        const double rr = a.b[c] - outer_ax(a, xo, pend, pal, c, sx, sy);
        xn[c] = x_at(a, xo, pend, pal, c);
        rn2 += rr * rr;
        const float r32 = static_cast<float>(rr);
        a.r32[c] = r32;
        s_r[col * nzp + k] = r32;
      }
      __syncthreads();
      if (threadIdx.x < ncols) {
        const long long cb = base + static_cast<long long>(threadIdx.x) * nz;
        column_solve(s_r + threadIdx.x * nzp, a.dinv32 + cb, a.l32 + cb,
                     s_z + threadIdx.x * nzp, nz);
      }
      __syncthreads();
      for (int f = threadIdx.x; f < ncells; f += blockDim.x) {
        const long long c = base + f;
        const int col = f / nz, k = f - col * nz;
        const float z = s_z[col * nzp + k];
        a.z32[c] = z;
        zz += static_cast<double>(z) * z;
        zr += static_cast<double>(z) * s_r[col * nzp + k];
      }
      __syncthreads();
    }
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
    if (o == 0) bnorm = a.warm ? sqrt(reduce_partials(q3, G)) : rnorm;
    if (!isfinite(rnorm)) {
      reason = -9;
      break;
    }
    // A warm start always takes one correction, so that h^n itself, which
    // can meet the residual test, is never returned unrefined.
    if ((o > 0 || !a.warm) && rnorm <= fmax(a.outer_rtol * bnorm, a.atol)) {
      reason = (rnorm < a.atol) ? 3 : 2;
      break;
    }
    if (outer >= a.max_outer || total >= a.max_total) {
      reason = -3;
      break;
    }
    ++outer;
    if (threadIdx.x == 0) s_pal = 0.0f;  // the outer pass applied it
    for (long long c = t0; c < N; c += stride) a.d32[c] = 0.0f;
    // Inner FP32 PCG on A d = r32.
    // Each inner solve reduces its start by inner_rtol, the last one only as
    // far as the outer target needs (with a factor 2 of margin).
    const double need = (rnorm > 0.0) ? 0.5 * a.outer_rtol * bnorm / rnorm : a.inner_rtol;
    const double itol = fmax(a.inner_rtol, need) * zn0;
    double betaold = 1.0;
    for (int i = 0; i < a.max_inner && total < a.max_total; ++i) {
      if (beta == 0.0 || (i > 0 && beta * betaold <= 0.0)) break;
      const float bc = (i == 0) ? 0.0f : static_cast<float>(beta / betaold);
      const float* __restrict__ pold = (i & 1) ? a.p1 : a.p0;
      float* __restrict__ pnew = (i & 1) ? a.p0 : a.p1;
      const double pw = (i == 0) ? phase_a<V, true>(a, bc, pold, pnew, 0.0f, t0, stride)
                                 : phase_a<V, false>(a, bc, pold, pnew, s_pal, t0, stride);
      s = block_sum_all(pw);
      if (threadIdx.x == 0) q0[bid] = s;
      if (!grid_sync(a.st, G)) return;
      const double dpi = reduce_partials(q0, G);
      if (!(dpi > 0.0)) break;  // inner breakdown: keep d, the FP64 sweep decides
      const float al = static_cast<float>(beta / dpi);
      betaold = beta;
      ++total;
      if (threadIdx.x == 0) {  // d += al p_new, applied by the next phase A or outer pass
        s_pal = al;
        s_pbuf = (i & 1) ? 0 : 1;
      }
      zz = 0.0;
      zr = 0.0;
      if constexpr (E > 0) {
        for (long long col = gwarp; col < d.ncol; col += nwarp) {
          const long long cb = col * nz;
          const int k0 = lane * E;
          float wv[E], rv[E], lk[E], di[E], zv[E];
          ld_col<E>(a.w32, cb, lane, nz, vec, wv);
          ld_col<E>(a.r32, cb, lane, nz, vec, rv);
          ld_col<E>(a.l32, cb, lane, nz, vec, lk);
          ld_col<E>(a.dinv32, cb, lane, nz, vec, di);
#pragma unroll
          for (int e = 0; e < E; ++e) rv[e] -= al * wv[e];
          warp_column_solve<E>(lk, di, lane, nz, rv, zv);
          st_col<E>(a.r32, cb, lane, nz, vec, rv);
          st_col<E>(a.z32, cb, lane, nz, vec, zv);
#pragma unroll
          for (int e = 0; e < E; ++e) {
            if (k0 + e < nz) {
              zz += static_cast<double>(zv[e]) * zv[e];
              zr += static_cast<double>(zv[e]) * rv[e];
            }
          }
        }
      } else {
      for (long long t = bid; t < ntiles; t += G) {
        const long long base = t * tc * nz;
        const int ncols = static_cast<int>((d.ncol - t * tc) < tc ? (d.ncol - t * tc) : tc);
        const int ncells = ncols * nz;
        if constexpr (V == 4) {
          for (int f = 4 * threadIdx.x; f < ncells; f += 4 * blockDim.x) {
            const long long c = base + f;
            const int col = f / nz, k = f - col * nz;
            const float4 w = ld4(a.w32 + c);
            float4 r = ld4(a.r32 + c);
            r.x -= al * w.x;
            r.y -= al * w.y;
            r.z -= al * w.z;
            r.w -= al * w.w;
            st4(a.r32 + c, r);
            float* sr = s_r + col * nzp + k;
            sr[0] = r.x;
            sr[1] = r.y;
            sr[2] = r.z;
            sr[3] = r.w;
          }
        } else {
          for (int f = threadIdx.x; f < ncells; f += blockDim.x) {
            const long long c = base + f;
            const int col = f / nz, k = f - col * nz;
            const float r = a.r32[c] - al * a.w32[c];
            a.r32[c] = r;
            s_r[col * nzp + k] = r;
          }
        }
        __syncthreads();
        if (threadIdx.x < ncols) {
          const long long cb = base + static_cast<long long>(threadIdx.x) * nz;
          column_solve(s_r + threadIdx.x * nzp, a.dinv32 + cb, a.l32 + cb,
                       s_z + threadIdx.x * nzp, nz);
        }
        __syncthreads();
        if constexpr (V == 4) {
          for (int f = 4 * threadIdx.x; f < ncells; f += 4 * blockDim.x) {
            const long long c = base + f;
            const int col = f / nz, k = f - col * nz;
            const float* sz = s_z + col * nzp + k;
            const float* sr = s_r + col * nzp + k;
            const float4 z = make_float4(sz[0], sz[1], sz[2], sz[3]);
            st4(a.z32 + c, z);
            zz += static_cast<double>(z.x) * z.x + static_cast<double>(z.y) * z.y +
                  static_cast<double>(z.z) * z.z + static_cast<double>(z.w) * z.w;
            zr += static_cast<double>(z.x) * sr[0] + static_cast<double>(z.y) * sr[1] +
                  static_cast<double>(z.z) * sr[2] + static_cast<double>(z.w) * sr[3];
          }
        } else {
          for (int f = threadIdx.x; f < ncells; f += blockDim.x) {
            const long long c = base + f;
            const int col = f / nz, k = f - col * nz;
            const float z = s_z[col * nzp + k];
            a.z32[c] = z;
            zz += static_cast<double>(z) * z;
            zr += static_cast<double>(z) * s_r[col * nzp + k];
          }
        }
        __syncthreads();
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

// Blocks per SM of the mixed solves: as many as fit without register spills
// (three; two for 8 cells per lane and for the batched forms, whose member
// records add registers).  At four the 64-register cap spilled 126 bytes a
// thread and the 512x512x128 solve ran 5 % slower (12.5 against 11.8 ms).
template <int V, int E>
constexpr int mixed_min_blocks(bool batch) {
  return (E == 8 || (batch && (V == 4 || E == 8))) ? 2 : 3;
}

template <int V, int E>
__global__ void __launch_bounds__(kCgBlock, mixed_min_blocks<V, E>(false)) k_cg_mixed(MixedArgs a) {
  cg_mixed_body<V, E>(a, blockIdx.x, gridDim.x);
}

// One cooperative launch over several domains of every (V, E) class:
// instance i owns first[i+1] - first[i] block slots and runs its own solve in
// its class's form (`variant`); the blocks take the slots from `queue` in
// queue order (as k_cg64_batch).  One launch for all classes, so the classes
// share the device instead of following one another; the dynamic shared
// memory is the largest any member needs.
template <int V>
__device__ __forceinline__ void cg_mixed_any(const MixedArgs& a, int e, int sb, int sg) {
  switch (e) {
    case 0: cg_mixed_body<V, 0>(a, sb, sg); break;
    case 1: cg_mixed_body<V, 1>(a, sb, sg); break;
    case 2: cg_mixed_body<V, 2>(a, sb, sg); break;
    case 4: cg_mixed_body<V, 4>(a, sb, sg); break;
    default: cg_mixed_body<V, 8>(a, sb, sg); break;
  }
}

__global__ void __launch_bounds__(kCgBlock, 2)
    k_cg_mixed_batch(const MixedArgs* __restrict__ tab, const int* __restrict__ first, int n,
                     int* queue, const int* __restrict__ order, const int* __restrict__ ofirst) {
  __shared__ MixedArgs sa;
  __shared__ int sb, sg, slot;
  for (;;) {
    if (threadIdx.x == 0) {
      slot = atomicAdd(queue, 1);
      if (slot < first[n]) {
        const int q = instance_of(ofirst, n, slot);
        const int i = order[q];
        sa = tab[i];
        sb = slot - ofirst[q];
        sg = first[i + 1] - first[i];
      }
    }
    __syncthreads();
    if (slot >= first[n]) break;
    if (sa.variant / 16 == 4) {
      cg_mixed_any<4>(sa, sa.variant % 16, sb, sg);
    } else {
      cg_mixed_any<1>(sa, sa.variant % 16, sb, sg);
    }
    __syncthreads();  // every thread is done with sa before the next slot's
  }
}

int host_tile_cols(int nz) {
  int tc = kTileCells / nz;
  if (tc < 1) tc = 1;
  if (tc > 64) tc = 64;
  return tc;
}

size_t mixed_smem(int nz) { return 2 * sizeof(float) * host_tile_cols(nz) * (nz + 1); }
size_t factor_smem(int nz) {
  return factor_lane_cells(nz) ? 0 : 2 * sizeof(double) * host_tile_cols(nz) * (nz + 1);
}

MixedArgs make_mixed_args(const Device& D, double atol, int maxit, double outer_rtol,
                          int max_outer) {
  const int tc = host_tile_cols(D.d.nz);
  MixedArgs a;
  a.d = D.d;
  a.diag = D.diag;
  a.gxp = D.gxp;
  a.gyp = D.gyp;
  a.gzp = D.gzp;
  a.b = D.rhs;
  a.x0 = D.x;
  a.x1 = D.xalt;
  a.diag32 = D.diag32;
  a.gxp32 = D.gxp32;
  a.gyp32 = D.gyp32;
  a.gzp32 = D.gzp32;
  a.dinv32 = D.dinv32;
  a.l32 = D.l32;
  a.r32 = D.r32;
  a.z32 = D.z32;
  a.p0 = D.p032;
  a.p1 = D.p132;
  a.w32 = D.w32;
  a.d32 = D.d32;
  a.part = D.cgpart;
  a.st = &D.out->cg;
  a.outer_rtol = outer_rtol;
  // Reduction asked of every inner solve but the last: 1e-4 minimised the
  // total inner iterations of the two corrections on slab crops (96^2 and
  // 128^2 x 128 systems: 22, 24, 18 against 24, 26, 20 at 1e-5).
  a.inner_rtol = 1.0e-4;
  a.atol = atol;
  a.max_inner = maxit;
  a.max_outer = max_outer;
  a.max_total = maxit;
  a.tc = tc;
  a.warm = 1;
  return a;
}

}  // namespace

int cg32_grid(int sm_count, long long ncell) {
  (void)ncell;
  return sm_count;  // refined per domain in launch_cg_mixed (depends on nz)
}

cudaError_t launch_line_factor(Device& D) {
  const int nz = D.d.nz;
  const int fe = factor_lane_cells(nz);
  if (fe) {
    const int fgrid = line_factor_blocks(D);
    auto k = fe == 1 ? k_line_factor_warp<1> : fe == 2 ? k_line_factor_warp<2>
           : fe == 4 ? k_line_factor_warp<4> : k_line_factor_warp<8>;
    k<<<fgrid, kFactorBlock, 0, D.stream>>>(D.d, D.diag, D.gxp, D.gyp, D.gzp, D.diag32, D.gxp32,
                                            D.gyp32, D.gzp32, D.dinv32, D.l32);
    ++D.launches;
    return cudaGetLastError();
  }
  const size_t fsm = factor_smem(nz);
  const cudaError_t ea = raise_smem_limit(reinterpret_cast<const void*>(k_line_factor), fsm);
  if (ea != cudaSuccess) return ea;
  const int tc = host_tile_cols(nz);
  const int fgrid = line_factor_blocks(D);
  k_line_factor<<<fgrid, kFactorBlock, fsm, D.stream>>>(D.d, D.diag, D.gxp, D.gyp, D.gzp,
                                                        D.diag32, D.gxp32, D.gyp32, D.gzp32,
                                                        D.dinv32, D.l32, tc);
  ++D.launches;
  return cudaGetLastError();
}

cudaError_t launch_cg_mixed(Device& D, double rtol, double atol, int maxit, double outer_rtol,
                            int max_outer) {
  (void)rtol;
  const int nz = D.d.nz;
  if (host_tile_cols(nz) * nz > kTileCells && nz > kTileCells) return cudaErrorInvalidValue;
  const size_t msm = mixed_smem(nz);
  const bool vec = (nz % 4 == 0);
  const bool wcol = nz <= 32 * kMaxE;
  const int ecol = !wcol ? 0 : nz <= 32 ? 1 : nz <= 64 ? 2 : nz <= 128 ? 4 : 8;
  using Kern = void (*)(MixedArgs);
  static const Kern table[2][5] = {
      {k_cg_mixed<1, 0>, k_cg_mixed<1, 1>, k_cg_mixed<1, 2>, k_cg_mixed<1, 4>, k_cg_mixed<1, 8>},
      {k_cg_mixed<4, 0>, k_cg_mixed<4, 1>, k_cg_mixed<4, 2>, k_cg_mixed<4, 4>, k_cg_mixed<4, 8>}};
  const int slot = ecol == 0 ? 0 : ecol == 1 ? 1 : ecol == 2 ? 2 : ecol == 4 ? 3 : 4;
  const void* kern = reinterpret_cast<const void*>(table[vec ? 1 : 0][slot]);
  const size_t ksm = wcol ? 0 : msm;
  if (!wcol)
    raise_smem_limit(kern, msm);
  const int tc = host_tile_cols(nz);
  const long long ntiles = (D.d.ncol + tc - 1) / tc;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCgBlock, ksm);
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  // 3 x g reduction partials fit the 4 x sm_count x 4 doubles allocated at create.
  if (per_sm > 4) per_sm = 4;
  long long g = static_cast<long long>(per_sm) * D.sm_count;
  if (!wcol && g > ntiles) g = ntiles;
  if (g < 1) g = 1;
  cudaMemsetAsync(&D.out->cg, 0, sizeof(CgState), D.stream);
  MixedArgs a = make_mixed_args(D, atol, maxit, outer_rtol, max_outer);
  void* args[] = {&a};
  ++D.launches;
  D.cg_grid32 = static_cast<int>(g);
  return cudaLaunchCooperativeKernel(kern, dim3(g), dim3(kCgBlock), args, ksm, D.stream);
}


// ---------------------------------------------------------------- batched solves
namespace {

// Line-solve layout of a column depth: E cells per lane (warp per column,
// nz <= 32 E) or 0 (shared-memory tiles).
int line_e(int nz, bool tiled) {
  if (tiled || nz > 32 * kMaxE) return 0;
  return nz <= 32 ? 1 : nz <= 64 ? 2 : nz <= 128 ? 4 : 8;
}

}  // namespace

int mixed_variant(const Device& D, bool tiled) {
  const int v = (D.d.nz % 4 == 0) ? 4 : 1;
  return v * 16 + line_e(D.d.nz, tiled);
}

size_t mixed_args_bytes() { return sizeof(MixedArgs); }

void mixed_fill_args(const Device& D, const SolveParams& p, int variant, void* dst) {
  MixedArgs a = make_mixed_args(D, p.atol, p.maxit, p.outer_rtol, p.max_outer);
  a.variant = variant;
  std::memcpy(dst, &a, sizeof(a));
}

size_t mixed_batch_smem(const Device& D, int variant) {
  return (variant % 16 == 0) ? mixed_smem(D.d.nz) : 0;
}

const void* mixed_batch_kernel() { return reinterpret_cast<const void*>(k_cg_mixed_batch); }

// ---------------------------------------------------------------- batched line factor
namespace {

__global__ void __launch_bounds__(kFactorBlock) k_line_factor_batch(const StepArgs* tab,
                                                                    const int* first, int n) {
  __shared__ StepArgs sa;
  __shared__ int si;
  if (threadIdx.x == 0) si = instance_of(first, n, blockIdx.x);
  __syncthreads();
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(tab + si);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sa);
  for (int w = threadIdx.x; w < static_cast<int>(sizeof(StepArgs) / 8); w += blockDim.x)
    dst[w] = src[w];
  const int bid = blockIdx.x - first[si], G = first[si + 1] - first[si];
  __syncthreads();
  switch (factor_lane_cells(sa.d.nz)) {
    case 1:
      line_factor_warp_body<1>(sa.d, sa.diag, sa.gxp, sa.gyp, sa.gzp, sa.diag32, sa.gxp32,
                               sa.gyp32, sa.gzp32, sa.dinv32, sa.l32, bid, G);
      break;
    case 2:
      line_factor_warp_body<2>(sa.d, sa.diag, sa.gxp, sa.gyp, sa.gzp, sa.diag32, sa.gxp32,
                               sa.gyp32, sa.gzp32, sa.dinv32, sa.l32, bid, G);
      break;
    case 4:
      line_factor_warp_body<4>(sa.d, sa.diag, sa.gxp, sa.gyp, sa.gzp, sa.diag32, sa.gxp32,
                               sa.gyp32, sa.gzp32, sa.dinv32, sa.l32, bid, G);
      break;
    case 8:
      line_factor_warp_body<8>(sa.d, sa.diag, sa.gxp, sa.gyp, sa.gzp, sa.diag32, sa.gxp32,
                               sa.gyp32, sa.gzp32, sa.dinv32, sa.l32, bid, G);
      break;
    default:
      line_factor_body(sa.d, sa.diag, sa.gxp, sa.gyp, sa.gzp, sa.diag32, sa.gxp32, sa.gyp32,
                       sa.gzp32, sa.dinv32, sa.l32, sa.tc, bid, G);
  }
}

}  // namespace

int line_tile_cols(int nz) { return host_tile_cols(nz); }

int line_factor_blocks(const Device& D) {
  if (factor_lane_cells(D.d.nz)) {  // one warp per column, kFactorBlock / 32 per block
    const long long per = kFactorBlock / 32;
    return static_cast<int>(std::min<long long>((D.d.ncol + per - 1) / per, 16LL * D.sm_count));
  }
  const int tc = host_tile_cols(D.d.nz);
  const long long ntiles = (D.d.ncol + tc - 1) / tc;
  return static_cast<int>(std::min<long long>(ntiles, 4LL * D.sm_count));
}

size_t line_factor_smem(int nz) { return factor_smem(nz); }

cudaError_t launch_line_factor_batch(const PhaseTables& t, cudaStream_t s) {
  const cudaError_t e =
      raise_smem_limit(reinterpret_cast<const void*>(k_line_factor_batch), t.factor_smem);
  if (e != cudaSuccess) return e;
  k_line_factor_batch<<<t.grid_factor, kFactorBlock, t.factor_smem, s>>>(t.tab, t.first_factor,
                                                                        t.n);
  return cudaGetLastError();
}

}  // namespace fgw
