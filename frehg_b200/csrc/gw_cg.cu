// The predictor's linear solve on the B200: Jacobi-preconditioned conjugate
// gradients on the matrix-free 7-point head system, with the algorithm and
// stopping rule of PETSc's KSPCG as the reference configures it
// (src/core/LinearSystem.cpp:147-151, -gw_pc_type jacobi lane): x0 = 0,
// z = r .* (1 / diag), Hestenes-Stiefel recurrences beta = z'r,
// p = z + (beta / beta_old) p, alpha = beta / p'Ap, convergence on the
// preconditioned norm ||z|| <= max(rtol ||D^-1 b||, atol), divergence at
// 1e5 ||D^-1 b||, non-finite norms, indefinite matrix / preconditioner and
// max_iterations.
//
// One persistent cooperative launch runs the whole solve.  Per iteration:
//   phase A: p_new = z + b p_old (for the seven stencil points), w = A p_new,
//            partial p'w;
//   grid barrier; every block reduces the partials in block order;
//   phase B: x += a p, r -= a w, z = r / diag, partials z'z and z'r;
//   grid barrier; reduction; convergence test.
// Every thread takes two consecutive cells (cg64v_body), with 16-byte pair
// loads where nz is even and separate loads where it is odd.
// Per cell and iteration this moves 16 FP64 words (128 B) through HBM:
// phase A reads z, p_old, diag, gxp, gyp, gzp and writes p_new, w; phase B
// reads x, p_new, r, w, diag and writes x, r, z.  Neighbour reads are served
// by L1/L2 because the grid-stride sweep keeps all resident blocks inside a
// few j-rows of each other.
//
// The grid barrier is a bounded spin on a generation counter: a wait that
// exceeds kSpinLimit polls sets CgState::err, and every block leaves at its
// next barrier, so a launch that lost co-residency ends with an error status
// instead of hanging.
#include <cfloat>
#include <cstdio>
#include <cstring>

#include "gw_coop.cuh"
#include "gw_internal.h"

namespace fgw {

namespace {

using namespace coop;

struct Cg64Args {
  Dims d;
  const double *diag, *gxp, *gyp, *gzp, *b;
  double *x, *r, *z, *p0, *p1, *w;
  double* part;  // 3 x G
  CgState* st;
  double rtol, atol;
  int maxit;
  int variant;  // batched solves: 1 = 16-byte pair accesses (nz even), 0 = separate loads
};

__device__ inline int sgn(double v) { return (v > 0.0) - (v < 0.0); }

// The same solve with two consecutive cells per thread.  With ALIGNED (nz
// even, so every pair and every i/j-neighbour pair is 16-byte aligned) the
// pairs move as 16-byte loads and stores: half the load instructions per cell
// and twice the bytes in flight per request.  Otherwise (nz odd) the pair's
// two cells load separately, still two cells' loads in flight per thread, and
// an odd cell count leaves a last cell that one thread takes alone.  The
// arithmetic per cell is the one-cell-per-thread form's (cg64_cell_*, which
// also take that last cell); against it, the separate-load pairs took a
// 256x256x127 solve from 95.4 to 57 ms.
__device__ inline double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ inline void st2(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
template <bool ALIGNED>
__device__ inline double2 ldp(const double* p) {
  if constexpr (ALIGNED) {
    return ld2(p);
  } else {
    return make_double2(p[0], p[1]);
  }
}
template <bool ALIGNED>
__device__ inline void stp(double* p, double a, double b) {
  if constexpr (ALIGNED) {
    st2(p, a, b);
  } else {
    p[0] = a;
    p[1] = b;
  }
}

// The three per-cell steps of one cell alone (the order of terms of the pair
// code), for the last cell of an odd count.
__device__ inline void cg64_cell_init(const Cg64Args& a, long long c, double& zz, double& zr) {
  const double rc = a.b[c];
  a.x[c] = 0.0;
  a.r[c] = rc;
  a.p0[c] = 0.0;
  a.p1[c] = 0.0;
  const double z = rc * (1.0 / a.diag[c]);
  a.z[c] = z;
  zz += z * z;
  zr += z * rc;
}
__device__ inline void cg64_cell_stencil(const Cg64Args& a, long long c, double bc,
                                         const double* __restrict__ pold,
                                         double* __restrict__ pnew, double& pw) {
  const long long sx = a.d.sx, sy = a.d.sy;
  const double pc = a.z[c] + bc * pold[c];
  const double pym = a.z[c - sy] + bc * pold[c - sy];
  const double pxm = a.z[c - sx] + bc * pold[c - sx];
  const double pzm = a.z[c - 1] + bc * pold[c - 1];
  const double pzp = a.z[c + 1] + bc * pold[c + 1];
  const double pxp = a.z[c + sx] + bc * pold[c + sx];
  const double pyp = a.z[c + sy] + bc * pold[c + sy];
  double wv = a.gyp[c - sy] * pym;
  wv += a.gxp[c - sx] * pxm;
  wv += a.gzp[c - 1] * pzm;
  wv += a.diag[c] * pc;
  wv += a.gzp[c] * pzp;
  wv += a.gxp[c] * pxp;
  wv += a.gyp[c] * pyp;
  pnew[c] = pc;
  a.w[c] = wv;
  pw += pc * wv;
}
__device__ inline void cg64_cell_update(const Cg64Args& a, long long c, double al,
                                        const double* __restrict__ pnew, double& zz,
                                        double& zr) {
  const double pc = pnew[c];
  a.x[c] += al * pc;
  const double rc = a.r[c] - al * a.w[c];
  a.r[c] = rc;
  const double z = rc * (1.0 / a.diag[c]);
  a.z[c] = z;
  zz += z * z;
  zr += z * rc;
}

template <bool ALIGNED>
__device__ __forceinline__ void cg64v_body(const Cg64Args& a, const int bid, const int G) {
  const long long N2 = a.d.ncell / 2, sx = a.d.sx, sy = a.d.sy;
  // The last cell of an odd count, taken by the grid's last thread.
  const bool tail = !ALIGNED && (a.d.ncell & 1) && bid == G - 1 &&
                    threadIdx.x == blockDim.x - 1;
  const long long ct = a.d.ncell - 1;
  const long long stride = static_cast<long long>(G) * blockDim.x;
  const long long t0 = bid * static_cast<long long>(blockDim.x) + threadIdx.x;
  double* const pzz = a.part;
  double* const pzr = a.part + G;
  double* const ppw = a.part + 2 * G;

  double zz = 0.0, zr = 0.0;
  for (long long q = t0; q < N2; q += stride) {
    const long long c = 2 * q;
    const double2 rc = ldp<ALIGNED>(a.b + c);
    const double2 dg = ldp<ALIGNED>(a.diag + c);
    stp<ALIGNED>(a.x + c, 0.0, 0.0);
    stp<ALIGNED>(a.r + c, rc.x, rc.y);
    stp<ALIGNED>(a.p0 + c, 0.0, 0.0);
    stp<ALIGNED>(a.p1 + c, 0.0, 0.0);
    const double z0 = rc.x * (1.0 / dg.x), z1 = rc.y * (1.0 / dg.y);
    stp<ALIGNED>(a.z + c, z0, z1);
    zz += z0 * z0;
    zz += z1 * z1;
    zr += z0 * rc.x;
    zr += z1 * rc.y;
  }
  if (tail) cg64_cell_init(a, ct, zz, zr);
  double s = block_sum_all(zz);
  if (threadIdx.x == 0) pzz[bid] = s;
  s = block_sum_all(zr);
  if (threadIdx.x == 0) pzr[bid] = s;
  if (!grid_sync(a.st, G)) return;
  double dp = sqrt(reduce_partials(pzz, G));
  double beta = reduce_partials(pzr, G);
  const double rnorm0 = dp;
  const double ttol = fmax(a.rtol * rnorm0, a.atol);
  int reason = 0, its = 0;
  const auto test = [&](double rn) {
    if (!isfinite(rn)) reason = -9;
    else if (rn <= ttol) reason = (rn < a.atol) ? 3 : 2;
    else if (rn >= 1.0e5 * rnorm0) reason = -4;
  };
  test(dp);
  double betaold = 1.0, dpi = 0.0, dpiold = 0.0;
  int i = 0;
  while (reason == 0) {
    its = i + 1;
    if (beta == 0.0) {
      reason = 3;
      break;
    }
    if (i > 0 && beta * betaold < 0.0) {
      reason = -8;
      break;
    }
    const double bc = (i == 0) ? 0.0 : beta / betaold;
    const double* __restrict__ pold = (i & 1) ? a.p1 : a.p0;
    double* __restrict__ pnew = (i & 1) ? a.p0 : a.p1;
    double pw = 0.0;
    for (long long q = t0; q < N2; q += stride) {
      const long long c = 2 * q;
      const double2 zc = ldp<ALIGNED>(a.z + c), pc = ldp<ALIGNED>(pold + c);
      const double2 zxm = ldp<ALIGNED>(a.z + c - sx), pxm = ldp<ALIGNED>(pold + c - sx);
      const double2 zxp = ldp<ALIGNED>(a.z + c + sx), pxp = ldp<ALIGNED>(pold + c + sx);
      const double2 zym = ldp<ALIGNED>(a.z + c - sy), pym = ldp<ALIGNED>(pold + c - sy);
      const double2 zyp = ldp<ALIGNED>(a.z + c + sy), pyp = ldp<ALIGNED>(pold + c + sy);
      const double zkm = a.z[c - 1], pkm = pold[c - 1];
      const double zkp = a.z[c + 2], pkp = pold[c + 2];
      const double2 dg = ldp<ALIGNED>(a.diag + c);
      const double2 gx = ldp<ALIGNED>(a.gxp + c), gxm = ldp<ALIGNED>(a.gxp + c - sx);
      const double2 gy = ldp<ALIGNED>(a.gyp + c), gym = ldp<ALIGNED>(a.gyp + c - sy);
      const double2 gz = ldp<ALIGNED>(a.gzp + c);
      const double gzm = a.gzp[c - 1];
      const double P0 = zc.x + bc * pc.x, P1 = zc.y + bc * pc.y;
      const double Pkm = zkm + bc * pkm, Pkp = zkp + bc * pkp;
      const double Pxm0 = zxm.x + bc * pxm.x, Pxm1 = zxm.y + bc * pxm.y;
      const double Pxp0 = zxp.x + bc * pxp.x, Pxp1 = zxp.y + bc * pxp.y;
      const double Pym0 = zym.x + bc * pym.x, Pym1 = zym.y + bc * pym.y;
      const double Pyp0 = zyp.x + bc * pyp.x, Pyp1 = zyp.y + bc * pyp.y;
      double w0 = gym.x * Pym0;
      w0 += gxm.x * Pxm0;
      w0 += gzm * Pkm;
      w0 += dg.x * P0;
      w0 += gz.x * P1;
      w0 += gx.x * Pxp0;
      w0 += gy.x * Pyp0;
      double w1 = gym.y * Pym1;
      w1 += gxm.y * Pxm1;
      w1 += gz.x * P0;
      w1 += dg.y * P1;
      w1 += gz.y * Pkp;
      w1 += gx.y * Pxp1;
      w1 += gy.y * Pyp1;
      stp<ALIGNED>(pnew + c, P0, P1);
      stp<ALIGNED>(a.w + c, w0, w1);
      pw += P0 * w0;
      pw += P1 * w1;
    }
    if (tail) cg64_cell_stencil(a, ct, bc, pold, pnew, pw);
    s = block_sum_all(pw);
    if (threadIdx.x == 0) ppw[bid] = s;
    if (!grid_sync(a.st, G)) return;
    dpiold = dpi;
    dpi = reduce_partials(ppw, G);
    betaold = beta;
    if (dpi == 0.0 || (i > 0 && sgn(dpi) * sgn(dpiold) < 0)) {
      reason = -10;
      break;
    }
    const double al = beta / dpi;
    zz = 0.0;
    zr = 0.0;
    for (long long q = t0; q < N2; q += stride) {
      const long long c = 2 * q;
      const double2 pc = ldp<ALIGNED>(pnew + c), xc = ldp<ALIGNED>(a.x + c), rc0 = ldp<ALIGNED>(a.r + c);
      const double2 wc = ldp<ALIGNED>(a.w + c), dg = ldp<ALIGNED>(a.diag + c);
      stp<ALIGNED>(a.x + c, xc.x + al * pc.x, xc.y + al * pc.y);
      const double r0 = rc0.x - al * wc.x, r1 = rc0.y - al * wc.y;
      stp<ALIGNED>(a.r + c, r0, r1);
      const double z0 = r0 * (1.0 / dg.x), z1 = r1 * (1.0 / dg.y);
      stp<ALIGNED>(a.z + c, z0, z1);
      zz += z0 * z0;
      zz += z1 * z1;
      zr += z0 * r0;
      zr += z1 * r1;
    }
    if (tail) cg64_cell_update(a, ct, al, pnew, zz, zr);
    s = block_sum_all(zz);
    if (threadIdx.x == 0) pzz[bid] = s;
    s = block_sum_all(zr);
    if (threadIdx.x == 0) pzr[bid] = s;
    if (!grid_sync(a.st, G)) return;
    dp = sqrt(reduce_partials(pzz, G));
    test(dp);
    if (reason != 0) break;
    beta = reduce_partials(pzr, G);
    ++i;
    if (i >= a.maxit) {
      reason = -3;
      break;
    }
  }
  if (bid == 0 && threadIdx.x == 0) {
    a.st->dp = dp;
    a.st->rnorm0 = rnorm0;
    a.st->its = its;
    a.st->reason = reason;
    a.st->outer = 1;
  }
}

// Two blocks per SM: at three the 80-register cap spilled (24 bytes a thread)
// and the 512x512x128 FP64 solve took 251 ms against 236.
__global__ void __launch_bounds__(kCgBlock, 2) k_cg64v(Cg64Args a) {
  cg64v_body<true>(a, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(kCgBlock, 2) k_cg64u(Cg64Args a) {
  cg64v_body<false>(a, blockIdx.x, gridDim.x);
}

// One cooperative launch over several domains: instance i owns
// first[i+1] - first[i] block slots and runs its own solve on them, in the
// paired or the separate-load two-cell form by its `variant`; each block takes the next
// slot from `queue` (zeroed before the launch) until all are handed out, the
// instances' slots in queue order (`order`, slot offsets `ofirst`), so a
// block whose instance has converged goes on to a waiting instance.  The
// slot's index within its instance, not the block, fixes the block's share
// of the instance's cells.
__global__ void __launch_bounds__(kCgBlock, 3)
    k_cg64_batch(const Cg64Args* __restrict__ tab, const int* __restrict__ first, int n,
                 int* queue, const int* __restrict__ order, const int* __restrict__ ofirst) {
  __shared__ Cg64Args sa;
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
    if (sa.variant) {
      cg64v_body<true>(sa, sb, sg);
    } else {
      cg64v_body<false>(sa, sb, sg);
    }
    __syncthreads();  // every thread is done with sa before the next slot's
  }
}

}  // namespace

int cg64_grid(int sm_count, long long ncell) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg64u, kCgBlock, 0);
  int per_sm_v = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_v, k_cg64v, kCgBlock, 0);
  if (per_sm_v < per_sm) per_sm = per_sm_v;
  if (per_sm < 1) per_sm = 1;
  const long long want = (ncell + kCgBlock - 1) / kCgBlock;
  long long g = static_cast<long long>(per_sm) * sm_count;
  if (want < g) g = want;
  return static_cast<int>(g < 1 ? 1 : g);
}

namespace {

Cg64Args make_cg64_args(const Device& D, double rtol, double atol, int maxit) {
  Cg64Args a;
  a.d = D.d;
  a.diag = D.diag;
  a.gxp = D.gxp;
  a.gyp = D.gyp;
  a.gzp = D.gzp;
  a.b = D.rhs;
  a.x = D.x;
  a.r = D.r;
  a.z = D.z;
  a.p0 = D.p0;
  a.p1 = D.p1;
  a.w = D.w;
  a.part = D.cgpart;
  a.st = &D.out->cg;
  a.rtol = rtol;
  a.atol = atol;
  a.maxit = maxit;
  return a;
}

}  // namespace

cudaError_t launch_cg64(Device& D, double rtol, double atol, int maxit) {
  cudaMemsetAsync(&D.out->cg, 0, sizeof(CgState), D.stream);
  Cg64Args a = make_cg64_args(D, rtol, atol, maxit);
  void* args[] = {&a};
  ++D.launches;
  const void* kern = (D.d.nz % 2 == 0) ? reinterpret_cast<const void*>(k_cg64v)
                                       : reinterpret_cast<const void*>(k_cg64u);
  return cudaLaunchCooperativeKernel(kern, dim3(D.cg_grid), dim3(kCgBlock), args, 0, D.stream);
}

size_t cg64_args_bytes() { return sizeof(Cg64Args); }

void cg64_fill_args(const Device& D, const SolveParams& p, int variant, void* dst) {
  Cg64Args a = make_cg64_args(D, p.rtol, p.atol, p.maxit);
  a.variant = variant;
  std::memcpy(dst, &a, sizeof(a));
}

const void* cg64_batch_kernel() { return reinterpret_cast<const void*>(k_cg64_batch); }

}  // namespace fgw
