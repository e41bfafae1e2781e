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

#include "gw_internal.h"

namespace fgw {

namespace {

constexpr int kCgBlock = 256;
constexpr long long kSpinLimit = 20000000LL;  // ~2-4 s of polling

__device__ inline unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ inline int ld_relaxed_int(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for a cooperative (co-resident) launch.  Returns false
// when the barrier gave up; the caller then leaves the kernel.
__device__ bool grid_sync(CgState* st, unsigned nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    if (ld_relaxed_int(&st->err) != 0) {
      good = 0;
    } else {
      const unsigned my = ld_acquire(&st->bar_gen);
      __threadfence();
      const unsigned arrived = atomicAdd(&st->bar_count, 1u) + 1u;
      if (arrived == nblocks) {
        atomicExch(&st->bar_count, 0u);
        __threadfence();
        atomicAdd(&st->bar_gen, 1u);
      } else {
        long long spins = 0;
        while (ld_acquire(&st->bar_gen) == my) {
          if (++spins > kSpinLimit || ld_relaxed_int(&st->err) != 0) {
            atomicExch(&st->err, 1);
            good = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block sum; result broadcast to every thread.
__device__ double block_sum_all(double v) {
  __shared__ double sh[32];
  __shared__ double res;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
    v = warp_sum(v);
    if (lane == 0) res = v;
  }
  __syncthreads();
  const double out = res;
  __syncthreads();
  return out;
}

// Sum of the G per-block partials, identical in every block.
__device__ double reduce_partials(const double* part, int G) {
  double v = 0.0;
  for (int b = threadIdx.x; b < G; b += blockDim.x) v += part[b];
  return block_sum_all(v);
}

struct Cg64Args {
  Dims d;
  const double *diag, *gxp, *gyp, *gzp, *b;
  double *x, *r, *z, *p0, *p1, *w;
  double* part;  // 3 x G
  CgState* st;
  double rtol, atol;
  int maxit;
};

__device__ inline int sgn(double v) { return (v > 0.0) - (v < 0.0); }

__global__ void __launch_bounds__(kCgBlock, 3) k_cg64(Cg64Args a) {
  const long long N = a.d.ncell, sx = a.d.sx, sy = a.d.sy;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long t0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const int G = gridDim.x;
  double* const pzz = a.part;
  double* const pzr = a.part + G;
  double* const ppw = a.part + 2 * G;

  // r = b, x = 0, p = 0, z = D^-1 r; partial z'z, z'r.
  double zz = 0.0, zr = 0.0;
  for (long long c = t0; c < N; c += stride) {
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
  double s = block_sum_all(zz);
  if (threadIdx.x == 0) pzz[blockIdx.x] = s;
  s = block_sum_all(zr);
  if (threadIdx.x == 0) pzr[blockIdx.x] = s;
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
    // Phase A: direction update fused into the stencil product.
    double pw = 0.0;
    for (long long c = t0; c < N; c += stride) {
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
    s = block_sum_all(pw);
    if (threadIdx.x == 0) ppw[blockIdx.x] = s;
    if (!grid_sync(a.st, G)) return;
    dpiold = dpi;
    dpi = reduce_partials(ppw, G);
    betaold = beta;
    if (dpi == 0.0 || (i > 0 && sgn(dpi) * sgn(dpiold) < 0)) {
      reason = -10;
      break;
    }
    const double al = beta / dpi;
    // Phase B: update and precondition.
    zz = 0.0;
    zr = 0.0;
    for (long long c = t0; c < N; c += stride) {
      const double pc = pnew[c];
      a.x[c] += al * pc;
      const double rc = a.r[c] - al * a.w[c];
      a.r[c] = rc;
      const double z = rc * (1.0 / a.diag[c]);
      a.z[c] = z;
      zz += z * z;
      zr += z * rc;
    }
    s = block_sum_all(zz);
    if (threadIdx.x == 0) pzz[blockIdx.x] = s;
    s = block_sum_all(zr);
    if (threadIdx.x == 0) pzr[blockIdx.x] = s;
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
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.st->dp = dp;
    a.st->rnorm0 = rnorm0;
    a.st->its = its;
    a.st->reason = reason;
    a.st->outer = 1;
  }
}

}  // namespace

int cg64_grid(int sm_count, long long ncell) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg64, kCgBlock, 0);
  if (per_sm < 1) per_sm = 1;
  const long long want = (ncell + kCgBlock - 1) / kCgBlock;
  long long g = static_cast<long long>(per_sm) * sm_count;
  if (want < g) g = want;
  return static_cast<int>(g < 1 ? 1 : g);
}

cudaError_t launch_cg64(Device& D, double rtol, double atol, int maxit) {
  cudaMemsetAsync(&D.out->cg, 0, sizeof(CgState), D.stream);
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
  void* args[] = {&a};
  ++D.launches;
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_cg64), dim3(D.cg_grid),
                                     dim3(kCgBlock), args, 0, D.stream);
}

int cg32_grid(int sm_count, long long ncell) { return cg64_grid(sm_count, ncell); }

cudaError_t launch_cg_mixed(Device& D, double rtol, double atol, int maxit, double outer_rtol,
                            int max_outer) {
  (void)D;
  (void)rtol;
  (void)atol;
  (void)maxit;
  (void)outer_rtol;
  (void)max_outer;
  return cudaErrorNotSupported;
}

}  // namespace fgw
