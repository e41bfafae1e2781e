// The per-column LDL^T factorization of the mixed solve's line
// preconditioner, one warp per column (nz <= 256): shared by the separate
// factor pass (gw_cg_mixed.cu) and the fused predictor (gw_kernels.cu), so
// both produce the same bits.
//
// Lane `lane` holds the E consecutive cells k = lane * E + e.  The pivot
// recurrence d_k = a_k - e_{k-1}^2 / d_{k-1} (a = diag, e = gzp) is the
// Moebius map of the matrix M_k = [[a_k, -e_{k-1}^2], [1, 0]] acting on
// (numerator, denominator), d_k = n_k / m_k with (n_k, m_k) the first column
// of M_k ... M_0.  A lane composes its E matrices, a Hillis-Steele warp scan
// composes the lanes', and each lane replays its cells from its exclusive
// prefix.  Products are rescaled by their largest entry at every step (the
// map is projective), so nothing overflows; the arithmetic is FP64
// throughout.  l_k = e_k / d_k as in the serial sweep; the FP32 casts of the
// four coefficients ride along.
#pragma once

#include "gw_device.cuh"

namespace fgw {

struct M2 {
  double a, b, c, d;  // [[a, b], [c, d]]
};

__device__ inline M2 m2_mul(const M2& x, const M2& y) {  // x * y, rescaled
  M2 r{x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c,
       x.c * y.b + x.d * y.d};
  const double s = fmax(fmax(fabs(r.a), fabs(r.b)), fmax(fabs(r.c), fabs(r.d)));
  if (s > 0.0 && isfinite(s)) {
    const double is = 1.0 / s;
    r.a *= is;
    r.b *= is;
    r.c *= is;
    r.d *= is;
  }
  return r;
}

__device__ inline M2 m2_shfl_up(const M2& x, int off) {
  return M2{__shfl_up_sync(0xffffffffu, x.a, off), __shfl_up_sync(0xffffffffu, x.b, off),
            __shfl_up_sync(0xffffffffu, x.c, off), __shfl_up_sync(0xffffffffu, x.d, off)};
}

// Factors the column at cell offset cb whose lane-held coefficients are av
// (diag), ev (gzp), xv (gxp), yv (gyp), cells k >= nz padded with a = 1 and
// zero legs; writes the FP32 casts and the factors (1/d_k, l_k).  Every lane
// of the warp must call it.
template <int E>
__device__ __forceinline__ void factor_column(int nz, long long cb, const double (&av)[E],
                                              const double (&ev)[E], const double (&xv)[E],
                                              const double (&yv)[E], float* __restrict__ diag32,
                                              float* __restrict__ gxp32, float* __restrict__ gyp32,
                                              float* __restrict__ gzp32, float* __restrict__ dinv32,
                                              float* __restrict__ l32) {
  const int lane = threadIdx.x & 31, k0 = lane * E;
  const double eprev_lane = __shfl_up_sync(0xffffffffu, ev[E - 1], 1);  // e_{k0-1}
  // This lane's maps, composed (later cells on the left).
  M2 L{1.0, 0.0, 0.0, 1.0};
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    if (k < nz) {
      const double ep = (k == 0) ? 0.0 : (e == 0 ? eprev_lane : ev[e - 1]);
      L = m2_mul(M2{av[e], -ep * ep, 1.0, 0.0}, L);
    }
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const M2 q = m2_shfl_up(L, off);
    if (lane >= off) L = m2_mul(L, q);
  }
  M2 X = m2_shfl_up(L, 1);
  if (lane == 0) X = M2{1.0, 0.0, 0.0, 1.0};
  double n = X.a, m = X.c;  // (numerator, denominator) of d_{k0-1}
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    if (k >= nz) break;
    const long long c = cb + k;
    const double ep = (k == 0) ? 0.0 : (e == 0 ? eprev_lane : ev[e - 1]);
    const double n2 = av[e] * n - ep * ep * m;
    m = n;
    n = n2;
    const double s = fmax(fabs(n), fabs(m));
    if (s > 0.0 && isfinite(s)) {
      n /= s;
      m /= s;
    }
    const double dk = n / m;
    diag32[c] = static_cast<float>(av[e]);
    gxp32[c] = static_cast<float>(xv[e]);
    gyp32[c] = static_cast<float>(yv[e]);
    gzp32[c] = static_cast<float>(ev[e]);
    dinv32[c] = (dk > 0.0 && isfinite(dk)) ? static_cast<float>(1.0 / dk)
                                           : static_cast<float>(1.0 / av[e]);
    l32[c] = (k + 1 < nz) ? static_cast<float>(ev[e] / dk) : 0.0f;
  }
}

// The same factorization for the FP64 line form: FP64 factors (1/d_k, l_k),
// no casts.
template <int E>
__device__ __forceinline__ void factor_column64(int nz, long long cb, const double (&av)[E],
                                                const double (&ev)[E], double* __restrict__ dinv,
                                                double* __restrict__ l) {
  const int lane = threadIdx.x & 31, k0 = lane * E;
  const double eprev_lane = __shfl_up_sync(0xffffffffu, ev[E - 1], 1);
  M2 L{1.0, 0.0, 0.0, 1.0};
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    if (k < nz) {
      const double ep = (k == 0) ? 0.0 : (e == 0 ? eprev_lane : ev[e - 1]);
      L = m2_mul(M2{av[e], -ep * ep, 1.0, 0.0}, L);
    }
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const M2 q = m2_shfl_up(L, off);
    if (lane >= off) L = m2_mul(L, q);
  }
  M2 X = m2_shfl_up(L, 1);
  if (lane == 0) X = M2{1.0, 0.0, 0.0, 1.0};
  double n = X.a, m = X.c;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    if (k >= nz) break;
    const long long c = cb + k;
    const double ep = (k == 0) ? 0.0 : (e == 0 ? eprev_lane : ev[e - 1]);
    const double n2 = av[e] * n - ep * ep * m;
    m = n;
    n = n2;
    const double s = fmax(fabs(n), fabs(m));
    if (s > 0.0 && isfinite(s)) {
      n /= s;
      m /= s;
    }
    const double dk = n / m;
    dinv[c] = (dk > 0.0 && isfinite(dk)) ? 1.0 / dk : 1.0 / av[e];
    l[c] = (k + 1 < nz) ? ev[e] / dk : 0.0;
  }
}

}  // namespace fgw
