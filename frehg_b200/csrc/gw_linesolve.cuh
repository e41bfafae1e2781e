// The line preconditioner's column solve z = T^-1 r, one warp per column
// (nz <= 32 * kMaxE), in the precision T of the inner iteration: FP32 for
// the mixed form (gw_cg_mixed.cu), FP64 for the FP64 line form
// (gw_cg_line64.cu).
//
// Lane `lane` holds the E consecutive cells k = lane * E + e of the column
// (E a power of two with 32 E >= nz).  With the unit lower bidiagonal factor
// L (subdiagonal l) and pivots 1/dinv, z = T^-1 r is
//   y_k = r_k - l_{k-1} y_{k-1}            (k ascending, y_0 = r_0)
//   z_k = dinv_k y_k - l_k z_{k+1}         (k descending, z_{nz-1} = dinv y)
// Each step is an affine map of its predecessor.  A lane composes its E maps,
// a Hillis-Steele scan over the 32 lanes composes the lane maps (inclusive
// for the forward sweep, suffix for the backward one), and each lane then
// replays its E steps from its exclusive prefix.  Cells past nz hold the
// identity map.
//
// Every load of a column is issued before any of its stores: the arrays are
// distinct, but the compiler cannot prove it, and loads placed after a store
// would wait for it.
#pragma once

#include <type_traits>

namespace fgw {

constexpr int kMaxE = 8;
constexpr unsigned kFull = 0xffffffffu;

__device__ inline float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ inline double fma_t(double a, double b, double c) { return fma(a, b, c); }

template <typename T>
__device__ inline void scan_affine_up(T& A, T& B, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T Ap = __shfl_up_sync(kFull, A, off);
    const T Bp = __shfl_up_sync(kFull, B, off);
    if (lane >= off) {
      B = fma_t(A, Bp, B);
      A *= Ap;
    }
  }
}

template <typename T>
__device__ inline void scan_affine_down(T& C, T& Dv, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T Cn = __shfl_down_sync(kFull, C, off);
    const T Dn = __shfl_down_sync(kFull, Dv, off);
    if (lane + off < 32) {
      Dv = fma_t(C, Dn, Dv);
      C *= Cn;
    }
  }
}

// Load / store a lane's E cells of the column starting at cb.  `vec` (nz a
// multiple of E) makes every lane all-in or all-out, with E-aligned addresses
// (16-byte vector accesses: float2 / float4 for FP32, double2 for FP64).
template <int E, typename T>
__device__ inline void ld_col(const T* p, long long cb, int lane, int nz, bool vec, T (&v)[E]) {
  const int k0 = lane * E;
  if (vec) {
    if (k0 < nz) {
      const T* q = p + cb + k0;
      if constexpr (E == 1) {
        v[0] = q[0];
      } else if constexpr (std::is_same<T, float>::value && E == 2) {
        const float2 t = *reinterpret_cast<const float2*>(q);
        v[0] = t.x;
        v[1] = t.y;
      } else if constexpr (std::is_same<T, float>::value) {
#pragma unroll
        for (int e = 0; e < E; e += 4) {
          const float4 t = *reinterpret_cast<const float4*>(q + e);
          v[e] = t.x;
          v[e + 1] = t.y;
          v[e + 2] = t.z;
          v[e + 3] = t.w;
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; e += 2) {
          const double2 t = *reinterpret_cast<const double2*>(q + e);
          v[e] = t.x;
          v[e + 1] = t.y;
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = T(0);
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = (k0 + e < nz) ? p[cb + k0 + e] : T(0);
  }
}

template <int E, typename T>
__device__ inline void st_col(T* p, long long cb, int lane, int nz, bool vec, const T (&v)[E]) {
  const int k0 = lane * E;
  if (vec) {
    if (k0 < nz) {
      T* q = p + cb + k0;
      if constexpr (E == 1) {
        q[0] = v[0];
      } else if constexpr (std::is_same<T, float>::value && E == 2) {
        *reinterpret_cast<float2*>(q) = make_float2(v[0], v[1]);
      } else if constexpr (std::is_same<T, float>::value) {
#pragma unroll
        for (int e = 0; e < E; e += 4)
          *reinterpret_cast<float4*>(q + e) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
      } else {
#pragma unroll
        for (int e = 0; e < E; e += 2)
          *reinterpret_cast<double2*>(q + e) = make_double2(v[e], v[e + 1]);
      }
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (k0 + e < nz) p[cb + k0 + e] = v[e];
  }
}

// z = T^-1 r for the column whose factors this lane holds (lk = l_k,
// di = dinv_k of its E cells).
template <int E, typename T>
__device__ inline void warp_column_solve(const T (&lk)[E], const T (&di)[E], int lane, int nz,
                                         const T (&r)[E], T (&z)[E]) {
  const int k0 = lane * E;
  const T lprev = __shfl_up_sync(kFull, lk[E - 1], 1);  // l_{k0-1}
  T a[E];
  T A = T(1), B = T(0);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = k0 + e;
    a[e] = (k >= nz) ? T(1) : (k == 0) ? T(0) : -(e == 0 ? lprev : lk[e - 1]);
    const T b = (k < nz) ? r[e] : T(0);
    B = fma_t(a[e], B, b);
    A *= a[e];
  }
  scan_affine_up(A, B, lane);
  T y = __shfl_up_sync(kFull, B, 1);
  if (lane == 0) y = T(0);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    y = fma_t(a[e], y, (k0 + e < nz) ? r[e] : T(0));
    z[e] = y;
  }
  T c[E];
  T C = T(1), Dv = T(0);
#pragma unroll
  for (int e = E - 1; e >= 0; --e) {
    const int k = k0 + e;
    c[e] = (k >= nz) ? T(1) : (k + 1 < nz) ? -lk[e] : T(0);
    z[e] = (k < nz) ? di[e] * z[e] : T(0);
    Dv = fma_t(c[e], Dv, z[e]);
    C *= c[e];
  }
  scan_affine_down(C, Dv, lane);
  T zn = __shfl_down_sync(kFull, Dv, 1);
  if (lane == 31) zn = T(0);
#pragma unroll
  for (int e = E - 1; e >= 0; --e) {
    zn = fma_t(c[e], zn, z[e]);
    z[e] = zn;
  }
}

}  // namespace fgw
