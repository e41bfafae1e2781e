// Device-side building blocks of the B200 groundwater step: the van
// Genuchten-Mualem closures, the face-conductivity rules and the layout
// helpers shared by the kernels in gw_kernels.cu and gw_cg.cu.
//
// Layout.  Every cell field lives in the halo layout of the reference
// (src/core/Types.hpp:35-43): (ny+2, nx+2, nz) with k unit-stride, so cell
// (j, i, k) is at ((j * (nx+2)) + i) * nz + k.  z-face fields carry nz+1
// planes per column (plane k = face above cell k).  Solver vectors add a
// zero margin of one j-row on both ends so the 7-point stencil reads of
// ghost cells stay in bounds and multiply zero coefficients.
#pragma once

#include <cstdint>

namespace fgw {

enum BcCode : int { kNoFlux = 0, kHead = 1, kFlux = 2, kGravity = 3, kHydro = 4 };

struct Soil {
  double vga, vgn, ts, tr, aev;
};

// Static geometry and parameters of one domain, by value in every launch.
struct Dims {
  int nx, ny, nz;
  int nx2, ny2;          // nx + 2, ny + 2
  long long sx, sy;      // strides of i and j in a cell field (nz, (nx+2) nz)
  long long ncell;       // (ny+2)(nx+2)nz
  long long ncol;        // (ny+2)(nx+2)
  double dx, dy, az;
  double idx, idy;       // 1 / dx, 1 / dy
  double ss;             // specific storage
  int full3d, pc, harm, off, redistribute, terrain;
  // Multipliers of the divisions by nz and by nx + 2 (div_magic); the
  // domain's cell count is below 2^32.
  unsigned long long mz, mx2;
};

// The coupled top's device state (GwCoupling), one per coupled domain: the
// vent rule, min_depth, the mesh bed (offset frame) and the surface fields
// the step reads and writes, (ny+2)(nx+2) each, and the per-column exchange
// mode.  Kernels reach it through Fields::cpl, null in groundwater-only runs,
// so those keep the kernels' parameter blocks of the uncoupled step.
struct CplDev {
  int vent_all, book_bounce;
  double min_depth;
  const double* bath;
  double *eta, *dept, *seep, *avail, *gain, *bounce;
  int8_t* cmode;
};

// Density coupling (Baroclinic.cpp): the cell density ratio and the face
// means of the density and viscosity ratios, written at the start of every
// step from the attached scalars (halo layouts: x / y faces like qx / qy,
// z faces like qzF).  Kernels reach them through Fields::baro, null without
// an attached scalar (every ratio is then exactly 1).
struct BaroDev {
  const double *rrho, *rxp, *ryp, *rzp, *vxp, *vyp, *vzp;
  int dgrad;  // the post-allocation split against the face r (not 1)
};

// Device pointers of one domain (see gw_internal.h for ownership).
// One soil parameter field, read as f.field[c] either way: per-cell values
// in the halo layout (mirrored ghosts, m = ~0), or, for a field that is
// uniform over the domain, one value in device memory (m = 0: every index
// reads p[0], a broadcast from L1 instead of a stream from HBM).  The index
// mask costs one integer AND; a branch on uniformity made the kernels spill.
struct SoilField {
  const double* p;
  long long m;
  __host__ __device__ double operator[](long long c) const { return p[c & m]; }
};

struct Fields {
  // soil: ksx ksy ksz alpha n theta_s theta_r aev
  SoilField ksx, ksy, ksz, vga, vgn, wcs, wcr, aev;
  // geometry
  const double *dz, *bot, *ax, *ay, *sinx, *cosx, *siny, *cosy;
  const int8_t* act;   // 1 = active cell (gid >= 0), 0 = inactive or ghost
  // boundary markers, (ny+2)(nx+2); side codes live on the edge columns
  const int *topc, *botc, *xmc, *xpc, *ymc, *ypc;
  const double *topv, *botv, *xmv, *xpv, *ymv, *ypv;
  const CplDev* cpl;  // coupled top, null when off
  const BaroDev* baro;  // density coupling, null when off
};

__host__ __device__ inline long long cidx(const Dims& d, int j, int i, int k) {
  return (static_cast<long long>(j) * d.nx2 + i) * d.nz + k;
}
__host__ __device__ inline long long fidx(const Dims& d, int j, int i, int k) {
  return (static_cast<long long>(j) * d.nx2 + i) * (d.nz + 1) + k;
}
__host__ __device__ inline long long col2(const Dims& d, int j, int i) {
  return static_cast<long long>(j) * d.nx2 + i;
}
// Division of n < 2^32 by an invariant divisor q >= 2 as the high word of
// n * M with M = floor((2^64 - 1) / q) + 1 (Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994):
// n M / 2^64 = n / q + n e / 2^64 with 0 <= e < 1, and n q < 2^64 keeps the
// second term below the distance from n / q up to the next integer.  M = 0
// stands for q = 1.
__host__ __device__ inline unsigned long long div_magic(unsigned q) {
  return q < 2 ? 0ULL : ~0ULL / q + 1ULL;
}
__device__ inline unsigned div_by(unsigned long long n, unsigned long long m) {
  return m == 0ULL ? static_cast<unsigned>(n) : static_cast<unsigned>(__umul64hi(n, m));
}
__device__ inline void unflatten(const Dims& d, long long c, int& j, int& i, int& k) {
  const unsigned col = div_by(static_cast<unsigned long long>(c), d.mz);
  k = static_cast<int>(static_cast<unsigned>(c) - col * static_cast<unsigned>(d.nz));
  j = static_cast<int>(div_by(col, d.mx2));
  i = static_cast<int>(col - static_cast<unsigned>(j) * static_cast<unsigned>(d.nx2));
}
__device__ inline bool is_head(int code) { return code == kHead || code == kHydro; }

__device__ inline Soil soil_at(const Fields& f, long long c) {
  return Soil{f.vga[c], f.vgn[c], f.wcs[c], f.wcr[c], f.aev[c]};
}

// ---------------------------------------------------------------- closures
// The pointwise van Genuchten-Mualem relations of the frehg2 groundwater
// module (src/gw/VanGenuchten.hpp:45-128): theta(h) with the air-entry cutoff
// and [theta_r, theta_s] clamp, h(theta) with the theta_r + 1e-7 floor, C(h)
// and K(h) cut off at h > 0, K capped at Ks, dK/dtheta with the 0.9999
// theta_s limiter.  Every power goes through the CUDA math library's pow.

__device__ inline double vg_theta(const Soil& s, double h) {
  const double m = 1.0 - 1.0 / s.vgn;
  double wc;
  if (h > s.aev) {
    wc = s.ts;
  } else {
    const double se = pow(1.0 + pow(fabs(s.vga * h), s.vgn), -m);
    wc = s.tr + (s.ts - s.tr) * se;
  }
  if (wc > s.ts) {
    wc = s.ts;
  } else if (wc < s.tr) {
    wc = s.tr;
  }
  return wc;
}

__device__ inline double vg_head(const Soil& s, double wc) {
  const double m = 1.0 - 1.0 / s.vgn;
  if (wc - s.tr < 1.0e-7) wc = s.tr + 1.0e-7;
  if (wc < s.ts) {
    const double ratio = (s.ts - s.tr) / (wc - s.tr);
    return -(1.0 / s.vga) * pow(pow(ratio, 1.0 / m) - 1.0, 1.0 / s.vgn);
  }
  return 0.0;
}

// theta(h) and h(theta) of the classification, through logarithms: 2 log + 2
// exp in place of 2 pow each (the initial state keeps the pow forms above).
__device__ inline double vg_theta_fast(const Soil& s, double h) {
  const double m = 1.0 - 1.0 / s.vgn;
  double wc;
  if (h > s.aev) {
    wc = s.ts;
  } else {
    const double ah = fabs(s.vga * h);
    const double se = (ah > 0.0) ? exp(-m * log1p(exp(s.vgn * log(ah)))) : 1.0;
    wc = s.tr + (s.ts - s.tr) * se;
  }
  if (wc > s.ts) {
    wc = s.ts;
  } else if (wc < s.tr) {
    wc = s.tr;
  }
  return wc;
}

// h(theta) with 1/m = n / (n - 1) and 1/n taken before the logarithms, so
// the chain log -> expm1 -> log -> exp holds multiplications, not divisions
// (equal to the divided form up to rounding).
__device__ inline double vg_head_fast(const Soil& s, double wc) {
  const double im = s.vgn / (s.vgn - 1.0), in = 1.0 / s.vgn;
  if (wc - s.tr < 1.0e-7) wc = s.tr + 1.0e-7;
  if (wc < s.ts) {
    const double ratio = (s.ts - s.tr) / (wc - s.tr);
    const double x = expm1(log(ratio) * im);  // ratio^(1/m) - 1
    return -(1.0 / s.vga) * exp(log(x) * in);
  }
  return 0.0;
}

// The closures below share t = |alpha h|^n, u = 1 + t and Se = u^-m between
// K(h) and C(h), and rewrite the reference's nested powers by exact identities
// (Se^(1/m) = 1/u, so 1 - Se^(1/m) = t/u; Se^(1/2) = sqrt(Se);
// u^(m+1) = u / Se; |alpha h|^(n-1) = t / |alpha h|).  The values agree with the
// reference's expression trees to rounding (the t/u form also avoids the
// cancellation of 1 - Se^(1/m) near saturation), at 3 powers per cell for K and
// C together instead of 8.  The powers go through logarithms shared between
// them: ln t = n ln|alpha h|, ln u = log1p(t), Se = exp(-m ln u) and
// (t/u)^m = exp(m (ln t - ln u)) -- 2 logarithms and 3 exponentials in place of
// 3 pow calls, whose own extended-precision logarithm made the closure passes
// FP64-pipe bound (relative error ~1e-15 against pow's ulp, far inside the step's
// parity bars; measured -1.2 ms per 512x512x128 step).
struct VgParts {
  double t, u, se, m, ah, lt, lu;  // lt = ln t, lu = ln u
};
__device__ inline VgParts vg_parts(const Soil& s, double h) {
  VgParts p;
  p.m = 1.0 - 1.0 / s.vgn;
  p.ah = fabs(s.vga * h);
  if (p.ah > 0.0) {
    p.lt = s.vgn * log(p.ah);
    p.t = exp(p.lt);
    p.lu = log1p(p.t);
    p.se = exp(-p.m * p.lu);
  } else {
    p.lt = -INFINITY;
    p.t = 0.0;
    p.lu = 0.0;
    p.se = 1.0;
  }
  p.u = 1.0 + p.t;
  return p;
}

// C(h) = dtheta/dh (capacityFromHead): 0 for h > 0.
__device__ inline double vg_capacity_from(const Soil& s, const VgParts& p, double h) {
  if (h > 0.0 || p.ah == 0.0) return 0.0;
  const double nume = s.vga * s.vgn * p.m * (s.ts - s.tr) * (p.t / p.ah);
  return nume * p.se / p.u;
}

__device__ inline double vg_capacity(const Soil& s, double h) {
  return vg_capacity_from(s, vg_parts(s, h), h);
}

// Relative-permeability pieces of K(h) shared by the three directional Ks of
// one cell: K = ((ks * root) * br) * br, capped at ks, ks for h > 0.
struct KrParts {
  double root, br;
  bool sat;
};
__device__ inline KrParts vg_kr_from(const VgParts& v, double h) {
  KrParts p;
  p.br = 1.0 - exp(v.m * (v.lt - v.lu));
  p.root = sqrt(v.se);
  p.sat = h > 0.0;
  return p;
}
__device__ inline KrParts vg_kr_parts(const Soil& s, double h) {
  return vg_kr_from(vg_parts(s, h), h);
}
__device__ inline double vg_k_from(const KrParts& p, double ks) {
  double k = ks * p.root * p.br * p.br;
  if (k > ks) k = ks;
  if (p.sat) k = ks;
  return k;
}
__device__ inline double vg_k(const Soil& s, double h, double ks) {
  return vg_k_from(vg_kr_parts(s, h), ks);
}

// dK/dtheta (conductivityDerivative) with Se^(-1/2) = 1/sqrt(Se),
// Se^((2-m)/(2m)) = Se^(1/m) / sqrt(Se) and (1 - Se^(1/m))^(m-1) =
// (1 - Se^(1/m))^m / (1 - Se^(1/m)): 2 powers instead of 6.
__device__ inline double vg_dkdtheta(const Soil& s, double wc, double ks) {
  if (wc > 0.9999 * s.ts && wc < s.ts) wc = 0.9999 * s.ts;
  const double m = 1.0 - 1.0 / s.vgn, im = s.vgn / (s.vgn - 1.0);
  const double idt = 1.0 / (s.ts - s.tr);
  const double se = (wc - s.tr) * idt;
  const double s1m = exp(log(se) * im);  // Se^(1/m); Se = 0 gives 0
  const double q = 1.0 - s1m;
  const double t0 = exp(m * log(q));     // (1 - Se^(1/m))^m
  const double irs = rsqrt(se);          // Se^(-1/2)
  const double t1 = 0.5 * ks * irs * (1.0 - t0) * (1.0 - t0);
  const double t2 = 2.0 * ks * (s1m * irs) * (1.0 - t0) * (t0 / q);
  return (t1 + t2) * idt;
}

// Harmonic-Ks x arithmetic-kr face rule (src/gw/FaceConductivity.hpp:48-59)
// from the flanks' own conductivities ka = K(h_a, Ks_a), kb = K(h_b, Ks_b).
__device__ inline double face_harm(double ka, double ksa, double la, double kb, double ksb,
                                   double lb) {
  if (ksa <= 0.0 || ksb <= 0.0) return 0.0;
  const double ksh = (la + lb) / (la / ksa + lb / ksb);
  return ksh * 0.5 * (ka / ksa + kb / ksb);
}

// ---------------------------------------------------------------- face rules
// Face conductivities of one pass (predictor or corrector), built from the
// per-cell directional conductivities Kc = K(h_c, Ks_c) of that pass with the
// reference's overrides applied in its order (src/gw/Predictor.cpp:105-386):
// interior mean -> domain-edge rule -> top rule -> use_full3d -> inactive seal.
struct PassK {
  const double *kcx, *kcy, *kcz;  // per-cell K with Ksx, Ksy, Ksz
  const double* wc;               // moisture at the pass (use_full3d test)
};

// x face between (j, i) and (j, i+1), i in [0, nx], j in [1, ny].
__device__ inline double face_kx(const Dims& d, const Fields& f, const PassK& p, int j, int i,
                                 int k) {
  const long long a = cidx(d, j, i, k), b = a + d.sx;
  double kf;
  if (d.harm) {
    kf = face_harm(p.kcx[a], f.ksx[a], 1.0, p.kcx[b], f.ksx[b], 1.0);
  } else {
    kf = 0.5 * (p.kcx[a] + p.kcx[b]);
  }
  if (i == 0) {  // west edge face, owned by cell i = 1
    const int code = f.xmc[col2(d, j, 1)];
    if (code == kNoFlux) kf = 0.0;
    else if (is_head(code)) kf = p.kcx[b];
  } else if (i == d.nx) {
    const int code = f.xpc[col2(d, j, d.nx)];
    if (code == kNoFlux) kf = 0.0;
    else if (is_head(code)) kf = p.kcx[a];
  }
  if (!d.full3d) {
    if ((f.act[a] && p.wc[a] < f.wcs[a]) || (f.act[b] && p.wc[b] < f.wcs[b])) kf = 0.0;
  }
  const bool ina = (i >= 1) && !f.act[a];
  const bool inb = (i + 1 <= d.nx) && !f.act[b];
  if (ina || inb) kf = 0.0;
  return kf;
}

// y face between (j, i) and (j+1, i), j in [0, ny], i in [1, nx].
__device__ inline double face_ky(const Dims& d, const Fields& f, const PassK& p, int j, int i,
                                 int k) {
  const long long a = cidx(d, j, i, k), b = a + d.sy;
  double kf;
  if (d.harm) {
    kf = face_harm(p.kcy[a], f.ksy[a], 1.0, p.kcy[b], f.ksy[b], 1.0);
  } else {
    kf = 0.5 * (p.kcy[a] + p.kcy[b]);
  }
  if (j == 0) {
    const int code = f.ymc[col2(d, 1, i)];
    if (code == kNoFlux) kf = 0.0;
    else if (is_head(code)) kf = p.kcy[b];
  } else if (j == d.ny) {
    const int code = f.ypc[col2(d, d.ny, i)];
    if (code == kNoFlux) kf = 0.0;
    else if (is_head(code)) kf = p.kcy[a];
  }
  if (!d.full3d) {
    if ((f.act[a] && p.wc[a] < f.wcs[a]) || (f.act[b] && p.wc[b] < f.wcs[b])) kf = 0.0;
  }
  const bool ina = (j >= 1) && !f.act[a];
  const bool inb = (j + 1 <= d.ny) && !f.act[b];
  if (ina || inb) kf = 0.0;
  return kf;
}

// z face plane k in [0, nz] of interior column (j, i): the face above cell k.
__device__ inline double face_kz(const Dims& d, const Fields& f, const PassK& p, int j, int i,
                                 int k) {
  const long long base = cidx(d, j, i, 0);
  const bool below = (k < d.nz) && f.act[base + k];
  const bool above = (k >= 1) && f.act[base + k - 1];
  // Seal (applied last in the reference): a face with an inactive cell on
  // either side is closed.  This also closes the face above the top cell of
  // a masked column (k > 0), whose top rule the seal overrides.
  if ((k < d.nz && !below) || (k >= 1 && !above)) return 0.0;
  if (k == 0) {
    const int code = f.topc[col2(d, j, i)];
    if (code == kHead) return f.ksz[base];
    if (code == kNoFlux) return 0.0;
    return p.kcz[base];
  }
  if (k == d.nz) {
    return (f.botc[col2(d, j, i)] == kNoFlux) ? 0.0 : p.kcz[base + d.nz - 1];
  }
  const long long up = base + k - 1, lo = base + k;
  if (d.harm) return face_harm(p.kcz[up], f.ksz[up], f.dz[up], p.kcz[lo], f.ksz[lo], f.dz[lo]);
  return 0.5 * (p.kcz[up] + p.kcz[lo]);
}


// ---------------------------------------------------------------- face rules on loaded values
// The rules of face_kx / face_ky / face_kz, evaluated on values the caller
// has already loaded, so a kernel can issue every load of a cell before its
// first branch on loaded data.
struct Flank {
  double kc, ks;  // K(h, Ks) of the pass and Ks along the face normal
  double w, ws;   // the pass moisture and theta_s (use_full3d test)
  int8_t act;
};

// Lateral face between flank a (lower index) and flank b.  lo_edge / hi_edge:
// the face is the domain's low / high boundary face in this direction, whose
// BC code is `code`.
__device__ inline double face_lat(const Dims& d, const Flank& a, const Flank& b, bool lo_edge,
                                  bool hi_edge, int code) {
  double kf = d.harm ? face_harm(a.kc, a.ks, 1.0, b.kc, b.ks, 1.0) : 0.5 * (a.kc + b.kc);
  if (lo_edge) {
    if (code == kNoFlux) kf = 0.0;
    else if (is_head(code)) kf = b.kc;
  } else if (hi_edge) {
    if (code == kNoFlux) kf = 0.0;
    else if (is_head(code)) kf = a.kc;
  }
  if (!d.full3d) {
    if ((a.act && a.w < a.ws) || (b.act && b.w < b.ws)) kf = 0.0;
  }
  if ((!lo_edge && !a.act) || (!hi_edge && !b.act)) kf = 0.0;
  return kf;
}

struct ZFlank {
  double kc, ks, dz;
  int8_t act;
};

// z face plane k of a column: u = cell k-1 (above), l = cell k (below);
// dep = the column's surface depth (coupled runs).
template <bool CPL>
__device__ inline double face_z(const Dims& d, const ZFlank& u, const ZFlank& l, int k, int topc,
                                int botc, double dep) {
  const bool below = (k < d.nz) && l.act;
  const bool above = (k >= 1) && u.act;
  if ((k < d.nz && !below) || (k >= 1 && !above)) return 0.0;
  if (k == 0) {
    if (CPL) {  // coupled top (Predictor.cpp:293-302)
      if (d.pc) return (dep > 0.0) ? l.ks : l.kc;
      return (dep > 0.0) ? 0.5 * (l.ks + l.kc) : l.kc;
    }
    if (topc == kHead) return l.ks;
    if (topc == kNoFlux) return 0.0;
    return l.kc;
  }
  if (k == d.nz) return (botc == kNoFlux) ? 0.0 : u.kc;
  if (d.harm) return face_harm(u.kc, u.ks, u.dz, l.kc, l.ks, l.dz);
  return 0.5 * (u.kc + l.kc);
}

}  // namespace fgw
