/* gw_oracle.c — serial FP64 restatement of the frehg2 groundwater step.
 *
 * TEST INFRASTRUCTURE (see gw_oracle.h).  Storage follows the reference's
 * halo layout: 3D fields are (ny+2, nx+2, nz) with k fastest and a one-cell
 * halo in j and i (src/core/Types.hpp:35-43); z-face fields carry nz+1
 * planes, plane k being the face above cell k (RichardsSolver.hpp:584-591).
 * Single rank: every domain edge is a physical boundary and halo exchanges
 * are no-ops.  The density / viscosity ratios of the reference formulas sit
 * at the reference's places in every expression; without an attached scalar
 * they stay exactly 1 (RichardsSolver.cpp:141-150), and multiplying by 1.0 is
 * exact.  Expressions keep the reference's evaluation order.
 */
#include "gw_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static _Thread_local char g_err[512];
static void set_err(const char* m) { snprintf(g_err, sizeof g_err, "%s", m); }
const char* oracle_gw_last_error(void) { return g_err; }

enum { NOFLUX = 0, HEAD = 1, FLUX = 2, GRAVITY = 3, HYDRO = 4 };

struct oracle_gw {
  int nx, ny, nz;
  size_t n2, n3, n3f; /* (ny+2)(nx+2), *nz, *(nz+1) */
  double dx, dy, az;
  int follow_terrain, uniform;
  double offset, box_top;
  /* geometry (TerrainMetric) */
  double *bath, *dz, *bot, *ax, *ay, *sinx, *cosx, *siny, *cosy;
  int *ktop; /* ny*nx */
  int* gid;  /* n3, -1 inactive */
  long long nactive;
  /* soil, mirrored ghosts */
  double *ksx, *ksy, *ksz, *vga, *vgn, *wcs, *wcr, *aev;
  double ss;
  /* state */
  double *h, *hn, *wc, *wcn, *ch, *kx, *ky, *kz, *qx, *qy, *qz, *vloss;
  double *room, *sup, *sdown, *wcsnap, *hsnap;
  /* boundary markers, (ny+2)(nx+2) */
  int *topc, *botc, *xmc, *xpc, *ymc, *ypc;
  double *topv, *botv, *xmv, *xpv, *ymv, *ypv;
  /* switches */
  int full3d, pc, harm, off, redistribute, schead;
  double dt_min, dt_max, dq_grow, dq_shrink, co_max, dtg_next;
  double rtol, atol;
  int maxit;
  /* linear system: per active row 7 legs + neighbor rows */
  double* vals7;
  long* cols7;
  double *rhs, *sol;
  int have_state;
  frehg_gw_step_info last;
  /* coupled top (GwCoupling, src/gw/RichardsSolver.hpp:132-175): surface
   * fields (ny+2)(nx+2), the per-column exchange mode and the step's books */
  int cpl, vent_all, book_bounce;
  double min_depth;
  double *eta, *dept, *seep, *avail, *gain, *bounce, *qss;
  int* cmode;
  double cpl_exch, cpl_bounce, cpl_vent, cpl_thin, cpl_evap, pc_clamp;
  /* coupler (src/coupling/Coupler.hpp): sync flag, surface dt, adaptive
   * subsurface dt and clock */
  int csync;
  double cdt, cdtg, ctsub, clast_dt;
  /* transport window (RichardsSolver.hpp:229-248): face volumes of the window
   * in the qx / qy / qzF layouts, the walks' path records, vented volume */
  int win;
  double *wx, *wy, *wz, *pcorr, *wvent;
  /* density coupling (RichardsSolver.hpp:191-225, Baroclinic.cpp): the
   * attached scalars (cells n3, surfaces n2), the coefficients, and the cell
   * and face ratios (x / y faces n3, z faces n3f), 1 until a step computes
   * them from an attached scalar */
  int baro, saline, thermal, dgrad;
  double beta_s, beta_sv, beta_t, t_ref;
  double *s3, *s2, *t3, *t2;
  double *rrho, *rvisc, *rxp, *ryp, *rzp, *vxp, *vyp, *vzp;
};

#define I2(s, j, i) ((size_t)(j) * (size_t)((s)->nx + 2) + (size_t)(i))
#define I3(s, j, i, k) (I2(s, j, i) * (size_t)(s)->nz + (size_t)(k))
#define IF(s, j, i, k) (I2(s, j, i) * (size_t)((s)->nz + 1) + (size_t)(k))

/* ------------------------------------------------------------------ closures
 * src/gw/VanGenuchten.hpp:45-128 (legacy subroutines.c:280-483). */
typedef struct { double vga, vgn, ts, tr, aev; } soil_t;

static double vg_theta(soil_t s, double h) { /* waterContentFromHead :45-60 */
  const double m = 1.0 - 1.0 / s.vgn;
  double wc;
  if (h > s.aev) {
    wc = s.ts;
  } else {
    const double se = pow(1.0 + pow(fabs(s.vga * h), s.vgn), -m);
    wc = s.tr + (s.ts - s.tr) * se;
  }
  if (wc > s.ts) wc = s.ts;
  else if (wc < s.tr) wc = s.tr;
  return wc;
}

static double vg_head(soil_t s, double wc) { /* headFromWaterContent :65-77 */
  const double eps = 1.0e-7;
  const double m = 1.0 - 1.0 / s.vgn;
  if (wc - s.tr < eps) wc = s.tr + eps;
  if (wc < s.ts) {
    const double ratio = (s.ts - s.tr) / (wc - s.tr);
    return -(1.0 / s.vga) * pow(pow(ratio, 1.0 / m) - 1.0, 1.0 / s.vgn);
  }
  return 0.0;
}

static double vg_cap(soil_t s, double h) { /* capacityFromHead :82-92 */
  if (h > 0.0) return 0.0;
  const double m = 1.0 - 1.0 / s.vgn;
  const double ah = fabs(s.vga * h);
  const double nume = s.vga * s.vgn * m * (s.ts - s.tr) * pow(ah, s.vgn - 1.0);
  const double deno = pow(1.0 + pow(ah, s.vgn), m + 1.0);
  return nume / deno;
}

static double vg_k(soil_t s, double h, double ks) { /* conductivityFromHead :99-111 */
  const double m = 1.0 - 1.0 / s.vgn;
  const double se = pow(1.0 + pow(fabs(s.vga * h), s.vgn), -m);
  const double br = 1.0 - pow(1.0 - pow(se, 1.0 / m), m);
  double k = ks * pow(se, 0.5) * br * br;
  if (k > ks) k = ks;
  if (h > 0.0) k = ks;
  return k;
}

static double vg_dkdtheta(soil_t s, double wc, double ks) { /* conductivityDerivative :117-128 */
  if (wc > 0.9999 * s.ts && wc < s.ts) wc = 0.9999 * s.ts;
  const double m = 1.0 - 1.0 / s.vgn;
  const double se = (wc - s.tr) / (s.ts - s.tr);
  const double t0 = pow(1.0 - pow(se, 1.0 / m), m);
  const double t1 = 0.5 * ks * pow(se, -0.5) * (1.0 - t0) * (1.0 - t0);
  const double t2 = 2.0 * ks * pow(se, (2.0 - m) / (2.0 * m)) * (1.0 - t0) *
                    pow(1.0 - pow(se, 1.0 / m), m - 1.0);
  return (t1 + t2) / (s.ts - s.tr);
}

/* FaceConductivity.hpp:48-59 (harmonic Ks x arithmetic kr). */
static double face_harm(soil_t a, double ha, double ksa, double la, soil_t b, double hb,
                        double ksb, double lb) {
  if (ksa <= 0.0 || ksb <= 0.0) return 0.0;
  const double ksh = (la + lb) / (la / ksa + lb / ksb);
  const double kra = vg_k(a, ha, ksa) / ksa;
  const double krb = vg_k(b, hb, ksb) / ksb;
  return ksh * 0.5 * (kra + krb);
}

double oracle_vg_theta(double a, double n, double ts, double tr, double aev, double h) {
  soil_t s = {a, n, ts, tr, aev};
  return vg_theta(s, h);
}
double oracle_vg_head(double a, double n, double ts, double tr, double aev, double wc) {
  soil_t s = {a, n, ts, tr, aev};
  return vg_head(s, wc);
}
double oracle_vg_capacity(double a, double n, double ts, double tr, double aev, double h) {
  soil_t s = {a, n, ts, tr, aev};
  return vg_cap(s, h);
}
double oracle_vg_conductivity(double a, double n, double ts, double tr, double aev, double h,
                              double ks) {
  soil_t s = {a, n, ts, tr, aev};
  return vg_k(s, h, ks);
}
double oracle_vg_dkdtheta(double a, double n, double ts, double tr, double aev, double wc,
                          double ks) {
  soil_t s = {a, n, ts, tr, aev};
  return vg_dkdtheta(s, wc, ks);
}

static soil_t soil_at(const oracle_gw* s, size_t c) {
  soil_t r = {s->vga[c], s->vgn[c], s->wcs[c], s->wcr[c], s->aev[c]};
  return r;
}

static int is_head(int code) { return code == HEAD || code == HYDRO; }

/* ------------------------------------------------------------------ setup */
static void* xcalloc(size_t n, size_t sz) {
  void* p = calloc(n ? n : 1, sz);
  return p;
}

void oracle_gw_destroy(oracle_gw* s) {
  if (!s) return;
  double** dbl[] = {&s->bath, &s->dz, &s->bot, &s->ax, &s->ay, &s->sinx, &s->cosx, &s->siny,
                    &s->cosy, &s->ksx, &s->ksy, &s->ksz, &s->vga, &s->vgn, &s->wcs, &s->wcr,
                    &s->aev, &s->h, &s->hn, &s->wc, &s->wcn, &s->ch, &s->kx, &s->ky, &s->kz,
                    &s->qx, &s->qy, &s->qz, &s->vloss, &s->room, &s->sup, &s->sdown,
                    &s->wcsnap, &s->hsnap, &s->topv, &s->botv, &s->xmv, &s->xpv, &s->ymv,
                    &s->ypv, &s->vals7, &s->rhs, &s->sol, &s->eta, &s->dept, &s->seep,
                    &s->avail, &s->gain, &s->bounce, &s->qss, &s->wx, &s->wy, &s->wz,
                    &s->pcorr, &s->wvent, &s->s3, &s->s2, &s->t3, &s->t2, &s->rrho,
                    &s->rvisc, &s->rxp, &s->ryp, &s->rzp, &s->vxp, &s->vyp, &s->vzp};
  for (size_t n = 0; n < sizeof dbl / sizeof dbl[0]; ++n) free(*dbl[n]);
  free(s->ktop);
  free(s->gid);
  free(s->topc);
  free(s->botc);
  free(s->xmc);
  free(s->xpc);
  free(s->ymc);
  free(s->ypc);
  free(s->cols7);
  free(s->cmode);
  free(s);
}

/* fillEdgeGhosts2 / fillEdgeGhosts3 (TerrainMetric.cpp:17-62) and
 * mirrorEdgeGhosts (RichardsSolver.cpp:24-57): single-rank edge mirrors. */
static void mirror3(const oracle_gw* s, double* f, int nzf) {
  const int nx = s->nx, ny = s->ny;
  for (int k = 0; k < nzf; ++k) {
    for (int j = 1; j <= ny; ++j) {
      f[I2(s, j, 0) * nzf + k] = f[I2(s, j, 1) * nzf + k];
      f[I2(s, j, nx + 1) * nzf + k] = f[I2(s, j, nx) * nzf + k];
    }
    for (int i = 0; i <= nx + 1; ++i) {
      f[I2(s, 0, i) * nzf + k] = f[I2(s, 1, i) * nzf + k];
      f[I2(s, ny + 1, i) * nzf + k] = f[I2(s, ny, i) * nzf + k];
    }
  }
}

/* TerrainMetric::readBathymetry / buildRegularMesh / buildTerrainMesh /
 * buildMetrics (TerrainMetric.cpp:101-430). */
static int build_geometry(oracle_gw* s, const frehg_gw_desc* d) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  double lmin = 0.0, lmax = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      const double b = d->bath ? d->bath[(size_t)(j - 1) * nx + (i - 1)] : 0.0;
      s->bath[I2(s, j, i)] = b;
      lmin = (b < lmin) ? b : lmin;
      lmax = (b > lmax) ? b : lmax;
    }
  s->offset = (lmin < 0.0) ? -lmin : 0.0;
  lmax += s->offset;
  s->box_top = lmax;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) s->bath[I2(s, j, i)] += s->offset;
  mirror3(s, s->bath, 1);

  double total = 0.0;
  for (int k = 0; k < nz; ++k) total += d->dz_layers[k];

  if (s->follow_terrain) {
    /* buildTerrainMesh :232-293 */
    const double box_bottom = s->box_top - total;
    double incre = 0.0, w = 1.0;
    const double stretch = d->dz_stretch;
    for (int k = 0; k < nz; ++k) {
      incre += w;
      w *= stretch;
    }
    int shallow = 0;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double bath = s->bath[I2(s, j, i)];
        if (bath <= box_bottom) shallow = 1;
        double dzc = s->uniform ? d->dz_layers[0] : (bath - box_bottom) / incre;
        double bot = bath;
        for (int k = 0; k < nz; ++k) {
          if (s->uniform) dzc = d->dz_layers[k];
          bot -= dzc;
          s->dz[I3(s, j, i, k)] = dzc;
          s->bot[I3(s, j, i, k)] = bot;
          if (!s->uniform) dzc *= stretch;
        }
        s->ktop[(size_t)(j - 1) * nx + (i - 1)] = 0;
      }
    if (shallow && !s->uniform) {
      set_err("domain.follow_terrain requires every bed elevation above the box bottom");
      return FREHG_GW_EINVAL;
    }
  } else {
    /* buildRegularMesh :158-230 */
    double* bot1d = (double*)xcalloc((size_t)nz, sizeof(double));
    double level = s->box_top;
    for (int k = 0; k < nz; ++k) {
      level -= d->dz_layers[k];
      bot1d[k] = level;
    }
    int* active = (int*)xcalloc((size_t)nz, sizeof(int));
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double bath = s->bath[I2(s, j, i)];
        for (int k = 0; k < nz; ++k) {
          active[k] = 0;
          s->bot[I3(s, j, i, k)] = bot1d[k];
          s->dz[I3(s, j, i, k)] = d->dz_layers[k];
        }
        for (int k = 0; k < nz; ++k) {
          const size_t c = I3(s, j, i, k);
          const double dzk = d->dz_layers[k];
          if (s->bot[c] >= bath - 1.0e-5) {
            active[k] = 0;
            if (s->bot[c] - bath < dzk) s->bot[c] = bath;
          } else {
            active[k] = 1;
            if (bath - s->bot[c] <= dzk) {
              if (bath - s->bot[c] >= 0.25 * dzk) {
                s->dz[c] = bath - s->bot[c];
              } else if (k + 1 < nz) {
                active[k] = 0;
                s->dz[c + 1] += bath - s->bot[c];
              }
            }
          }
        }
        int top = nz;
        for (int k = 0; k < nz; ++k)
          if (active[k] == 1) {
            top = k;
            break;
          }
        s->ktop[(size_t)(j - 1) * nx + (i - 1)] = top;
      }
    free(active);
    free(bot1d);
  }
  mirror3(s, s->dz, nz);
  mirror3(s, s->bot, nz);

  /* buildMetrics :295-430 */
  for (size_t c = 0; c < s->n3; ++c) {
    s->sinx[c] = 0.0;
    s->cosx[c] = 1.0;
    s->siny[c] = 0.0;
    s->cosy[c] = 1.0;
  }
  if (s->follow_terrain) {
    for (int j = 0; j <= ny + 1; ++j)
      for (int i = 1; i <= nx - 1; ++i)
        for (int k = 0; k < nz; ++k) {
          const size_t c = I3(s, j, i, k), e = I3(s, j, i + 1, k);
          const double zc = s->bot[c] + 0.5 * s->dz[c];
          const double zp = s->bot[e] + 0.5 * s->dz[e];
          const double hd = fabs(zp - zc);
          const double dist = sqrt(hd * hd + s->dx * s->dx);
          s->sinx[c] = hd / dist;
          s->cosx[c] = s->dx / dist;
        }
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 0; i <= nx + 1; ++i)
        for (int k = 0; k < nz; ++k) {
          const size_t c = I3(s, j, i, k), n = I3(s, j + 1, i, k);
          const double zc = s->bot[c] + 0.5 * s->dz[c];
          const double zp = s->bot[n] + 0.5 * s->dz[n];
          const double hd = fabs(zp - zc);
          const double dist = sqrt(hd * hd + s->dy * s->dy);
          s->siny[c] = hd / dist;
          s->cosy[c] = s->dy / dist;
        }
  }
  for (int j = 0; j <= ny + 1; ++j)
    for (int i = 0; i <= nx + 1; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = I3(s, j, i, k);
        if (s->follow_terrain) {
          const double dze = (i <= nx) ? s->dz[I3(s, j, i + 1, k)] : s->dz[c];
          const double dzn = (j <= ny) ? s->dz[I3(s, j + 1, i, k)] : s->dz[c];
          s->ax[c] = 0.5 * (s->dz[c] + dze) * s->cosx[c] * s->dy;
          s->ay[c] = 0.5 * (s->dz[c] + dzn) * s->cosy[c] * s->dx;
        } else {
          s->ax[c] = s->dy * s->dz[c];
          s->ay[c] = s->dx * s->dz[c];
        }
      }
  return FREHG_GW_OK;
}

/* Grid::buildGlobalIds (Grid.cpp:160-238): compressed ids, (j, i, k) order. */
static void build_gids(oracle_gw* s) {
  for (size_t c = 0; c < s->n3; ++c) s->gid[c] = -1;
  long long next = 0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      const int kt = s->ktop[(size_t)(j - 1) * s->nx + (i - 1)];
      for (int k = kt; k < s->nz; ++k) s->gid[I3(s, j, i, k)] = (int)next++;
    }
  s->nactive = next;
}

oracle_gw* oracle_gw_create(const frehg_gw_desc* d) {
  g_err[0] = 0;
  if (!d || d->abi_version != FREHG_GW_ABI_VERSION || d->nx < 1 || d->ny < 1 || d->nz < 1 ||
      !d->dz_layers || !d->ksx || !d->ksy || !d->ksz || !d->vg_alpha || !d->vg_n ||
      !d->theta_s || !d->theta_r || !d->aev || !d->top_code || !d->bot_code || !d->xm_code ||
      !d->xp_code || !d->ym_code || !d->yp_code) {
    set_err("oracle_gw_create: invalid descriptor");
    return NULL;
  }
  if (!d->saturated_contact_head) {
    set_err("oracle_gw_create: saturated_contact legacy is order-dependent; not restated");
    return NULL;
  }
  oracle_gw* s = (oracle_gw*)xcalloc(1, sizeof(oracle_gw));
  s->nx = d->nx;
  s->ny = d->ny;
  s->nz = d->nz;
  s->n2 = (size_t)(d->ny + 2) * (size_t)(d->nx + 2);
  s->n3 = s->n2 * (size_t)d->nz;
  s->n3f = s->n2 * (size_t)(d->nz + 1);
  s->dx = d->dx;
  s->dy = d->dy;
  s->az = d->dx * d->dy;
  s->follow_terrain = d->follow_terrain;
  s->uniform = d->terrain_uniform;
  s->ss = d->specific_storage;
  s->full3d = d->use_full3d;
  s->pc = d->pc_consistent;
  s->harm = d->pc_consistent && d->face_harmonic;
  s->off = d->reallocation_off;
  s->redistribute = d->surplus_redistribute;
  s->schead = d->saturated_contact_head;
  s->dt_min = d->dt_min;
  s->dt_max = d->dt_max;
  s->dq_grow = d->dq_grow;
  s->dq_shrink = d->dq_shrink;
  s->co_max = d->courant_max;
  s->dtg_next = d->dt_init;
  s->rtol = d->rtol;
  s->atol = d->atol;
  s->maxit = d->max_iterations;

  const size_t n2 = s->n2, n3 = s->n3, n3f = s->n3f;
  s->bath = xcalloc(n2, sizeof(double));
  double** f3[] = {&s->dz, &s->bot, &s->ax, &s->ay, &s->sinx, &s->cosx, &s->siny, &s->cosy,
                   &s->ksx, &s->ksy, &s->ksz, &s->vga, &s->vgn, &s->wcs, &s->wcr, &s->aev,
                   &s->h, &s->hn, &s->wc, &s->wcn, &s->ch, &s->kx, &s->ky, &s->qx, &s->qy,
                   &s->vloss, &s->room, &s->sup, &s->sdown, &s->wcsnap, &s->hsnap};
  for (size_t n = 0; n < sizeof f3 / sizeof f3[0]; ++n) *f3[n] = xcalloc(n3, sizeof(double));
  s->kz = xcalloc(n3f, sizeof(double));
  s->qz = xcalloc(n3f, sizeof(double));
  /* the ratio fields start at 1 (RichardsSolver.cpp:141-150) */
  double** r3[] = {&s->rrho, &s->rvisc, &s->rxp, &s->ryp, &s->vxp, &s->vyp};
  for (size_t n = 0; n < 6; ++n) {
    *r3[n] = xcalloc(n3, sizeof(double));
    for (size_t c = 0; c < n3; ++c) (*r3[n])[c] = 1.0;
  }
  s->rzp = xcalloc(n3f, sizeof(double));
  s->vzp = xcalloc(n3f, sizeof(double));
  for (size_t f = 0; f < n3f; ++f) s->rzp[f] = s->vzp[f] = 1.0;
  s->ktop = xcalloc((size_t)d->nx * d->ny, sizeof(int));
  s->gid = xcalloc(n3, sizeof(int));
  int** c2[] = {&s->topc, &s->botc, &s->xmc, &s->xpc, &s->ymc, &s->ypc};
  for (size_t n = 0; n < 6; ++n) *c2[n] = xcalloc(n2, sizeof(int));
  double** v2[] = {&s->topv, &s->botv, &s->xmv, &s->xpv, &s->ymv, &s->ypv};
  for (size_t n = 0; n < 6; ++n) *v2[n] = xcalloc(n2, sizeof(double));

  if (build_geometry(s, d) != FREHG_GW_OK) {
    oracle_gw_destroy(s);
    return NULL;
  }
  build_gids(s);

  /* stageSoil (RichardsSolver.cpp:261-328): interior values, mirrored ghosts. */
  const double* src[] = {d->ksx, d->ksy, d->ksz, d->vg_alpha, d->vg_n, d->theta_s, d->theta_r,
                         d->aev};
  double* dst[] = {s->ksx, s->ksy, s->ksz, s->vga, s->vgn, s->wcs, s->wcr, s->aev};
  for (int f = 0; f < 8; ++f) {
    for (int j = 1; j <= s->ny; ++j)
      for (int i = 1; i <= s->nx; ++i)
        for (int k = 0; k < s->nz; ++k)
          dst[f][I3(s, j, i, k)] =
              src[f][((size_t)(j - 1) * s->nx + (i - 1)) * s->nz + (size_t)k];
    mirror3(s, dst[f], s->nz);
  }

  /* buildBoundaryLists (RichardsSolver.cpp:429-524): static markers. */
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      s->topc[I2(s, j, i)] = d->top_code[(size_t)(j - 1) * s->nx + (i - 1)];
      s->botc[I2(s, j, i)] = d->bot_code[(size_t)(j - 1) * s->nx + (i - 1)];
    }
  for (int j = 1; j <= s->ny; ++j) {
    s->xmc[I2(s, j, 1)] = d->xm_code[j - 1];
    s->xpc[I2(s, j, s->nx)] = d->xp_code[j - 1];
  }
  for (int i = 1; i <= s->nx; ++i) {
    s->ymc[I2(s, 1, i)] = d->ym_code[i - 1];
    s->ypc[I2(s, s->ny, i)] = d->yp_code[i - 1];
  }

  s->vals7 = xcalloc((size_t)s->nactive * 7, sizeof(double));
  s->cols7 = xcalloc((size_t)s->nactive * 7, sizeof(long));
  s->rhs = xcalloc((size_t)s->nactive, sizeof(double));
  s->sol = xcalloc((size_t)s->nactive, sizeof(double));
  /* buildCooPattern (RichardsSolver.cpp:680-727): [diag, xm, xp, ym, yp, zm, zp]. */
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const int row = s->gid[I3(s, j, i, k)];
        if (row < 0) continue;
        long* c = s->cols7 + 7 * (size_t)row;
        c[0] = row;
        c[1] = s->gid[I3(s, j, i - 1, k)];
        c[2] = s->gid[I3(s, j, i + 1, k)];
        c[3] = s->gid[I3(s, j - 1, i, k)];
        c[4] = s->gid[I3(s, j + 1, i, k)];
        c[5] = (k > 0) ? s->gid[I3(s, j, i, k - 1)] : -1;
        c[6] = (k + 1 < s->nz) ? s->gid[I3(s, j, i, k + 1)] : -1;
      }
  return s;
}

/* updateBoundaryValues (RichardsSolver.cpp:526-566); hydrostatic stages move
 * into the offset frame (:529-533). */
int oracle_gw_set_bc_values(oracle_gw* s, const double* top, const double* bot,
                            const double* xm, const double* xp, const double* ym,
                            const double* yp) {
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      const size_t c = I2(s, j, i), q = (size_t)(j - 1) * s->nx + (i - 1);
      if (top) s->topv[c] = top[q] + (s->topc[c] == HYDRO ? s->offset : 0.0);
      if (bot) s->botv[c] = bot[q] + (s->botc[c] == HYDRO ? s->offset : 0.0);
    }
  for (int j = 1; j <= s->ny; ++j) {
    const size_t w = I2(s, j, 1), e = I2(s, j, s->nx);
    if (xm) s->xmv[w] = xm[j - 1] + (s->xmc[w] == HYDRO ? s->offset : 0.0);
    if (xp) s->xpv[e] = xp[j - 1] + (s->xpc[e] == HYDRO ? s->offset : 0.0);
  }
  for (int i = 1; i <= s->nx; ++i) {
    const size_t so = I2(s, 1, i), no = I2(s, s->ny, i);
    if (ym) s->ymv[so] = ym[i - 1] + (s->ymc[so] == HYDRO ? s->offset : 0.0);
    if (yp) s->ypv[no] = yp[i - 1] + (s->ypc[no] == HYDRO ? s->offset : 0.0);
  }
  return FREHG_GW_OK;
}

/* ------------------------------------------------------------------ ghosts */
/* enforceHeadBc + ghostHead (Predictor.cpp:66-87, 757-817): hydrostatic edges
 * scale by the edge face's density ratio r.  In a coupled run a hydrostatic
 * stage above the edge column's bed follows the live surface there:
 * (bed - zc) r + depth (depth r on the plus sides). */
static double ghost_head(const oracle_gw* s, int code, double value, double interior, double zc,
                         size_t col, double r, int plus) {
  if (code == HEAD) return value;
  if (code == HYDRO) {
    if (s->cpl && value > s->bath[col]) {
      const double hydro = (s->bath[col] - zc) * r;
      return plus ? hydro + s->dept[col] * r : hydro + s->dept[col];
    }
    return (value - zc) * r;
  }
  return interior;
}

static void enforce_head_bc(oracle_gw* s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int j = 1; j <= ny; ++j)
    for (int k = 0; k < nz; ++k) {
      size_t c = I3(s, j, 1, k);
      double zc = s->bot[c] + 0.5 * s->dz[c];
      s->h[I3(s, j, 0, k)] = ghost_head(s, s->xmc[I2(s, j, 1)], s->xmv[I2(s, j, 1)], s->h[c], zc,
                                        I2(s, j, 1), s->rxp[I3(s, j, 0, k)], 0);
      c = I3(s, j, nx, k);
      zc = s->bot[c] + 0.5 * s->dz[c];
      s->h[I3(s, j, nx + 1, k)] = ghost_head(s, s->xpc[I2(s, j, nx)], s->xpv[I2(s, j, nx)],
                                             s->h[c], zc, I2(s, j, nx), s->rxp[c], 1);
    }
  for (int i = 1; i <= nx; ++i)
    for (int k = 0; k < nz; ++k) {
      size_t c = I3(s, 1, i, k);
      double zc = s->bot[c] + 0.5 * s->dz[c];
      s->h[I3(s, 0, i, k)] = ghost_head(s, s->ymc[I2(s, 1, i)], s->ymv[I2(s, 1, i)], s->h[c], zc,
                                        I2(s, 1, i), s->ryp[I3(s, 0, i, k)], 0);
      c = I3(s, ny, i, k);
      zc = s->bot[c] + 0.5 * s->dz[c];
      s->h[I3(s, ny + 1, i, k)] = ghost_head(s, s->ypc[I2(s, ny, i)], s->ypv[I2(s, ny, i)],
                                             s->h[c], zc, I2(s, ny, i), s->ryp[c], 1);
    }
}

/* updateBaroclinicFaces (Baroclinic.cpp:46-186): with an attached scalar, the
 * cell ratios over the whole halo box, then their face means between active
 * flanks.  Minus-side edge faces average the interior cell with its ghost (a
 * head edge takes the ghost's ratio one-sided), plus-side edge faces take the
 * ghost's ratio under a head edge and stay 1 otherwise, the face above a
 * column's top cell averages it with the surface scalar's ratio (coupled) or
 * its own (uncoupled), the bottom boundary face stays 1. */
static void update_baroclinic(oracle_gw* s) {
  if (!s->baro || (!s->saline && !s->thermal)) return;
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double bs = s->beta_s, bsv = s->beta_sv, bt = s->beta_t, t0 = s->t_ref;
  for (size_t c = 0; c < s->n3; ++c) {
    const double sv = s->saline ? s->s3[c] : 0.0;
    const double dtv = s->thermal ? s->t3[c] - t0 : 0.0;
    s->rrho[c] = 1.0 + bs * sv - bt * dtv;
    s->rvisc[c] = 1.0 / (1.0 + bsv * sv);
  }
  for (int j = 1; j <= ny; ++j) /* x faces, slot i = face i+1/2 */
    for (int i = 0; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        double rr = 1.0, rv = 1.0;
        if (i == 0) {
          if (s->gid[I3(s, j, 1, k)] >= 0) {
            const size_t a = I3(s, j, 1, k), g = I3(s, j, 0, k);
            if (is_head(s->xmc[I2(s, j, 1)])) {
              rr = s->rrho[g];
              rv = s->rvisc[g];
            } else {
              rr = 0.5 * (s->rrho[a] + s->rrho[g]);
              rv = 0.5 * (s->rvisc[a] + s->rvisc[g]);
            }
          }
        } else if (i == nx) {
          if (s->gid[I3(s, j, i, k)] >= 0 && is_head(s->xpc[I2(s, j, i)])) {
            rr = s->rrho[I3(s, j, i + 1, k)];
            rv = s->rvisc[I3(s, j, i + 1, k)];
          }
        } else if (s->gid[I3(s, j, i, k)] >= 0 && s->gid[I3(s, j, i + 1, k)] >= 0) {
          const size_t a = I3(s, j, i, k), b = I3(s, j, i + 1, k);
          rr = 0.5 * (s->rrho[a] + s->rrho[b]);
          rv = 0.5 * (s->rvisc[a] + s->rvisc[b]);
        }
        s->rxp[I3(s, j, i, k)] = rr;
        s->vxp[I3(s, j, i, k)] = rv;
      }
  for (int j = 0; j <= ny; ++j) /* y faces */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        double rr = 1.0, rv = 1.0;
        if (j == 0) {
          if (s->gid[I3(s, 1, i, k)] >= 0) {
            const size_t a = I3(s, 1, i, k), g = I3(s, 0, i, k);
            if (is_head(s->ymc[I2(s, 1, i)])) {
              rr = s->rrho[g];
              rv = s->rvisc[g];
            } else {
              rr = 0.5 * (s->rrho[a] + s->rrho[g]);
              rv = 0.5 * (s->rvisc[a] + s->rvisc[g]);
            }
          }
        } else if (j == ny) {
          if (s->gid[I3(s, j, i, k)] >= 0 && is_head(s->ypc[I2(s, j, i)])) {
            rr = s->rrho[I3(s, j + 1, i, k)];
            rv = s->rvisc[I3(s, j + 1, i, k)];
          }
        } else if (s->gid[I3(s, j, i, k)] >= 0 && s->gid[I3(s, j + 1, i, k)] >= 0) {
          const size_t a = I3(s, j, i, k), b = I3(s, j + 1, i, k);
          rr = 0.5 * (s->rrho[a] + s->rrho[b]);
          rv = 0.5 * (s->rvisc[a] + s->rvisc[b]);
        }
        s->ryp[I3(s, j, i, k)] = rr;
        s->vyp[I3(s, j, i, k)] = rv;
      }
  for (int j = 1; j <= ny; ++j) /* z faces, plane k above cell k */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k <= nz; ++k) {
        const int below = (k < nz) && s->gid[I3(s, j, i, k)] >= 0;
        const int above = (k >= 1) && s->gid[I3(s, j, i, k - 1)] >= 0;
        double rr = 1.0, rv = 1.0;
        if (below && above) {
          const size_t a = I3(s, j, i, k - 1), b = I3(s, j, i, k);
          rr = 0.5 * (s->rrho[a] + s->rrho[b]);
          rv = 0.5 * (s->rvisc[a] + s->rvisc[b]);
        } else if (below) {
          const size_t b = I3(s, j, i, k), col = I2(s, j, i);
          const double sg = s->saline ? (s->cpl ? s->s2[col] : s->s3[b]) : 0.0;
          const double tg = s->thermal ? (s->cpl ? s->t2[col] : s->t3[b]) - t0 : 0.0;
          rr = 0.5 * (s->rrho[b] + 1.0 + bs * sg - bt * tg);
          rv = 0.5 * (s->rvisc[b] + 1.0 / (1.0 + bsv * sg));
        }
        s->rzp[IF(s, j, i, k)] = rr;
        s->vzp[IF(s, j, i, k)] = rv;
      }
}

/* enforceMoistureBc (Corrector.cpp:709-756). */
static void enforce_moisture_bc(oracle_gw* s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int j = 1; j <= ny; ++j)
    for (int k = 0; k < nz; ++k) {
      s->wc[I3(s, j, 0, k)] =
          is_head(s->xmc[I2(s, j, 1)]) ? s->wcs[I3(s, j, 1, k)] : s->wc[I3(s, j, 1, k)];
      s->wc[I3(s, j, nx + 1, k)] =
          is_head(s->xpc[I2(s, j, nx)]) ? s->wcs[I3(s, j, nx, k)] : s->wc[I3(s, j, nx, k)];
    }
  for (int i = 1; i <= nx; ++i)
    for (int k = 0; k < nz; ++k) {
      s->wc[I3(s, 0, i, k)] =
          is_head(s->ymc[I2(s, 1, i)]) ? s->wcs[I3(s, 1, i, k)] : s->wc[I3(s, 1, i, k)];
      s->wc[I3(s, ny + 1, i, k)] =
          is_head(s->ypc[I2(s, ny, i)]) ? s->wcs[I3(s, ny, i, k)] : s->wc[I3(s, ny, i, k)];
    }
}

/* applyInitialConditions (RichardsSolver.cpp:331-427). */
int oracle_gw_init_state(oracle_gw* s, int form, double constant, const double* field) {
  for (size_t c = 0; c < s->n3; ++c) {
    s->h[c] = 0.0;
    s->wc[c] = 0.0;
  }
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t c = I3(s, j, i, k);
        const soil_t so = soil_at(s, c);
        const double zc = s->bot[c] + 0.5 * s->dz[c];
        const size_t col = (size_t)(j - 1) * s->nx + (i - 1);
        double value = constant;
        if (field) value = (form == FREHG_GW_IC_WATER_TABLE) ? field[col] : field[col * s->nz + k];
        double h = 0.0, wc = 0.0;
        if (form == FREHG_GW_IC_MOISTURE) {
          wc = value;
          h = (wc >= so.ts) ? (s->bath[I2(s, j, i)] - zc) : vg_head(so, wc);
        } else if (form == FREHG_GW_IC_HEAD) {
          h = value;
          wc = vg_theta(so, h);
        } else if (form == FREHG_GW_IC_WATER_TABLE) {
          h = (value + s->offset) - zc;
          wc = vg_theta(so, h);
        } else {
          set_err("oracle_gw_init_state: unknown form");
          return FREHG_GW_EINVAL;
        }
        s->h[c] = h;
        s->wc[c] = wc;
      }
  enforce_head_bc(s);
  enforce_moisture_bc(s);
  memcpy(s->hn, s->h, s->n3 * sizeof(double));
  memcpy(s->wcn, s->wc, s->n3 * sizeof(double));
  s->have_state = 1;
  return FREHG_GW_OK;
}

/* A restart read followed by refreshDerivedState (RichardsSolver.cpp:880-890). */
int oracle_gw_set_state(oracle_gw* s, const double* head, const double* wc) {
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t q = ((size_t)(j - 1) * s->nx + (i - 1)) * s->nz + (size_t)k;
        s->h[I3(s, j, i, k)] = head[q];
        s->wc[I3(s, j, i, k)] = wc[q];
      }
  update_baroclinic(s);
  enforce_head_bc(s);
  enforce_moisture_bc(s);
  memcpy(s->hn, s->h, s->n3 * sizeof(double));
  memcpy(s->wcn, s->wc, s->n3 * sizeof(double));
  s->have_state = 1;
  return FREHG_GW_OK;
}

/* ------------------------------------------------------------------ predictor */
/* computeFaceConductivityImpl<PC, HARM> (Predictor.cpp:105-386). */
/* classifyCoupledTopImpl<PC> (Corrector.cpp:55-115): per column, 1 = a wet
 * surface whose saturated demand the window's water funds (Dirichlet top),
 * 2 = a wet surface it cannot fund (supply-limited flux), 3 = (consistent
 * form) a dry surface over a top cell pressurized past dz/2, 0 = dry. */
static void classify_coupled_top(oracle_gw* s, double dtg) {
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      const size_t col = I2(s, j, i);
      int kt = s->ktop[(size_t)(j - 1) * s->nx + (i - 1)];
      if (kt >= s->nz) kt = -1;
      if (kt < 0 || s->dept[col] <= 0.0) {
        if (s->pc && kt >= 0) {
          const size_t c = I3(s, j, i, kt);
          if (s->h[c] > s->rzp[IF(s, j, i, kt)] * 0.5 * s->dz[c]) {
            s->cmode[col] = 3;
            continue;
          }
        }
        s->cmode[col] = 0;
        continue;
      }
      const size_t c = I3(s, j, i, kt);
      const double ks = s->ksz[c];
      const double qEst = 2.0 * ks * (s->h[c] - s->dept[col]) / s->dz[c] - ks;
      s->cmode[col] = (qEst < 0.0 && -qEst * dtg > s->avail[col]) ? 2 : 1;
    }
}

static void face_conductivity(oracle_gw* s) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  for (int j = 1; j <= ny; ++j) /* gw_face_k_x */
    for (int i = 0; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t a = I3(s, j, i, k), b = I3(s, j, i + 1, k);
        if (s->harm) {
          s->kx[a] = face_harm(soil_at(s, a), s->h[a], s->ksx[a], 1.0, soil_at(s, b), s->h[b],
                               s->ksx[b], 1.0);
        } else {
          const double km = vg_k(soil_at(s, a), s->h[a], s->ksx[a]);
          const double kp = vg_k(soil_at(s, b), s->h[b], s->ksx[b]);
          s->kx[a] = 0.5 * (km + kp);
        }
      }
  for (int j = 0; j <= ny; ++j) /* gw_face_k_y */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t a = I3(s, j, i, k), b = I3(s, j + 1, i, k);
        if (s->harm) {
          s->ky[a] = face_harm(soil_at(s, a), s->h[a], s->ksy[a], 1.0, soil_at(s, b), s->h[b],
                               s->ksy[b], 1.0);
        } else {
          const double km = vg_k(soil_at(s, a), s->h[a], s->ksy[a]);
          const double kp = vg_k(soil_at(s, b), s->h[b], s->ksy[b]);
          s->ky[a] = 0.5 * (km + kp);
        }
      }
  for (int j = 1; j <= ny; ++j) /* gw_face_k_z */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k <= nz; ++k) {
        const size_t f = IF(s, j, i, k);
        if (k == 0) {
          s->kz[f] = 0.0;
          continue;
        }
        if (k == nz) {
          const size_t c = I3(s, j, i, nz - 1);
          s->kz[f] = (s->botc[I2(s, j, i)] == NOFLUX) ? 0.0 : vg_k(soil_at(s, c), s->h[c], s->ksz[c]);
          continue;
        }
        const size_t lo = I3(s, j, i, k), up = I3(s, j, i, k - 1);
        if (s->gid[lo] >= 0 && s->gid[up] < 0) {
          s->kz[f] = vg_k(soil_at(s, lo), s->h[lo], s->ksz[lo]);
          continue;
        }
        if (s->gid[up] < 0) {
          s->kz[f] = 0.0;
          continue;
        }
        if (s->harm) {
          s->kz[f] = face_harm(soil_at(s, up), s->h[up], s->ksz[up], s->dz[up], soil_at(s, lo),
                               s->h[lo], s->ksz[lo], s->dz[lo]);
        } else {
          const double km = vg_k(soil_at(s, up), s->h[up], s->ksz[up]);
          const double kp = vg_k(soil_at(s, lo), s->h[lo], s->ksz[lo]);
          s->kz[f] = 0.5 * (km + kp);
        }
      }
  /* gw_face_k_edges: sealed no-flux edges, interior K at head edges. */
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = I3(s, j, i, k);
        int code;
        if (i == 1) {
          code = s->xmc[I2(s, j, i)];
          if (code == NOFLUX) s->kx[I3(s, j, i - 1, k)] = 0.0;
          else if (is_head(code)) s->kx[I3(s, j, i - 1, k)] = vg_k(soil_at(s, c), s->h[c], s->ksx[c]);
        }
        if (i == nx) {
          code = s->xpc[I2(s, j, i)];
          if (code == NOFLUX) s->kx[c] = 0.0;
          else if (is_head(code)) s->kx[c] = vg_k(soil_at(s, c), s->h[c], s->ksx[c]);
        }
        if (j == 1) {
          code = s->ymc[I2(s, j, i)];
          if (code == NOFLUX) s->ky[I3(s, j - 1, i, k)] = 0.0;
          else if (is_head(code)) s->ky[I3(s, j - 1, i, k)] = vg_k(soil_at(s, c), s->h[c], s->ksy[c]);
        }
        if (j == ny) {
          code = s->ypc[I2(s, j, i)];
          if (code == NOFLUX) s->ky[c] = 0.0;
          else if (is_head(code)) s->ky[c] = vg_k(soil_at(s, c), s->h[c], s->ksy[c]);
        }
      }
  /* gw_face_k_top (Predictor.cpp:278-310): uncoupled, head -> Ksz, no-flux
   * -> 0, otherwise K(h); coupled, a wet surface gives Ksz (consistent) or
   * the mean of Ksz and K(h) (legacy), a dry one K(h). */
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = I3(s, j, i, k);
        const int top = s->gid[c] >= 0 && (k == 0 || s->gid[c - 1] < 0);
        if (!top) continue;
        const double own = vg_k(soil_at(s, c), s->h[c], s->ksz[c]);
        if (s->cpl) {
          if (s->pc) s->kz[IF(s, j, i, k)] = (s->dept[I2(s, j, i)] > 0.0) ? s->ksz[c] : own;
          else s->kz[IF(s, j, i, k)] = (s->dept[I2(s, j, i)] > 0.0) ? 0.5 * (s->ksz[c] + own) : own;
          continue;
        }
        const int code = s->topc[I2(s, j, i)];
        s->kz[IF(s, j, i, k)] = (code == HEAD) ? s->ksz[c] : (code == NOFLUX ? 0.0 : own);
      }
  if (!s->full3d) { /* gw_face_k_full3d_x/_y */
    for (int j = 1; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i)
        for (int k = 0; k < nz; ++k) {
          const size_t a = I3(s, j, i, k), b = I3(s, j, i + 1, k);
          if ((s->gid[a] >= 0 && s->wc[a] < s->wcs[a]) || (s->gid[b] >= 0 && s->wc[b] < s->wcs[b]))
            s->kx[a] = 0.0;
        }
    for (int j = 0; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        for (int k = 0; k < nz; ++k) {
          const size_t a = I3(s, j, i, k), b = I3(s, j + 1, i, k);
          if ((s->gid[a] >= 0 && s->wc[a] < s->wcs[a]) || (s->gid[b] >= 0 && s->wc[b] < s->wcs[b]))
            s->ky[a] = 0.0;
        }
  }
  /* gw_face_k_seal_x/_y/_z: faces flanked by an inactive in-domain cell, last. */
  for (int j = 1; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const int ina = (i >= 1 && i <= nx) && s->gid[I3(s, j, i, k)] < 0;
        const int inb = (i + 1 >= 1 && i + 1 <= nx) && s->gid[I3(s, j, i + 1, k)] < 0;
        if (ina || inb) s->kx[I3(s, j, i, k)] = 0.0;
      }
  for (int j = 0; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const int ina = (j >= 1 && j <= ny) && s->gid[I3(s, j, i, k)] < 0;
        const int inb = (j + 1 >= 1 && j + 1 <= ny) && s->gid[I3(s, j + 1, i, k)] < 0;
        if (ina || inb) s->ky[I3(s, j, i, k)] = 0.0;
      }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k <= nz; ++k) {
        const int above = (k >= 1) && s->gid[I3(s, j, i, k - 1)] < 0;
        const int below = (k < nz) && s->gid[I3(s, j, i, k)] < 0;
        if (above || below) s->kz[IF(s, j, i, k)] = 0.0;
      }
}

/* assembleSystemImpl<PC> (Predictor.cpp:400-698), no ET; the coupled top's
 * Dirichlet leg and RHS by exchange mode (:527-547, :627-674). */
static void assemble(oracle_gw* s, double dtg) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double dx = s->dx, dy = s->dy, az = s->az, ss = s->ss;
  for (int j = 1; j <= ny; ++j) /* gw_capacity */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = I3(s, j, i, k);
        s->ch[c] = vg_cap(soil_at(s, c), s->hn[c]);
      }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = I3(s, j, i, k);
        const int row = s->gid[c];
        if (row < 0) continue;
        const size_t cw = I3(s, j, i - 1, k), ce = I3(s, j, i + 1, k);
        const size_t cs = I3(s, j - 1, i, k), cn = I3(s, j + 1, i, k);
        const size_t col = I2(s, j, i);
        const int east = (i == nx), west = (i == 1), north = (j == ny), south = (j == 1);
        const int top = (k == 0) || (s->gid[c - 1] < 0);
        const double volume = az * s->dz[c];
        double gxp = -s->kx[c] * dtg * s->rxp[c] * s->vxp[c] * s->cosx[c] / (dx * dx) *
                     (s->ax[c] * dx);
        double gxm = -s->kx[cw] * dtg * s->rxp[cw] * s->vxp[cw] * s->cosx[cw] / (dx * dx) *
                     (s->ax[cw] * dx);
        double gyp = -s->ky[c] * dtg * s->ryp[c] * s->vyp[c] * s->cosy[c] / (dy * dy) *
                     (s->ay[c] * dy);
        double gym = -s->ky[cs] * dtg * s->ryp[cs] * s->vyp[cs] * s->cosy[cs] / (dy * dy) *
                     (s->ay[cs] * dy);
        if (east && is_head(s->xpc[col])) gxp *= 2.0;
        if (west && is_head(s->xmc[col])) gxm *= 2.0;
        if (north && is_head(s->ypc[col])) gyp *= 2.0;
        if (south && is_head(s->ymc[col])) gym *= 2.0;
        double dzf = (k == nz - 1) ? 0.5 * s->dz[c] : 0.5 * (s->dz[c] + s->dz[c + 1]);
        const size_t fp = IF(s, j, i, k + 1), fm = IF(s, j, i, k);
        const double gzp = -s->kz[fp] * dtg * s->rzp[fp] * s->vzp[fp] / (s->dz[c] * dzf) * volume;
        dzf = top ? 0.5 * s->dz[c] : 0.5 * (s->dz[c] + s->dz[c - 1]);
        const double gzm = -s->kz[fm] * dtg * s->rzp[fm] * s->vzp[fm] / (s->dz[c] * dzf) * volume;

        const double storage = (s->ch[c] + ss * s->wcn[c] / s->wcs[c]) * s->rrho[c];
        double gct = storage * volume - (gxp + gxm + gyp + gym);
        if (east && s->xpc[col] == FLUX) gct += gxp;
        if (west && s->xmc[col] == FLUX) gct += gxm;
        if (north && s->ypc[col] == FLUX) gct += gyp;
        if (south && s->ymc[col] == FLUX) gct += gym;
        if (!(k == nz - 1 && s->botc[col] != HEAD)) gct -= gzp;
        if (top) {
          int dirichlet = s->cpl ? (s->cmode[col] == 1) : (s->topc[col] == HEAD);
          if (s->pc) dirichlet = dirichlet || (s->cpl && s->cmode[col] == 3);
          if (dirichlet) gct -= gzm;
        } else {
          gct -= gzm;
        }

        double b = storage * s->hn[c] * volume;
        b -= dtg * volume * s->kz[fp] * s->rzp[fp] * s->rzp[fp] * s->vzp[fp] / s->dz[c];
        b += dtg * volume * s->kz[fm] * s->rzp[fm] * s->rzp[fm] * s->vzp[fm] / s->dz[c];
        if (s->follow_terrain && s->pc) {
          /* the along-layer terms in the z-gravity form r^2 v (consistent) */
          double sg = (s->bot[ce] > s->bot[c]) ? 1.0 : -1.0;
          b += sg * dtg * s->ax[c] * s->kx[c] * s->rxp[c] * s->rxp[c] * s->vxp[c] * s->sinx[c];
          sg = (s->bot[c] > s->bot[cw]) ? -1.0 : 1.0;
          b += sg * dtg * s->ax[cw] * s->kx[cw] * s->rxp[cw] * s->rxp[cw] * s->vxp[cw] *
               s->sinx[cw];
          sg = (s->bot[cn] > s->bot[c]) ? 1.0 : -1.0;
          b += sg * dtg * s->ay[c] * s->ky[c] * s->ryp[c] * s->ryp[c] * s->vyp[c] * s->siny[c];
          sg = (s->bot[c] > s->bot[cs]) ? -1.0 : 1.0;
          b += sg * dtg * s->ay[cs] * s->ky[cs] * s->ryp[cs] * s->ryp[cs] * s->vyp[cs] *
               s->siny[cs];
        } else if (s->follow_terrain) {
          double sg = (s->bot[ce] > s->bot[c]) ? 1.0 : -1.0;
          b += sg * dtg * s->ax[c] * s->kx[c] * s->sinx[c];
          sg = (s->bot[c] > s->bot[cw]) ? -1.0 : 1.0;
          b += sg * dtg * s->ax[cw] * s->kx[cw] * s->sinx[cw];
          sg = (s->bot[cn] > s->bot[c]) ? 1.0 : -1.0;
          b += sg * dtg * s->ay[c] * s->ky[c] * s->siny[c];
          sg = (s->bot[c] > s->bot[cs]) ? -1.0 : 1.0;
          b += sg * dtg * s->ay[cs] * s->ky[cs] * s->siny[cs];
        }
        if (east) {
          if (s->xpc[col] == FLUX) b += s->rxp[c] * s->ax[c] * s->xpv[col] * dtg;
          else b -= gxp * s->hn[ce];
        }
        if (west) {
          if (s->xmc[col] == FLUX) b += s->rxp[cw] * s->ax[cw] * s->xmv[col] * dtg;
          else b -= gxm * s->hn[cw];
        }
        if (north) {
          if (s->ypc[col] == FLUX) b += s->ryp[c] * s->ay[c] * s->ypv[col] * dtg;
          else b -= gyp * s->hn[cn];
        }
        if (south) {
          if (s->ymc[col] == FLUX) b += s->ryp[cs] * s->ay[cs] * s->ymv[col] * dtg;
          else b -= gym * s->hn[cs];
        }
        if (k == nz - 1) {
          if (s->botc[col] == FLUX) {
            const size_t fb = IF(s, j, i, nz);
            b += dtg * s->rzp[fb] * volume *
                 (s->botv[col] + s->kz[fb] * s->rzp[fb] * s->vzp[fb]) / s->dz[c];
          } else if (s->botc[col] == HEAD) {
            b -= gzp * s->botv[col];
          }
        }
        if (top && s->cpl) {
          const int m = s->cmode[col];
          if (m == 1) {
            b -= gzm * s->dept[col];
          } else if (s->pc && m == 3) {
            /* the ghost head is 0: the leg is in the diagonal only */
          } else if (m == 2) {
            const double roomTop = fmax(0.0, (0.9999 * s->wcs[c] - s->wcn[c]) * s->dz[c]);
            const double take = fmin(s->avail[col], roomTop);
            const double qSupply = -take / dtg;
            b += -dtg * s->rzp[fm] * volume * (qSupply + s->kz[fm] * s->rzp[fm] * s->vzp[fm]) /
                 s->dz[c];
          } else {
            double qtop = 0.0;
            if (s->topc[col] == FLUX) {
              const double v = s->topv[col];
              if ((v > 0.0 && s->wcn[c] < s->wcs[c]) || (v < 0.0 && s->wcn[c] > s->wcr[c])) qtop = v;
            }
            b += -dtg * s->rzp[fm] * volume * (qtop + s->kz[fm] * s->rzp[fm] * s->vzp[fm]) /
                 s->dz[c];
          }
        } else if (top) {
          if (s->topc[col] == HEAD) {
            b -= gzm * s->topv[col];
          } else if (s->topc[col] == FLUX) {
            b += -dtg * s->rzp[fm] * volume *
                 (s->topv[col] + s->kz[fm] * s->rzp[fm] * s->vzp[fm]) / s->dz[c];
          }
        }
        double* v = s->vals7 + 7 * (size_t)row;
        v[0] = gct;
        v[1] = gxm;
        v[2] = gxp;
        v[3] = gym;
        v[4] = gyp;
        v[5] = gzm;
        v[6] = gzp;
        s->rhs[row] = b;
      }
}

/* ------------------------------------------------------------------ solver
 * PETSc KSPCG + PCJACOBI semantics (PETSc src/ksp/ksp/impls/cg/cg.c,
 * KSPConvergedDefault; call sites LinearSystem.cpp:147-151, :320): x0 = 0,
 * norm ||D^-1 r||, converged when <= max(rtol ||D^-1 b||, atol), diverged at
 * 1e5 ||D^-1 b|| or non-finite, DIVERGED_ITS at maxit.  The row sum follows
 * the CSR column order (ym, xm, zm, diag, zp, xp, yp for (j, i, k) gids). */
static void spmv7(long n, const double* v7, const long* c7, const double* x, double* y) {
  static const int order[7] = {3, 1, 5, 0, 6, 2, 4};
  for (long m = 0; m < n; ++m) {
    const double* v = v7 + 7 * m;
    const long* c = c7 + 7 * m;
    double acc = 0.0;
    for (int q = 0; q < 7; ++q) {
      const int leg = order[q];
      if (c[leg] >= 0) acc += v[leg] * x[c[leg]];
    }
    y[m] = acc;
  }
}

static double dotv(long n, const double* a, const double* b) {
  double acc = 0.0;
  for (long m = 0; m < n; ++m) acc += a[m] * b[m];
  return acc;
}

int oracle_cg7(long n, const double* v7, const long* c7, const double* bvec, double* x,
               double rtol, double atol, int maxit, double* resid) {
  double* dinv = (double*)xcalloc((size_t)n, sizeof(double));
  double* r = (double*)xcalloc((size_t)n, sizeof(double));
  double* z = (double*)xcalloc((size_t)n, sizeof(double));
  double* p = (double*)xcalloc((size_t)n, sizeof(double));
  double* w = (double*)xcalloc((size_t)n, sizeof(double));
  for (long m = 0; m < n; ++m) {
    const double dg = v7[7 * m];
    dinv[m] = (dg != 0.0) ? 1.0 / dg : 1.0;
    x[m] = 0.0;
    r[m] = bvec[m];
    z[m] = r[m] * dinv[m];
  }
  double dp = sqrt(dotv(n, z, z));
  const double rnorm0 = dp;
  const double ttol = fmax(rtol * rnorm0, atol);
  int reason = 0, its = 0;
#define TEST(rn)                                  \
  do {                                            \
    if (!isfinite(rn)) reason = -9;               \
    else if ((rn) <= ttol) reason = 2;            \
    else if ((rn) >= 1.0e5 * rnorm0) reason = -4; \
  } while (0)
  TEST(dp);
  if (reason == 0) {
    double beta = dotv(n, z, r), betaold = 1.0, dpi = 0.0, dpiold = 0.0;
    int i = 0;
    do {
      its = i + 1;
      if (beta == 0.0) {
        reason = 3;
        break;
      } else if (i > 0 && beta * betaold < 0.0) {
        reason = -8;
        break;
      }
      if (i == 0) {
        memcpy(p, z, (size_t)n * sizeof(double));
      } else {
        const double bb = beta / betaold;
        for (long m = 0; m < n; ++m) p[m] = z[m] + bb * p[m];
      }
      dpiold = dpi;
      spmv7(n, v7, c7, p, w);
      dpi = dotv(n, p, w);
      betaold = beta;
      if (dpi == 0.0 || (i > 0 && ((dpi > 0) - (dpi < 0)) * ((dpiold > 0) - (dpiold < 0)) < 0)) {
        reason = -10;
        break;
      }
      const double a = beta / dpi;
      for (long m = 0; m < n; ++m) x[m] += a * p[m];
      for (long m = 0; m < n; ++m) r[m] -= a * w[m];
      for (long m = 0; m < n; ++m) z[m] = r[m] * dinv[m];
      dp = sqrt(dotv(n, z, z));
      TEST(dp);
      if (reason != 0) break;
      beta = dotv(n, z, r);
      ++i;
    } while (i < maxit);
    if (i >= maxit) reason = -3;
  }
#undef TEST
  if (resid) *resid = dp;
  free(dinv);
  free(r);
  free(z);
  free(p);
  free(w);
  return reason < 0 ? reason : its;
}

/* ------------------------------------------------------------------ corrector */
/* computeFluxesImpl<PC, HARM> (Corrector.cpp:135-533), uncoupled, no ET. */
static void fluxes(oracle_gw* s, double dtg) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double dx = s->dx, dy = s->dy, az = s->az;
  for (int j = 1; j <= ny; ++j) /* gw_flux_x */
    for (int i = 0; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t f = I3(s, j, i, k);
        const double faceA = s->ax[f];
        double q = 0.0;
        if (i == 0) {
          const size_t c = I3(s, j, 1, k);
          const double kf = vg_k(soil_at(s, c), s->h[c], s->ksx[c]);
          q = faceA * kf * s->vxp[f] * s->cosx[f] * (s->h[c] - s->h[f]) / (0.5 * dx);
        } else {
          const size_t c = f, e = I3(s, j, i + 1, k);
          const double kc = vg_k(soil_at(s, c), s->h[c], s->ksx[c]);
          double kf, delta = dx;
          const double sg = (s->bot[e] > s->bot[c]) ? 1.0 : -1.0;
          if (i == nx) {
            kf = kc;
            delta = 0.5 * dx;
          } else {
            if (s->pc) {
              kf = s->harm ? face_harm(soil_at(s, c), s->h[c], s->ksx[c], 1.0, soil_at(s, e),
                                       s->h[e], s->ksx[e], 1.0)
                           : 0.5 * (vg_k(soil_at(s, c), s->h[c], s->ksx[c]) +
                                    vg_k(soil_at(s, e), s->h[e], s->ksx[e]));
            } else {
              const double kn = vg_k(soil_at(s, e), s->h[e], s->ksx[c]);
              kf = 0.5 * (kc + kn);
            }
            if (s->gid[c] < 0 || s->gid[e] < 0) kf = 0.0;
          }
          if (s->pc) /* along-layer gravity with r v (the theta update adds the second r) */
            q = faceA * (kf * s->vxp[f] * s->cosx[f] * (s->h[e] - s->h[c]) / delta +
                         sg * kf * s->rxp[f] * s->vxp[f] * s->sinx[f]);
          else
            q = faceA * (kf * s->vxp[f] * s->cosx[f] * (s->h[e] - s->h[c]) / delta +
                         sg * kf * s->sinx[f]);
          if (!s->full3d && ((s->gid[c] >= 0 && s->wc[c] < s->wcs[c]) ||
                             (s->gid[e] >= 0 && s->wc[e] < s->wcs[e])))
            q = 0.0;
        }
        if (i == 0) {
          const int code = s->xmc[I2(s, j, 1)];
          if (code == NOFLUX) q = 0.0;
          else if (code == FLUX) q = -s->xmv[I2(s, j, 1)] * faceA;
        } else if (i == nx) {
          const int code = s->xpc[I2(s, j, nx)];
          if (code == NOFLUX) q = 0.0;
          else if (code == FLUX) q = s->xpv[I2(s, j, nx)] * faceA;
        }
        s->qx[f] = q;
      }
  for (int j = 0; j <= ny; ++j) /* gw_flux_y */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t f = I3(s, j, i, k);
        const double faceA = s->ay[f];
        double q = 0.0;
        if (j == 0) {
          const size_t c = I3(s, 1, i, k);
          const double kf = vg_k(soil_at(s, c), s->h[c], s->ksy[c]);
          q = faceA * kf * s->vyp[f] * s->cosy[f] * (s->h[c] - s->h[f]) / (0.5 * dy);
        } else {
          const size_t c = f, n = I3(s, j + 1, i, k);
          const double kc = vg_k(soil_at(s, c), s->h[c], s->ksy[c]);
          double kf, delta = dy;
          const double sg = (s->bot[n] > s->bot[c]) ? 1.0 : -1.0;
          if (j == ny) {
            kf = kc;
            delta = 0.5 * dy;
          } else {
            if (s->pc) {
              kf = s->harm ? face_harm(soil_at(s, c), s->h[c], s->ksy[c], 1.0, soil_at(s, n),
                                       s->h[n], s->ksy[n], 1.0)
                           : 0.5 * (vg_k(soil_at(s, c), s->h[c], s->ksy[c]) +
                                    vg_k(soil_at(s, n), s->h[n], s->ksy[n]));
            } else {
              const double kn = vg_k(soil_at(s, n), s->h[n], s->ksy[c]);
              kf = 0.5 * (kc + kn);
            }
            if (s->gid[c] < 0 || s->gid[n] < 0) kf = 0.0;
          }
          if (s->pc)
            q = faceA * (kf * s->vyp[f] * s->cosy[f] * (s->h[n] - s->h[c]) / delta +
                         sg * kf * s->ryp[f] * s->vyp[f] * s->siny[f]);
          else
            q = faceA * (kf * s->vyp[f] * s->cosy[f] * (s->h[n] - s->h[c]) / delta +
                         sg * kf * s->siny[f]);
          if (!s->full3d && ((s->gid[c] >= 0 && s->wc[c] < s->wcs[c]) ||
                             (s->gid[n] >= 0 && s->wc[n] < s->wcs[n])))
            q = 0.0;
        }
        if (j == 0) {
          const int code = s->ymc[I2(s, 1, i)];
          if (code == NOFLUX) q = 0.0;
          else if (code == FLUX) q = -s->ymv[I2(s, 1, i)] * faceA;
        } else if (j == ny) {
          const int code = s->ypc[I2(s, ny, i)];
          if (code == NOFLUX) q = 0.0;
          else if (code == FLUX) q = s->ypv[I2(s, ny, i)] * faceA;
        }
        s->qy[f] = q;
      }
  for (int j = 1; j <= ny; ++j) /* gw_flux_z */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k <= nz; ++k) {
        const size_t col = I2(s, j, i);
        const double rz = s->rzp[IF(s, j, i, k)], vz = s->vzp[IF(s, j, i, k)];
        const int below = (k < nz) && s->gid[I3(s, j, i, k)] >= 0;
        const int above = (k >= 1) && s->gid[I3(s, j, i, k - 1)] >= 0;
        double q = 0.0;
        if (below && !above && s->cpl) {
          /* coupled exchange face (Corrector.cpp:388-465): the ghost head is
           * the surface depth; infiltration debits the window's budget */
          const size_t c = I3(s, j, i, k);
          const double ks = s->ksz[c], depth = s->dept[col];
          const int m = s->cmode[col];
          const double delta = 0.5 * s->dz[c];
          if (m == 2) {
            const double roomTop = fmax(0.0, (0.9999 * s->wcs[c] - s->wc[c]) * s->dz[c]);
            const double take = fmin(s->avail[col], roomTop);
            q = -take * az / dtg;
            s->avail[col] -= take;
          } else if (m == 1) {
            q = az * ks * vz * ((s->h[c] - depth) / delta - rz);
            if (q < 0.0) {
              const double need = -q * dtg / az;
              if (need > s->avail[col]) {
                q = -s->avail[col] * az / dtg;
                s->avail[col] = 0.0;
              } else {
                s->avail[col] -= need;
              }
            }
          } else if (s->pc && m == 3) {
            q = az * ks * vz * ((s->h[c] - depth) / delta - rz);
            if (q <= 0.0) {
              s->pc_clamp += -q * dtg;
              q = 0.0;
            }
          } else {
            const double kGhost = vg_k(soil_at(s, c), depth, ks);
            const double kCell = vg_k(soil_at(s, c), s->h[c], ks);
            const double kface = 0.5 * (kGhost + kCell);
            q = az * kface * vz * ((s->h[c] - depth) / delta - rz);
            if (q <= 0.0) q = 0.0;
            if (s->topc[col] == FLUX) {
              const double v = s->topv[col];
              if ((v > 0.0 && s->wc[c] > s->wcr[c]) || v < 0.0) q += v * az;
            }
          }
        } else if (below && !above) {
          const size_t c = I3(s, j, i, k);
          const int code = s->topc[col];
          if (code == FLUX) {
            q = s->topv[col] * az;
          } else if (code == HEAD) {
            const double delta = 0.5 * s->dz[c];
            q = az * s->ksz[c] * vz * ((s->h[c] - s->topv[col]) / delta - rz);
          }
        } else if (k == nz && above) {
          const size_t c = I3(s, j, i, k - 1);
          const int code = s->botc[col];
          const double kf = vg_k(soil_at(s, c), s->h[c], s->ksz[c]);
          if (code == FLUX) {
            q = s->botv[col] * az;
          } else if (code == GRAVITY) {
            q = -kf * vz * rz * az;
          } else if (code == HEAD) {
            const double delta = 0.5 * s->dz[c];
            q = az * kf * vz * ((s->botv[col] - s->h[c]) / delta - rz);
          }
        } else if (above && below) {
          const size_t up = I3(s, j, i, k - 1), lo = I3(s, j, i, k);
          double kf;
          if (s->pc) {
            kf = s->harm ? face_harm(soil_at(s, up), s->h[up], s->ksz[up], s->dz[up],
                                     soil_at(s, lo), s->h[lo], s->ksz[lo], s->dz[lo])
                         : 0.5 * (vg_k(soil_at(s, up), s->h[up], s->ksz[up]) +
                                  vg_k(soil_at(s, lo), s->h[lo], s->ksz[lo]));
          } else {
            const double ka = vg_k(soil_at(s, up), s->h[up], s->ksz[lo]);
            const double kb = vg_k(soil_at(s, lo), s->h[lo], s->ksz[lo]);
            kf = 0.5 * (ka + kb);
          }
          const double delta = 0.5 * (s->dz[up] + s->dz[lo]);
          q = az * kf * vz * ((s->h[lo] - s->h[up]) / delta - rz);
        }
        s->qz[IF(s, j, i, k)] = q;
      }
}

/* applyCoupledTopBookkeeping (Corrector.cpp:539-627), no ET: the exchanged
 * volume, the saturation bounce-back onto a dry surface, the seepage
 * accumulator and the evaporation correction. */
static void coupled_top_bookkeeping(oracle_gw* s, double dtg) {
  const double az = s->az;
  double sumE = 0.0, sumB = 0.0, sumV = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      const size_t col = I2(s, j, i);
      const int kt = s->ktop[(size_t)(j - 1) * s->nx + (i - 1)];
      if (kt < 0 || kt >= s->nz) continue;
      const size_t c = I3(s, j, i, kt);
      const double q = s->qz[IF(s, j, i, kt)];
      sumE += q * dtg;
      if (q < 0.0 && s->dept[col] <= s->min_depth) {
        const double volume = az * s->dz[c];
        if ((s->wcs[c] - s->wc[c]) < -q * dtg / volume) {
          const double d = -q * dtg / az;
          s->eta[col] += d;
          s->dept[col] += d;
          s->avail[col] += d;
          s->gain[col] += d;
          if (s->book_bounce) s->bounce[col] += d;
          sumB += d * az;
        }
      }
      s->seep[col] += q * dtg / az;
      if (s->topc[col] == FLUX && s->topv[col] > 0.0 && s->wc[c] > s->wcr[c] &&
          s->dept[col] <= s->min_depth) {
        s->seep[col] -= s->topv[col] * dtg;
        sumV += s->topv[col] * dtg * az;
      }
    }
  s->cpl_exch = sumE;
  s->cpl_bounce = sumB;
  s->cpl_evap = sumV;
}

/* updateWaterContent (Corrector.cpp:629-672). */
static double update_wc(oracle_gw* s, double dtg) {
  const double az = s->az, ss = s->ss;
  double sum = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t c = I3(s, j, i, k);
        if (s->gid[c] < 0) continue;
        const double volume = az * s->dz[c];
        const double r = s->rrho[c];
        const double coeff = volume * (r + r * ss * (s->h[c] - s->hn[c]) / s->wcs[c]);
        const size_t cw = I3(s, j, i - 1, k), cs = I3(s, j - 1, i, k);
        const size_t fp = IF(s, j, i, k + 1), fm = IF(s, j, i, k);
        const double dqx = dtg * (s->qx[c] * s->rxp[c] - s->qx[cw] * s->rxp[cw]);
        const double dqy = dtg * (s->qy[c] * s->ryp[c] - s->qy[cs] * s->ryp[cs]);
        const double dqz = dtg * (s->qz[fp] * s->rzp[fp] - s->qz[fm] * s->rzp[fm]);
        const double upd = (s->wcn[c] * r * volume + dqx + dqy + dqz) / coeff;
        s->wc[c] = upd;
        sum += upd * volume * r * ss * (s->h[c] - s->hn[c]) / s->wcs[c];
      }
  return sum;
}

/* ------------------------------------------------------------------ post-allocation
 * reallocateWaterContent (Reallocate.cpp:122-545), saturated_contact head,
 * uncoupled, no transport window, no per-cell diagnostics. */
typedef struct { double up, down; } split_t;

static split_t gradient_split(const oracle_gw* s, int j, int i, int k) { /* :205-274 */
  const double* hR = s->hsnap;
  double dh[6];
#define ACT(jj, ii, kk) ((kk) >= 0 && (kk) < s->nz && s->gid[I3(s, jj, ii, kk)] >= 0)
  const size_t c = I3(s, j, i, k);
  dh[0] = (ACT(j, i + 1, k) && s->kx[c] > 0.0) ? (hR[I3(s, j, i + 1, k)] - hR[c]) / s->dx : 0.0;
  dh[1] = (ACT(j, i - 1, k) && s->kx[I3(s, j, i - 1, k)] > 0.0)
              ? (hR[c] - hR[I3(s, j, i - 1, k)]) / s->dx : 0.0;
  dh[2] = (ACT(j + 1, i, k) && s->ky[c] > 0.0) ? (hR[I3(s, j + 1, i, k)] - hR[c]) / s->dy : 0.0;
  dh[3] = (ACT(j - 1, i, k) && s->ky[I3(s, j - 1, i, k)] > 0.0)
              ? (hR[c] - hR[I3(s, j - 1, i, k)]) / s->dy : 0.0;
  if (ACT(j, i, k + 1) && s->kz[IF(s, j, i, k + 1)] > 0.0) {
    const double dzp = 0.5 * (s->dz[c] + s->dz[c + 1]);
    dh[4] = (hR[c + 1] - hR[c]) / dzp - (s->dgrad ? s->rzp[IF(s, j, i, k + 1)] : 1.0);
  } else {
    dh[4] = 0.0;
  }
  if (ACT(j, i, k - 1) && s->kz[IF(s, j, i, k)] > 0.0) {
    const double dzm = 0.5 * (s->dz[c] + s->dz[c - 1]);
    dh[5] = (hR[c] - hR[c - 1]) / dzm - (s->dgrad ? s->rzp[IF(s, j, i, k)] : 1.0);
  } else {
    dh[5] = 0.0;
  }
#undef ACT
  if (!s->full3d) dh[0] = dh[1] = dh[2] = dh[3] = 0.0;
  double tot = 0.0, gx, gy, gz;
  if (dh[0] * dh[1] >= 0.0) {
    gx = 0.5 * (dh[0] + dh[1]);
    tot += fabs(gx);
  } else {
    gx = 0.0;
    tot += fabs(dh[0]) + fabs(dh[1]);
  }
  if (dh[2] * dh[3] >= 0.0) {
    gy = 0.5 * (dh[2] + dh[3]);
    tot += fabs(gy);
  } else {
    gy = 0.0;
    tot += fabs(dh[2]) + fabs(dh[3]);
  }
  if (dh[4] * dh[5] >= 0.0) {
    gz = 0.5 * (dh[4] + dh[5]);
    tot += fabs(gz);
  } else {
    gz = 0.0;
    tot += fabs(dh[4]) + fabs(dh[5]);
  }
  (void)gx;
  (void)gy;
  split_t r = {0.0, 0.0};
  if (tot > 0.0) {
    if (gz > 0.0) r.up = gz / tot;
    else if (gz < 0.0) r.down = -gz / tot;
    else {
      r.down = fabs(dh[4]) / tot;
      r.up = fabs(dh[5]) / tot;
    }
  }
  return r;
}

/* The transport window's record of one transfer (Reallocate.cpp:418-446):
 * from cell `from` to cell `to` (or through the column top when to < 0),
 * mirrored by the legacy rule on face `face` with `sign`; the correction
 * moves the rate onto every face the water crossed. */
static void path_record(oracle_gw* s, int j, int i, int from, int to, double vol, int face,
                        double sign, double dtg) {
  if (!s->win) return;
  const double rate = vol / dtg;
  s->pcorr[IF(s, j, i, face)] -= sign * rate;
  if (to < from) {
    for (int f = to + 1; f <= from; ++f) s->pcorr[IF(s, j, i, f)] += rate;
  } else {
    for (int f = from + 1; f <= to; ++f) s->pcorr[IF(s, j, i, f)] -= rate;
  }
}

static void reallocate(oracle_gw* s, double dtg, double* adjust, double* dropped_out) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double az = s->az;
  memcpy(s->wcsnap, s->wc, s->n3 * sizeof(double));
  memcpy(s->hsnap, s->h, s->n3 * sizeof(double));
  const double* wcR = s->wcsnap;
  const double* hR = s->hsnap;
  double sum = 0.0, drop = 0.0;
  for (int j = 1; j <= ny; ++j) /* gw_reallocate_classify */
    for (int i = 1; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) {
        const size_t c = I3(s, j, i, k);
        if (s->gid[c] < 0) {
          s->room[c] = s->sup[c] = s->sdown[c] = 0.0;
          continue;
        }
        const soil_t so = soil_at(s, c);
        const double volume = az * s->dz[c];
        const double before = s->wc[c];
        s->sup[c] = 0.0;
        s->sdown[c] = 0.0;
        if (before >= so.ts) {
          if (s->off) {
            s->room[c] = 0.0;
            continue;
          }
          const double excess = (before - so.ts) * volume;
          const split_t sp = gradient_split(s, j, i, k);
          s->sup[c] = excess * sp.up;
          s->sdown[c] = excess * sp.down;
          sum -= excess - s->sup[c] - s->sdown[c];
          drop += excess - s->sup[c] - s->sdown[c];
          s->wc[c] = so.ts;
          s->room[c] = 0.0;
          continue;
        }
        s->room[c] = (so.ts - before) * volume;
#define SAT(cc) (wcR[cc] >= s->wcs[cc] || hR[cc] > s->aev[cc])
        int adj = 0;
        if (k + 1 < nz && s->gid[c + 1] >= 0 && SAT(c + 1)) adj = 1;
        else if (s->kx[c] != 0.0 && SAT(I3(s, j, i + 1, k))) adj = 1;
        else if (s->kx[I3(s, j, i - 1, k)] != 0.0 && SAT(I3(s, j, i - 1, k))) adj = 1;
        else if (s->ky[c] != 0.0 && SAT(I3(s, j + 1, i, k))) adj = 1;
        else if (s->ky[I3(s, j - 1, i, k)] != 0.0 && SAT(I3(s, j - 1, i, k))) adj = 1;
        else {
          const int top = (k == 0) || (s->gid[c - 1] < 0);
          if (top) {
            if (s->cpl) {
              if (s->dept[I2(s, j, i)] > 0.0) adj = 1;
            } else if (s->topc[I2(s, j, i)] == HEAD && s->topv[I2(s, j, i)] >= 0.0) {
              adj = 1;
            }
          } else if (s->gid[c - 1] >= 0 && SAT(c - 1)) {
            adj = 1;
          }
        }
#undef SAT
        if (!adj) {
          if (before < 0.9999 * so.ts) s->h[c] = vg_head(so, before);
        } else if (s->off) {
          continue;
        } else {
          const double after = vg_theta(so, s->h[c]);
          s->wc[c] = after;
          s->room[c] = (so.ts - after) * volume;
          if (s->redistribute && after < before) {
            const double surplus = (before - after) * volume;
            const split_t sp = gradient_split(s, j, i, k);
            s->sup[c] = surplus * sp.up;
            s->sdown[c] = surplus * sp.down;
            sum -= surplus - s->sup[c] - s->sdown[c];
            drop += surplus - s->sup[c] - s->sdown[c];
          } else {
            sum += (after - before) * volume;
            if (after < before) drop += (before - after) * volume;
          }
        }
      }
  if (s->off) {
    *adjust = 0.0;
    *dropped_out = 0.0;
    s->cpl_vent = 0.0;
    s->cpl_thin = 0.0;
    return;
  }
  double lost = 0.0, vent = 0.0, thin = 0.0;
  for (int j = 1; j <= ny; ++j) /* gw_reallocate_send: k-sequential column walks */
    for (int i = 1; i <= nx; ++i) {
      const size_t col = I2(s, j, i);
      const int top_head = (s->topc[col] == HEAD);
      for (int k = 0; k < nz; ++k) {
        if (s->gid[I3(s, j, i, k)] < 0) continue;
        double dV = s->sup[I3(s, j, i, k)];
        if (dV > 0.0) {
          int ll = k;
          while (ll > 0 && s->gid[I3(s, j, i, ll - 1)] >= 0 && dV > 0.0) {
            --ll;
            const size_t c = I3(s, j, i, ll);
            if (s->room[c] > 0.0) {
              const double take = (s->room[c] > dV) ? dV : s->room[c];
              s->wc[c] += take / (az * s->dz[c]);
              s->room[c] -= take;
              s->qz[IF(s, j, i, ll + 1)] += take / dtg;
              path_record(s, j, i, k, ll, take, ll + 1, 1.0, dtg);
              dV -= take;
            }
          }
          if (dV > 0.0) {
            if (s->cpl) {
              /* coupled columns vent onto the surface (Reallocate.cpp:463-490) */
              const double d = dV / az;
              if (s->vent_all || s->dept[col] > 0.0 || d > s->min_depth) {
                if (!(s->dept[col] > 0.0 || d > s->min_depth)) thin += dV;
                s->eta[col] += d;
                s->dept[col] += d;
                s->avail[col] += d;
                s->gain[col] += d;
                s->qz[IF(s, j, i, ll)] += dV / dtg;
                path_record(s, j, i, k, ll - 1, dV, ll, 1.0, dtg);
                if (s->win) s->wvent[col] += dV;
                vent += dV;
              } else {
                lost -= dV;
              }
              dV = 0.0;
            } else if (top_head) {
              s->qz[IF(s, j, i, ll)] += dV / dtg;
              path_record(s, j, i, k, ll - 1, dV, ll, 1.0, dtg);
              dV = 0.0;
            } else {
              while (ll + 1 < nz && dV > 0.0) {
                ++ll;
                const size_t c = I3(s, j, i, ll);
                if (s->room[c] > 0.0) {
                  const double take = (s->room[c] > dV) ? dV : s->room[c];
                  s->wc[c] += take / (az * s->dz[c]);
                  s->room[c] -= take;
                  s->qz[IF(s, j, i, ll)] -= take / dtg;
                  path_record(s, j, i, k, ll, take, ll, -1.0, dtg);
                  dV -= take;
                }
              }
              lost -= dV;
              dV = 0.0;
            }
          }
        }
        dV = s->sdown[I3(s, j, i, k)];
        if (dV > 0.0) {
          int ll = k;
          while (ll + 1 < nz && dV > 0.0) {
            ++ll;
            const size_t c = I3(s, j, i, ll);
            if (s->room[c] > 0.0) {
              const double take = (s->room[c] > dV) ? dV : s->room[c];
              s->wc[c] += take / (az * s->dz[c]);
              s->room[c] -= take;
              s->qz[IF(s, j, i, ll)] -= take / dtg;
              path_record(s, j, i, k, ll, take, ll, -1.0, dtg);
              dV -= take;
            }
          }
          lost -= dV;
        }
      }
    }
  *adjust = sum + lost;
  *dropped_out = drop - lost;
  s->cpl_vent = vent;
  s->cpl_thin = thin;
}

/* finalizeWaterContent (Corrector.cpp:758-792). */
static double finalize_wc(oracle_gw* s) {
  double sum = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t c = I3(s, j, i, k);
        if (s->gid[c] < 0) continue;
        const double volume = s->az * s->dz[c];
        if (s->wc[c] > s->wcs[c]) {
          const double ex = (s->wc[c] - s->wcs[c]) * volume;
          s->vloss[c] += ex;
          sum += ex;
          s->wc[c] = s->wcs[c];
        } else if (s->wc[c] < s->wcr[c]) {
          const double de = (s->wcr[c] - s->wc[c]) * volume;
          s->vloss[c] -= de;
          sum -= de;
          s->wc[c] = s->wcr[c];
        }
      }
  return sum;
}

/* accumulateBoundaryFlux (RichardsSolver.cpp:961-1006). */
static double boundary_inflow(const oracle_gw* s, double dtg) {
  double sum = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t c = I3(s, j, i, k);
        if (s->gid[c] < 0) continue;
        if (k == 0 || s->gid[c - 1] < 0) sum -= s->qz[IF(s, j, i, k)] * dtg;
        if (k == s->nz - 1) sum += s->qz[IF(s, j, i, k + 1)] * dtg;
        if (i == 1) sum -= s->qx[I3(s, j, i - 1, k)] * dtg;
        if (i == s->nx) sum += s->qx[c] * dtg;
        if (j == 1) sum -= s->qy[I3(s, j - 1, i, k)] * dtg;
        if (j == s->ny) sum += s->qy[c] * dtg;
      }
  return sum;
}

/* adaptTimeStep (AdaptiveStep.cpp:44-118); the Max / Min reductions start at
 * the reducers' identities (lowest / max), as Kokkos's do. */
static double adapt(const oracle_gw* s, double dtg) {
  double dqmax = -DBL_MAX, dtco = DBL_MAX;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t c = I3(s, j, i, k);
        const int top = (k == 0) || (s->gid[c - 1] < 0);
        if (s->gid[c] < 0 || top) continue;
        const double qin = s->qx[c] / s->ax[c] + s->qy[c] / s->ay[c] + s->qz[IF(s, j, i, k + 1)] / s->az;
        const double qou = s->qx[I3(s, j, i - 1, k)] / s->ax[c] +
                           s->qy[I3(s, j - 1, i, k)] / s->ay[c] + s->qz[IF(s, j, i, k)] / s->az;
        const double dq = fabs(qin - qou) * dtg / s->dz[c];
        if (dq > dqmax) dqmax = dq;
        if (s->wc[c] < s->wcs[c]) {
          const double dk = vg_dkdtheta(soil_at(s, c), s->wc[c], s->ksz[c]);
          const double t = s->co_max * s->dz[c] / dk;
          if (t < dtco) dtco = t;
        }
      }
  double next = dtg;
  if (dqmax > s->dq_shrink) next = dtg * 0.75;
  else if (dqmax < s->dq_grow) next = dtg * 1.25;
  if (next > dtco) next = dtco;
  if (next > s->dt_max) next = s->dt_max;
  if (next < s->dt_min) next = s->dt_min;
  return next;
}

/* ------------------------------------------------------------------ step */
int oracle_gw_step(oracle_gw* s, double t, double dtg, frehg_gw_step_info* info) {
  (void)t;
  frehg_gw_step_info out;
  memset(&out, 0, sizeof out);
  if (!s->have_state) {
    set_err("oracle_gw_step: no state");
    return FREHG_GW_ESTATE;
  }
  /* step-start refresh (RichardsSolver.cpp:743-748): the ratios first, so
   * the hydrostatic edge ghosts see this step's */
  update_baroclinic(s);
  enforce_head_bc(s);
  enforce_moisture_bc(s);
  memcpy(s->hn, s->h, s->n3 * sizeof(double));
  memcpy(s->wcn, s->wc, s->n3 * sizeof(double));
  /* predictor (:750-763) */
  if (s->cpl) classify_coupled_top(s, dtg);
  face_conductivity(s);
  assemble(s, dtg);
  double resid = 0.0;
  const int its = oracle_cg7((long)s->nactive, s->vals7, s->cols7, s->rhs, s->sol, s->rtol,
                             s->atol, s->maxit, &resid);
  if (its < 0) {
    set_err("oracle_gw_step: CG diverged");
    return FREHG_GW_ESOLVER;
  }
  for (size_t c = 0; c < s->n3; ++c)
    if (s->gid[c] >= 0) s->h[c] = s->sol[s->gid[c]];
  enforce_head_bc(s);
  /* corrector (:768-774) */
  face_conductivity(s);
  fluxes(s, dtg);
  if (s->cpl) coupled_top_bookkeeping(s, dtg);
  out.ss_storage = update_wc(s, dtg);
  /* post-allocation and the clamp (:784-787) */
  double adjust = 0.0, dropped = 0.0;
  if (s->win) memset(s->pcorr, 0, s->n3f * sizeof(double));
  reallocate(s, dtg, &adjust, &dropped);
  out.realloc_adjust = adjust;
  out.realloc_dropped = dropped;
  out.vloss = finalize_wc(s);
  enforce_moisture_bc(s);
  out.boundary_in = boundary_inflow(s, dtg);
  if (s->win) { /* accumulateTransportWindow (RichardsSolver.cpp:826-847), every slot */
    for (size_t c = 0; c < s->n3; ++c) {
      s->wx[c] += s->qx[c] * dtg;
      s->wy[c] += s->qy[c] * dtg;
    }
    for (size_t f = 0; f < s->n3f; ++f) s->wz[f] += (s->qz[f] + s->pcorr[f]) * dtg;
  }
  s->dtg_next = adapt(s, dtg);
  out.cg_iterations = its;
  out.outer_iterations = 1;
  out.residual_norm = resid;
  out.next_dt = s->dtg_next;
  out.status = FREHG_GW_OK;
  s->last = out;
  if (info) *info = out;
  return FREHG_GW_OK;
}

double oracle_gw_next_dt(const oracle_gw* s) { return s->dtg_next; }

/* The predictor system of the last step: 7 legs per row [diag, xm, xp, ym,
 * yp, zm, zp], their neighbour rows (-1 = none) and the right-hand side. */
long oracle_gw_last_system(const oracle_gw* s, double* vals7, long* cols7, double* rhs) {
  if (vals7) memcpy(vals7, s->vals7, (size_t)s->nactive * 7 * sizeof(double));
  if (cols7) memcpy(cols7, s->cols7, (size_t)s->nactive * 7 * sizeof(long));
  if (rhs) memcpy(rhs, s->rhs, (size_t)s->nactive * sizeof(double));
  return (long)s->nactive;
}
long long oracle_gw_active_cells(const oracle_gw* s) { return s->nactive; }
double oracle_gw_elevation_offset(const oracle_gw* s) { return s->offset; }

/* ownedVolume (RichardsSolver.cpp:892-912). */
double oracle_gw_owned_volume(const oracle_gw* s) {
  double v = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i)
      for (int k = 0; k < s->nz; ++k) {
        const size_t c = I3(s, j, i, k);
        if (s->gid[c] >= 0) v += s->wc[c] * s->az * s->dz[c];
      }
  return v;
}

void oracle_gw_gid(const oracle_gw* s, int* gid, int* ktop) {
  if (gid) memcpy(gid, s->gid, s->n3 * sizeof(int));
  if (ktop) memcpy(ktop, s->ktop, (size_t)s->nx * s->ny * sizeof(int));
}

int oracle_gw_get_field(const oracle_gw* s, int field, double* out) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double* src = NULL;
  int kind = 0; /* 0 cell, 1 x-face, 2 y-face, 3 z-face */
  switch (field) {
    case FREHG_GW_FIELD_HEAD: src = s->h; break;
    case FREHG_GW_FIELD_WC: src = s->wc; break;
    case FREHG_GW_FIELD_WC_START: src = s->wcn; break;
    case FREHG_GW_FIELD_DZ: src = s->dz; break;
    case FREHG_GW_FIELD_BOT: src = s->bot; break;
    case FREHG_GW_FIELD_VLOSS: src = s->vloss; break;
    case FREHG_GW_FIELD_QX: src = s->qx; kind = 1; break;
    case FREHG_GW_FIELD_KX: src = s->kx; kind = 1; break;
    case FREHG_GW_FIELD_AX: src = s->ax; kind = 1; break;
    case FREHG_GW_FIELD_SINX: src = s->sinx; kind = 1; break;
    case FREHG_GW_FIELD_COSX: src = s->cosx; kind = 1; break;
    case FREHG_GW_FIELD_QY: src = s->qy; kind = 2; break;
    case FREHG_GW_FIELD_KY: src = s->ky; kind = 2; break;
    case FREHG_GW_FIELD_AY: src = s->ay; kind = 2; break;
    case FREHG_GW_FIELD_SINY: src = s->siny; kind = 2; break;
    case FREHG_GW_FIELD_COSY: src = s->cosy; kind = 2; break;
    case FREHG_GW_FIELD_QZ: src = s->qz; kind = 3; break;
    case FREHG_GW_FIELD_KZ: src = s->kz; kind = 3; break;
    case FREHG_GW_FIELD_RHO: src = s->rrho; break;
    case FREHG_GW_FIELD_VISC: src = s->rvisc; break;
    case FREHG_GW_FIELD_RHO_X: src = s->rxp; kind = 1; break;
    case FREHG_GW_FIELD_VISC_X: src = s->vxp; kind = 1; break;
    case FREHG_GW_FIELD_RHO_Y: src = s->ryp; kind = 2; break;
    case FREHG_GW_FIELD_VISC_Y: src = s->vyp; kind = 2; break;
    case FREHG_GW_FIELD_RHO_Z: src = s->rzp; kind = 3; break;
    case FREHG_GW_FIELD_VISC_Z: src = s->vzp; kind = 3; break;
    default: set_err("oracle_gw_get_field: unknown field"); return FREHG_GW_EINVAL;
  }
  size_t q = 0;
  if (kind == 3) {
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        for (int k = 0; k <= nz; ++k) out[q++] = src[IF(s, j, i, k)];
    return FREHG_GW_OK;
  }
  const int j0 = (kind == 2) ? 0 : 1, i0 = (kind == 1) ? 0 : 1;
  for (int j = j0; j <= ny; ++j)
    for (int i = i0; i <= nx; ++i)
      for (int k = 0; k < nz; ++k) out[q++] = src[I3(s, j, i, k)];
  return FREHG_GW_OK;
}

/* ------------------------------------------------------------------ coupled top
 * RichardsSolver::attachCoupling (src/gw/RichardsSolver.hpp:180-186) with the
 * surface fields owned here, zeroed. */
int oracle_gw_attach_coupling(oracle_gw* s, double min_depth, int vent_all, int book_bounce) {
  double** f[] = {&s->eta, &s->dept, &s->seep, &s->avail, &s->gain, &s->bounce, &s->qss};
  for (size_t n = 0; n < sizeof f / sizeof f[0]; ++n) {
    if (!*f[n]) *f[n] = xcalloc(s->n2, sizeof(double));
    if (!*f[n]) {
      set_err("oracle_gw_attach_coupling: out of memory");
      return FREHG_GW_ENOMEM;
    }
  }
  if (!s->cmode) s->cmode = xcalloc(s->n2, sizeof(int));
  s->cpl = 1;
  s->min_depth = min_depth;
  s->vent_all = vent_all;
  s->book_bounce = book_bounce;
  return FREHG_GW_OK;
}

static double* surface_field(oracle_gw* s, int which) {
  switch (which) {
    case FREHG_GW_SURF_ETA: return s->eta;
    case FREHG_GW_SURF_DEPTH: return s->dept;
    case FREHG_GW_SURF_SEEP_ACCUM: return s->seep;
    case FREHG_GW_SURF_AVAIL: return s->avail;
    case FREHG_GW_SURF_GAIN: return s->gain;
    case FREHG_GW_SURF_BOUNCE: return s->bounce;
    case FREHG_GW_SURF_QSS: return s->qss;
    default: return NULL;
  }
}

/* Surface field `which` (FREHG_GW_SURF_*), (ny+2)(nx+2): copied out when out
 * is given, then overwritten from in when in is given. */
int oracle_gw_surface(oracle_gw* s, int which, double* out, const double* in) {
  if (!s->cpl) {
    set_err("oracle_gw_surface: no coupling attached");
    return FREHG_GW_ESTATE;
  }
  if (which == FREHG_GW_SURF_MODE) {
    if (out)
      for (size_t n = 0; n < s->n2; ++n) out[n] = s->cmode[n];
    return FREHG_GW_OK;
  }
  double* f = surface_field(s, which);
  if (!f) {
    set_err("oracle_gw_surface: unknown field");
    return FREHG_GW_EINVAL;
  }
  if (out) memcpy(out, f, s->n2 * sizeof(double));
  if (in) memcpy(f, in, s->n2 * sizeof(double));
  return FREHG_GW_OK;
}

void oracle_gw_coupled_audit(const oracle_gw* s, frehg_gw_coupled_audit* out) {
  out->exchanged = s->cpl_exch;
  out->bounce = s->cpl_bounce;
  out->vent = s->cpl_vent;
  out->vent_thin = s->cpl_thin;
  out->evap = s->cpl_evap;
  out->pc_clamp_volume = s->pc_clamp;
}

/* Coupler::Coupler (src/coupling/Coupler.cpp:13-38): sync marches on the
 * common dt, subcycled starts the subsurface at dt_init. */
int oracle_gw_coupler_init(oracle_gw* s, const frehg_gw_coupler_opts* o) {
  if (!s->cpl) {
    set_err("oracle_gw_coupler_init: no coupling attached");
    return FREHG_GW_ESTATE;
  }
  s->csync = o->sync != 0;
  s->cdt = o->dt;
  s->cdtg = s->csync ? o->dt : o->dt_init;
  s->clast_dt = o->dt;
  s->ctsub = o->t_start;
  return FREHG_GW_OK;
}

/* The subsurface part of Coupler::step (Coupler.cpp:69-131) on a surface the
 * caller has already advanced to t with its depth refreshed: beginWindow
 * (Exchange.cpp:21-52), the sync or subcycled substeps, applySeepage
 * (:54-107) against the bed `bottom` ((ny+2)(nx+2)) and reduceAudit
 * (:109-127). */
int oracle_gw_coupler_step(oracle_gw* s, double t, double dt, const double* bottom,
                           frehg_gw_window_audit* out) {
  frehg_gw_window_audit a;
  memset(&a, 0, sizeof a);
  s->clast_dt = dt;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      s->avail[I2(s, j, i)] = s->dept[I2(s, j, i)];
      s->gain[I2(s, j, i)] = 0.0;
    }
  if (s->book_bounce)
    for (size_t n = 0; n < s->n2; ++n) s->bounce[n] = 0.0;
  for (;;) {
    double tt, dtg;
    if (s->csync) {
      if (a.substeps > 0) break;
      s->ctsub = t;
      tt = t;
      dtg = dt;
    } else {
      if (!(s->ctsub + s->cdtg <= t + 1.0e-9)) break;
      s->ctsub += s->cdtg;
      tt = s->ctsub;
      dtg = s->cdtg;
    }
    frehg_gw_step_info info;
    const int rc = oracle_gw_step(s, tt, dtg, &info);
    if (rc != FREHG_GW_OK) return rc;
    s->cdtg = s->dtg_next;
    a.gw.boundary_in += info.boundary_in;
    a.gw.ss_storage += info.ss_storage;
    a.gw.realloc_adjust += info.realloc_adjust;
    a.gw.realloc_dropped += info.realloc_dropped;
    a.gw.vloss += info.vloss;
    a.gw.cg_iterations += info.cg_iterations;
    a.cpl.exchanged += s->cpl_exch;
    a.cpl.bounce += s->cpl_bounce;
    a.cpl.vent += s->cpl_vent;
    a.cpl.vent_thin += s->cpl_thin;
    a.cpl.evap += s->cpl_evap;
    ++a.substeps;
  }
  a.cpl.pc_clamp_volume = s->pc_clamp;
  a.gw.next_dt = s->cdtg;
  double sumA = 0.0, sumD = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      const size_t col = I2(s, j, i);
      const double v = s->seep[col];
      s->qss[col] = v / dt;
      if (v < 0.0) {
        const double before = s->eta[col];
        s->eta[col] += v;
        if (s->eta[col] < bottom[col]) s->eta[col] = bottom[col];
        const double change = s->eta[col] - before;
        s->gain[col] += change;
        sumA += change;
        sumD += change - v;
        s->seep[col] = 0.0;
      } else if (s->dept[col] > s->min_depth || v > s->min_depth) {
        s->eta[col] += v;
        s->gain[col] += v;
        sumA += v;
        s->seep[col] = 0.0;
      }
    }
  const double cell = s->dx * s->dy;
  a.applied = sumA * cell;
  a.discarded = sumD * cell;
  double sumG = 0.0, sumH = 0.0;
  for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
      sumG += s->gain[I2(s, j, i)];
      sumH += s->seep[I2(s, j, i)];
    }
  a.surface_gain = sumG * cell;
  a.accum_volume = sumH * cell;
  if (out) *out = a;
  return FREHG_GW_OK;
}

/* Coupler::nextDt / currentDtg / gwLag (Coupler.hpp:76-96). */
void oracle_gw_coupler_state(const oracle_gw* s, double t, double* next_dt, double* dtg,
                             double* lag) {
  if (next_dt) *next_dt = s->csync ? s->cdtg : s->cdt;
  if (dtg) *dtg = s->cdtg;
  if (lag) *lag = s->csync ? 0.0 : (t - s->ctsub);
}

/* The mesh bed (TerrainMetric bath), offset frame, (ny+2)(nx+2) with the
 * mirrored halo. */
void oracle_gw_bath(const oracle_gw* s, double* out) { memcpy(out, s->bath, s->n2 * sizeof(double)); }

/* Coupler::restore (Coupler.hpp:98-100): the adaptive subsurface dt and the
 * subsurface clock t - lag. */
void oracle_gw_coupler_restore(oracle_gw* s, double t, double dtg, double lag) {
  s->cdtg = dtg;
  s->ctsub = t - lag;
}

/* RichardsSolver::enableTransportWindow / resetTransportWindow
 * (RichardsSolver.cpp:796-824). */
int oracle_gw_enable_transport_window(oracle_gw* s) {
  if (s->win) return FREHG_GW_OK;
  s->wx = xcalloc(s->n3, sizeof(double));
  s->wy = xcalloc(s->n3, sizeof(double));
  s->wz = xcalloc(s->n3f, sizeof(double));
  s->pcorr = xcalloc(s->n3f, sizeof(double));
  s->wvent = xcalloc(s->n2, sizeof(double));
  if (!s->wx || !s->wy || !s->wz || !s->pcorr || !s->wvent) {
    set_err("oracle_gw_enable_transport_window: out of memory");
    return FREHG_GW_ENOMEM;
  }
  s->win = 1;
  return FREHG_GW_OK;
}

void oracle_gw_reset_transport_window(oracle_gw* s) {
  if (!s->win) return;
  memset(s->wx, 0, s->n3 * sizeof(double));
  memset(s->wy, 0, s->n3 * sizeof(double));
  memset(s->wz, 0, s->n3f * sizeof(double));
  memset(s->wvent, 0, s->n2 * sizeof(double));
}

/* Window volumes in the halo layouts: 0 x faces (qx layout), 1 y faces, 2 z
 * faces (qzF layout, path records included), 3 the vented volume per column. */
int oracle_gw_window(const oracle_gw* s, int which, double* out) {
  if (!s->win) {
    set_err("oracle_gw_window: transport window not enabled");
    return FREHG_GW_ESTATE;
  }
  const double* src = which == 0 ? s->wx : which == 1 ? s->wy : which == 2 ? s->wz : s->wvent;
  const size_t n = which == 2 ? s->n3f : which == 3 ? s->n2 : s->n3;
  memcpy(out, src, n * sizeof(double));
  return FREHG_GW_OK;
}

/* ------------------------------------------------------------------ density coupling
 * attachScalar (baroclinic on) + attachTemperature + setDensityCoefficients
 * (RichardsSolver.hpp:191-225) with the scalar fields owned here, zeroed. */
int oracle_gw_attach_density(oracle_gw* s, int saline, int thermal, const frehg_gw_density* dc) {
  if (!dc || (!saline && !thermal)) {
    set_err("oracle_gw_attach_density: no scalar or no coefficients");
    return FREHG_GW_EINVAL;
  }
  s->baro = 1;
  s->saline = saline != 0;
  s->thermal = thermal != 0;
  s->beta_s = dc->beta_saline;
  s->beta_sv = dc->beta_saline_visc;
  s->beta_t = dc->thermal_expansion;
  s->t_ref = dc->reference_temperature;
  s->dgrad = dc->reallocation_gradient != 0;
  if (s->saline && !s->s3) {
    s->s3 = xcalloc(s->n3, sizeof(double));
    s->s2 = xcalloc(s->n2, sizeof(double));
  }
  if (s->thermal && !s->t3) {
    s->t3 = xcalloc(s->n3, sizeof(double));
    s->t2 = xcalloc(s->n2, sizeof(double));
  }
  return FREHG_GW_OK;
}

/* Scalar `which` (FREHG_GW_SCALAR_*): copied out when out is given, then
 * overwritten from in when in is given. */
int oracle_gw_scalar(oracle_gw* s, int which, double* out, const double* in) {
  double* f = which == FREHG_GW_SCALAR_SALINE ? s->s3 : which == FREHG_GW_SCALAR_SALINE_SURF ? s->s2
            : which == FREHG_GW_SCALAR_TEMP ? s->t3 : which == FREHG_GW_SCALAR_TEMP_SURF ? s->t2
                                                                                : NULL;
  if (!f) {
    set_err("oracle_gw_scalar: scalar not attached");
    return FREHG_GW_EINVAL;
  }
  const size_t n = (which == FREHG_GW_SCALAR_SALINE || which == FREHG_GW_SCALAR_TEMP) ? s->n3 : s->n2;
  if (out) memcpy(out, f, n * sizeof(double));
  if (in) memcpy(f, in, n * sizeof(double));
  return FREHG_GW_OK;
}
