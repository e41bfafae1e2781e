// Host set-up of one groundwater domain (see gw_setup.h).
//
// The mesh rules are the reference's subsurface geometry
// (src/gw/TerrainMetric.cpp): the elevation lift to a non-negative frame
// (:101-150), the regular mesh with its partial-cell rules anchored at the
// box top (:158-230), the terrain-following mesh in its scaled and uniform
// layer forms (:232-293), edge-mirrored ghosts (:17-62), per-face slope
// metrics from cell-centre elevations and the face areas (:295-408); the
// active mask is Grid::buildGlobalIds' k >= ktop rule (src/core/Grid.cpp:
// 160-215).  Soil ghosts mirror the interior (RichardsSolver.cpp:24-57).
#include "gw_setup.h"

#include <cstring>

#include <algorithm>
#include <cmath>

namespace fgw {

namespace {

struct Idx {
  int nx2, nz;
  long long c(int j, int i, int k) const { return (static_cast<long long>(j) * nx2 + i) * nz + k; }
  long long col(int j, int i) const { return static_cast<long long>(j) * nx2 + i; }
};

// Single-rank edge mirror of a halo-layout field with `nzf` values per column.
template <class T>
void mirror_edges(std::vector<T>& f, int nx, int ny, int nzf) {
  const long long nx2 = nx + 2;
  auto at = [&](int j, int i, int k) -> T& { return f[(j * nx2 + i) * nzf + k]; };
  for (int k = 0; k < nzf; ++k) {
    for (int j = 1; j <= ny; ++j) {
      at(j, 0, k) = at(j, 1, k);
      at(j, nx + 1, k) = at(j, nx, k);
    }
    for (int i = 0; i <= nx + 1; ++i) {
      at(0, i, k) = at(1, i, k);
      at(ny + 1, i, k) = at(ny, i, k);
    }
  }
}

bool valid_code(int c) { return c >= FREHG_GW_BC_NOFLUX && c <= FREHG_GW_BC_HEAD_HYDROSTATIC; }

}  // namespace

int soil_storage(const frehg_gw_desc& d, int f, double* u) {
  const double* src[8] = {d.ksx, d.ksy, d.ksz, d.vg_alpha, d.vg_n, d.theta_s, d.theta_r, d.aev};
  if (f < 0 || f > 7 || !src[f] || d.nx < 1 || d.ny < 1 || d.nz < 1) return kSoilOwn;
  const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
  const double* a = src[f];
  bool uniform = true;
  for (size_t c = 1; c < n && uniform; ++c) uniform = std::memcmp(a + c, a, sizeof(double)) == 0;
  if (uniform) {
    if (u) *u = a[0];
    return kSoilUniform;
  }
  // the first earlier match is never itself shared: that field would have
  // matched first; a uniform field is never equal to this non-uniform one
  for (int g = 0; g < f; ++g) {
    if (!src[g]) continue;
    if (src[g] == a || std::memcmp(src[g], a, n * sizeof(double)) == 0) return g;
  }
  return kSoilOwn;
}

int build_host_domain(const frehg_gw_desc& d, HostDomain& o, std::string& err) {
  if (d.abi_version != FREHG_GW_ABI_VERSION) {
    err = "frehg_gw_desc.abi_version mismatch";
    return FREHG_GW_EINVAL;
  }
  if (d.nx < 1 || d.ny < 1 || d.nz < 1 || !(d.dx > 0.0) || !(d.dy > 0.0)) {
    err = "extents and spacings must be positive";
    return FREHG_GW_EINVAL;
  }
  if (!d.dz_layers || !d.ksx || !d.ksy || !d.ksz || !d.vg_alpha || !d.vg_n || !d.theta_s ||
      !d.theta_r || !d.aev || !d.top_code || !d.bot_code || !d.xm_code || !d.xp_code ||
      !d.ym_code || !d.yp_code) {
    err = "missing descriptor array";
    return FREHG_GW_EINVAL;
  }
  if (!d.saturated_contact_head) {
    err = "saturated_contact legacy reads neighbours in place (loop-order dependent); "
          "only saturated_contact head is supported";
    return FREHG_GW_EUNSUPPORTED;
  }
  for (int k = 0; k < d.nz; ++k) {
    if (!(d.dz_layers[k] > 0.0)) {
      err = "dz_layers must be positive";
      return FREHG_GW_EINVAL;
    }
  }
  if (static_cast<long long>(d.nx + 2) * (d.ny + 2) * d.nz >= (1LL << 32)) {
    err = "(nx+2)(ny+2)nz must stay below 2^32 cells";
    return FREHG_GW_EINVAL;
  }
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  o.nx = nx;
  o.ny = ny;
  o.nz = nz;
  o.ncol = static_cast<long long>(nx + 2) * (ny + 2);
  o.ncell = o.ncol * nz;
  const Idx X{nx + 2, nz};
  const long long n3 = o.ncell;

  // Bathymetry and the elevation lift.
  o.bath.assign(o.ncol, 0.0);
  double lmin = 0.0, lmax = 0.0;
  for (int j = 1; j <= ny; ++j) {
    for (int i = 1; i <= nx; ++i) {
      const double b = d.bath ? d.bath[static_cast<long long>(j - 1) * nx + (i - 1)] : 0.0;
      if (!std::isfinite(b)) {
        err = "non-finite bed elevation";
        return FREHG_GW_EINVAL;
      }
      o.bath[X.col(j, i)] = b;
      lmin = std::min(lmin, b);
      lmax = std::max(lmax, b);
    }
  }
  o.offset = (lmin < 0.0) ? -lmin : 0.0;
  o.box_top = lmax + o.offset;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) o.bath[X.col(j, i)] += o.offset;
  mirror_edges(o.bath, nx, ny, 1);

  o.dz.assign(n3, 0.0);
  o.bot.assign(n3, 0.0);
  o.ktop.assign(static_cast<size_t>(nx) * ny, 0);
  double depth = 0.0;
  for (int k = 0; k < nz; ++k) depth += d.dz_layers[k];

  if (d.follow_terrain) {
    const double box_bottom = o.box_top - depth;
    double weights = 0.0, w = 1.0;
    for (int k = 0; k < nz; ++k) {
      weights += w;
      w *= d.dz_stretch;
    }
    for (int j = 1; j <= ny; ++j) {
      for (int i = 1; i <= nx; ++i) {
        const double bath = o.bath[X.col(j, i)];
        if (!d.terrain_uniform && bath <= box_bottom) {
          err = "follow_terrain (scaled layers) needs every bed above the box bottom";
          return FREHG_GW_EINVAL;
        }
        double layer = d.terrain_uniform ? d.dz_layers[0] : (bath - box_bottom) / weights;
        double bottom = bath;
        for (int k = 0; k < nz; ++k) {
          if (d.terrain_uniform) layer = d.dz_layers[k];
          bottom -= layer;
          o.dz[X.c(j, i, k)] = layer;
          o.bot[X.c(j, i, k)] = bottom;
          if (!d.terrain_uniform) layer *= d.dz_stretch;
        }
        o.ktop[static_cast<size_t>(j - 1) * nx + (i - 1)] = 0;
      }
    }
  } else {
    std::vector<double> layer_bottom(nz);
    double level = o.box_top;
    for (int k = 0; k < nz; ++k) {
      level -= d.dz_layers[k];
      layer_bottom[k] = level;
    }
    std::vector<int> active(nz);
    for (int j = 1; j <= ny; ++j) {
      for (int i = 1; i <= nx; ++i) {
        const double bath = o.bath[X.col(j, i)];
        for (int k = 0; k < nz; ++k) {
          o.bot[X.c(j, i, k)] = layer_bottom[k];
          o.dz[X.c(j, i, k)] = d.dz_layers[k];
          active[k] = 0;
        }
        for (int k = 0; k < nz; ++k) {
          const long long c = X.c(j, i, k);
          const double nominal = d.dz_layers[k];
          if (o.bot[c] >= bath - 1.0e-5) {
            // Cell above the bed: inactive; a crossing within one layer pins
            // its bottom to the bed.
            if (o.bot[c] - bath < nominal) o.bot[c] = bath;
          } else {
            active[k] = 1;
            const double keep = bath - o.bot[c];
            if (keep <= nominal) {
              if (keep >= 0.25 * nominal) {
                o.dz[c] = keep;  // shortened crossing layer
              } else if (k + 1 < nz) {
                active[k] = 0;  // sliver merged into the layer below
                o.dz[c + 1] += keep;
              }
            }
          }
        }
        int top = nz;
        for (int k = 0; k < nz; ++k) {
          if (active[k]) {
            top = k;
            break;
          }
        }
        o.ktop[static_cast<size_t>(j - 1) * nx + (i - 1)] = top;
      }
    }
  }
  mirror_edges(o.dz, nx, ny, nz);
  mirror_edges(o.bot, nx, ny, nz);

  // Slope metrics (terrain only; boundary faces keep sin 0, cos 1) and areas.
  o.sinx.assign(n3, 0.0);
  o.cosx.assign(n3, 1.0);
  o.siny.assign(n3, 0.0);
  o.cosy.assign(n3, 1.0);
  if (d.follow_terrain) {
    for (int j = 0; j <= ny + 1; ++j) {
      for (int i = 1; i <= nx - 1; ++i) {
        for (int k = 0; k < nz; ++k) {
          const long long a = X.c(j, i, k), b = X.c(j, i + 1, k);
          const double rise = std::fabs((o.bot[b] + 0.5 * o.dz[b]) - (o.bot[a] + 0.5 * o.dz[a]));
          const double run = std::sqrt(rise * rise + d.dx * d.dx);
          o.sinx[a] = rise / run;
          o.cosx[a] = d.dx / run;
        }
      }
    }
    for (int j = 1; j <= ny - 1; ++j) {
      for (int i = 0; i <= nx + 1; ++i) {
        for (int k = 0; k < nz; ++k) {
          const long long a = X.c(j, i, k), b = X.c(j + 1, i, k);
          const double rise = std::fabs((o.bot[b] + 0.5 * o.dz[b]) - (o.bot[a] + 0.5 * o.dz[a]));
          const double run = std::sqrt(rise * rise + d.dy * d.dy);
          o.siny[a] = rise / run;
          o.cosy[a] = d.dy / run;
        }
      }
    }
  }
  o.ax.assign(n3, 0.0);
  o.ay.assign(n3, 0.0);
  for (int j = 0; j <= ny + 1; ++j) {
    for (int i = 0; i <= nx + 1; ++i) {
      for (int k = 0; k < nz; ++k) {
        const long long c = X.c(j, i, k);
        if (d.follow_terrain) {
          const double dze = (i <= nx) ? o.dz[X.c(j, i + 1, k)] : o.dz[c];
          const double dzn = (j <= ny) ? o.dz[X.c(j + 1, i, k)] : o.dz[c];
          o.ax[c] = 0.5 * (o.dz[c] + dze) * o.cosx[c] * d.dy;
          o.ay[c] = 0.5 * (o.dz[c] + dzn) * o.cosy[c] * d.dx;
        } else {
          o.ax[c] = d.dy * o.dz[c];
          o.ay[c] = d.dx * o.dz[c];
        }
      }
    }
  }

  // Active mask: interior cells at or below the column's first active layer.
  o.act.assign(n3, 0);
  o.nactive = 0;
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      for (int k = o.ktop[static_cast<size_t>(j - 1) * nx + (i - 1)]; k < nz; ++k) {
        o.act[X.c(j, i, k)] = 1;
        ++o.nactive;
      }

  // Soil, interior then mirrored ghosts.
  const double* src[8] = {d.ksx, d.ksy, d.ksz, d.vg_alpha, d.vg_n, d.theta_s, d.theta_r, d.aev};
  for (int f = 0; f < 8; ++f) {
    o.soil[f].assign(n3, 0.0);
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i)
        for (int k = 0; k < nz; ++k) {
          const double v = src[f][(static_cast<long long>(j - 1) * nx + (i - 1)) * nz + k];
          if (!std::isfinite(v)) {
            err = "non-finite soil parameter";
            return FREHG_GW_EINVAL;
          }
          o.soil[f][X.c(j, i, k)] = v;
        }
    mirror_edges(o.soil[f], nx, ny, nz);
  }
  for (long long c = 0; c < n3; ++c) {
    if (o.act[c] && (!(o.soil[4][c] > 1.0) || !(o.soil[3][c] > 0.0) ||
                     !(o.soil[5][c] > o.soil[6][c]))) {
      err = "van Genuchten parameters need n > 1, alpha > 0, theta_s > theta_r";
      return FREHG_GW_EINVAL;
    }
  }

  // Boundary markers (buildBoundaryLists): per column top/bottom, per edge
  // column side codes.
  o.codes.assign(6 * o.ncol, 0);
  for (int j = 1; j <= ny; ++j) {
    for (int i = 1; i <= nx; ++i) {
      const long long q = static_cast<long long>(j - 1) * nx + (i - 1);
      if (!valid_code(d.top_code[q]) || !valid_code(d.bot_code[q])) {
        err = "invalid boundary code";
        return FREHG_GW_EINVAL;
      }
      o.codes[0 * o.ncol + X.col(j, i)] = d.top_code[q];
      o.codes[1 * o.ncol + X.col(j, i)] = d.bot_code[q];
    }
  }
  for (int j = 1; j <= ny; ++j) {
    if (!valid_code(d.xm_code[j - 1]) || !valid_code(d.xp_code[j - 1])) {
      err = "invalid boundary code";
      return FREHG_GW_EINVAL;
    }
    o.codes[2 * o.ncol + X.col(j, 1)] = d.xm_code[j - 1];
    o.codes[3 * o.ncol + X.col(j, nx)] = d.xp_code[j - 1];
  }
  for (int i = 1; i <= nx; ++i) {
    if (!valid_code(d.ym_code[i - 1]) || !valid_code(d.yp_code[i - 1])) {
      err = "invalid boundary code";
      return FREHG_GW_EINVAL;
    }
    o.codes[4 * o.ncol + X.col(1, i)] = d.ym_code[i - 1];
    o.codes[5 * o.ncol + X.col(ny, i)] = d.yp_code[i - 1];
  }
  return FREHG_GW_OK;
}

}  // namespace fgw
