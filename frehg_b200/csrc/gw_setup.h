// Host-side set-up of one groundwater domain: the subsurface mesh and its
// metrics, the active-cell mask and the boundary markers, all in the halo
// layout the kernels use.  Runs once per frehg_gw_create.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/frehg_gw.h"

namespace fgw {

struct HostDomain {
  int nx = 0, ny = 0, nz = 0;
  long long ncol = 0, ncell = 0;
  double offset = 0.0;   // elevation lift applied to every elevation
  double box_top = 0.0;  // top of the subsurface box, offset frame
  std::vector<double> bath;                      // ncol
  std::vector<double> dz, bot, ax, ay, sinx, cosx, siny, cosy;  // ncell
  std::vector<int> ktop;                         // ny*nx, nz = fully inactive column
  std::vector<int8_t> act;                       // ncell
  long long nactive = 0;
  std::vector<double> soil[8];                   // ksx ksy ksz alpha n ts tr aev, mirrored
  std::vector<int> codes;                        // 6 x ncol (top, bot, xm, xp, ym, yp)
};

// Validates the descriptor and builds the host domain.  Returns a
// frehg_gw_status; on failure `err` says why.
int build_host_domain(const frehg_gw_desc& desc, HostDomain& out, std::string& err);

// How soil field f (0..7: ksx ksy ksz alpha n theta_s theta_r aev) is kept
// on the device: kSoilUniform when every cell of the descriptor's array holds
// the same value (*u gets it; the device keeps that one value, not an
// array), the index g < f of an earlier field whose array holds the
// same bytes (an isotropic soil's ksx = ksy = ksz: one array serves both),
// or kSoilOwn.  Soil never changes after frehg_gw_create, so a shared array is
// never written.  The values the kernels read are the descriptor's either
// way; what changes is the bytes they move.
constexpr int kSoilOwn = -1;
constexpr int kSoilUniform = -2;
int soil_storage(const frehg_gw_desc& desc, int f, double* u);

}  // namespace fgw
