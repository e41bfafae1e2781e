// Internal interfaces of the B200 groundwater step: the per-domain device
// state owned by a frehg_gw_handle and the kernel launchers of
// gw_kernels.cu / gw_cg.cu called by the host orchestration in gw_api.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "gw_device.cuh"

namespace fgw {

// Device scalars of one predictor solve (PETSc KSPCG state), written by the
// CG kernels and read back once per step.
struct CgState {
  double dp;        // ||D^-1 r|| at exit
  double rnorm0;    // ||D^-1 b||
  int its;          // KSP iteration count
  int reason;       // KSPConvergedReason (>0 converged, <0 diverged)
  int outer;        // defect-correction sweeps (mixed precision)
  int err;          // barrier timeout flag (0 = none)
  unsigned bar_count;
  unsigned bar_gen;
};

// Step results assembled on the device by k_step_info.
struct StepOut {
  double boundary_in, ss_storage, realloc_adjust, realloc_dropped, vloss;
  double next_dt, volume;
  double dqmax, dtco;
  CgState cg;
};

// Slots of the per-block partial-reduction buffer.
enum PartialSlot {
  kPSs = 0,      // ss storage (update_wc)
  kPAdj = 1,     // realloc adjust (classify)
  kPDrop = 2,    // realloc dropped (classify)
  kPLost = 3,    // walk overflow (send walks, negative)
  kPVloss = 4,   // clamp volume (finalize)
  kPInflow = 5,  // boundary inflow
  kPDqmax = 6,   // max dq (adaptive controller)
  kPDtco = 7,    // min Courant dt
  kPVol = 8,     // owned volume after the step
  kPSlots = 9
};

// Launch geometry of the reducing cell kernels (fixed per domain so every
// reduction has the same shape, and therefore the same rounding, each step).
constexpr int kBlock = 256;

struct Device {
  Dims d{};
  Fields f{};
  // soil, geometry, masks (owned copies of f's pointers)
  double *ksx = nullptr, *ksy = nullptr, *ksz = nullptr, *vga = nullptr, *vgn = nullptr;
  double *wcs = nullptr, *wcr = nullptr, *aev = nullptr;
  double *dz = nullptr, *bot = nullptr, *ax = nullptr, *ay = nullptr;
  double *sinx = nullptr, *cosx = nullptr, *siny = nullptr, *cosy = nullptr;
  int8_t* act = nullptr;
  int *codes = nullptr;    // 6 x ncol: top, bot, xm, xp, ym, yp
  double* values = nullptr;  // 6 x ncol
  // state, ping-pong
  double* h[2] = {nullptr, nullptr};
  double* wc[2] = {nullptr, nullptr};
  int cur = 0;
  double *hp = nullptr, *wcu = nullptr;           // predicted head, corrected theta
  double* ch = nullptr;                           // C(h^n) of the storage term
  double *kcx = nullptr, *kcy = nullptr, *kcz = nullptr;  // per-cell K of the pass
  double *kx = nullptr, *ky = nullptr, *kzf = nullptr;    // corrector face K
  double *qx = nullptr, *qy = nullptr, *qzf = nullptr;    // fluxes
  double *vloss = nullptr, *room = nullptr, *sup = nullptr, *sdn = nullptr;
  int* colflag = nullptr;
  uint8_t* satf = nullptr;  // per-cell saturation flag of the post-allocation snapshot
  // linear system: coefficients and vectors carry a zero margin of sy cells
  // on both ends; the pointers below point at cell 0.
  double *diag = nullptr, *gxp = nullptr, *gyp = nullptr, *gzp = nullptr, *rhs = nullptr;
  double *x = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *w = nullptr;
  // mixed precision: FP32 copies and inner vectors (same margins)
  float *diag32 = nullptr, *gxp32 = nullptr, *gyp32 = nullptr, *gzp32 = nullptr;
  float *dinv32 = nullptr, *l32 = nullptr;  // LDL^T factors of the column blocks
  float *r32 = nullptr, *z32 = nullptr, *d32 = nullptr, *p032 = nullptr, *p132 = nullptr,
        *w32 = nullptr;
  double* xalt = nullptr;  // FP64 ping-pong partner of x (mixed outer sweeps)
  // reductions
  double* partial = nullptr;   // kPSlots x nblk
  double* cgpart = nullptr;    // 3 x cg grid
  int nblk = 0;                // grid of the reducing cell kernels
  int cg_grid = 0;             // co-resident grid of the CG kernel
  int cg_grid32 = 0;
  StepOut* out = nullptr;      // device
  StepOut* out_host = nullptr; // pinned
  std::vector<void*> allocs;   // everything to cudaFree
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  mutable long long launches = 0;  // kernels launched by this domain
};

// ---------------------------------------------------------------- launchers
void launch_ghosts(const Device& D, double* h, double* wc);
void launch_closure_pred(const Device& D, const double* h);
void launch_assemble(const Device& D, const double* hn, const double* wcn, double dtg);
void launch_closure_corr(const Device& D, const double* hn);
void launch_flux(const Device& D, const double* wcn, double dtg);
void launch_update_wc(const Device& D, const double* hn, const double* wcn, double dtg);
void launch_classify(const Device& D, double* wc_out, double* h_out);
void launch_walk(const Device& D, double* wc_out, double dtg);
void launch_finalize(const Device& D, double* wc_out, double dtg, double co_max);
void launch_step_info(const Device& D, double dtg, double dq_grow, double dq_shrink,
                      double dt_min, double dt_max);
void launch_volume(const Device& D, const double* wc);
void launch_init_state(const Device& D, int form, double constant, const double* field,
                       const double* bath, double offset);
// FP64 Jacobi-PCG (PETSc KSPCG semantics); returns a CUDA error code.
cudaError_t launch_cg64(Device& D, double rtol, double atol, int maxit);
// FP32-inner / FP64-outer defect correction.
// FP32 casts of the coefficients and the per-column LDL^T factors of the
// mixed solve's line preconditioner (one launch before launch_cg_mixed).
cudaError_t launch_line_factor(Device& D);
cudaError_t launch_cg_mixed(Device& D, double rtol, double atol, int maxit, double outer_rtol,
                            int max_outer);
int cg64_grid(int sm_count, long long ncell);

}  // namespace fgw
