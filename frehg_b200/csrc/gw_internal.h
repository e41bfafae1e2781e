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
  // coupled top: exchanged, bounce, vent, vent_thin, evap, the mode-3 clamp
  double cpl[6];
  // coupler window: applied, discarded, surface gain, held seepage (per area)
  double win[4];
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
  kPExch = 9,    // coupled top: exchanged volume (bookkeeping)
  kPBounce = 10, // coupled top: bounce-back volume (bookkeeping)
  kPEvap = 11,   // coupled top: evaporation correction (bookkeeping)
  kPClamp = 12,  // coupled top: the mode-3 upward-only clamp volume (bookkeeping)
  kPVent = 13,   // coupled top: vented volume (send walk)
  kPThin = 14,   // coupled top: vents the legacy rule would have dropped (send walk)
  kPSlots = 15
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
  uint8_t* satf = nullptr;
  // coupled top: surface fields (FREHG_GW_SURF_* order, (ny+2)(nx+2) each;
  // surf_own marks the ones allocated here) and the exchange mode
  double* surf[8] = {};
  bool surf_own[8] = {};
  int8_t* cmode = nullptr;
  CplDev* cpl_dev = nullptr;  // the kernels' copy of cpl_host (f.cpl when attached)
  CplDev cpl_host{};
  // transport window (null until enabled): face volumes in the qx / qy / qzF
  // layouts, the walks' path records (qzF layout), vented volume per column
  double *win_x = nullptr, *win_y = nullptr, *win_z = nullptr, *pcorr = nullptr,
         *win_vent = nullptr;  // per-cell saturation flag of the post-allocation snapshot
  // density coupling (null until attached): the scalars (FREHG_GW_SCALAR_*
  // order, halo layouts; null when that scalar is not attached), the ratio
  // fields (cells, x / y faces like qx / qy, z faces like qzF) and their
  // coefficients
  double* scal[4] = {};
  double *rrho = nullptr, *rvisc = nullptr, *rxp = nullptr, *ryp = nullptr, *rzp = nullptr,
         *vxp = nullptr, *vyp = nullptr, *vzp = nullptr;
  BaroDev* baro_dev = nullptr;  // the kernels' copy of baro_host (f.baro when attached)
  BaroDev baro_host{};
  int saline = 0, thermal = 0;
  double beta_s = 0.0, beta_sv = 0.0, beta_t = 0.0, t_ref = 0.0;
  // linear system: coefficients and vectors carry a zero margin of sy cells
  // on both ends; the pointers below point at cell 0.
  double *diag = nullptr, *gxp = nullptr, *gyp = nullptr, *gzp = nullptr, *rhs = nullptr;
  double *x = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr, *p1 = nullptr, *w = nullptr;
  // mixed precision: FP32 copies and inner vectors (same margins)
  float *diag32 = nullptr, *gxp32 = nullptr, *gyp32 = nullptr, *gzp32 = nullptr;
  float *dinv32 = nullptr, *l32 = nullptr;  // LDL^T factors of the column blocks
  float *r32 = nullptr, *z32 = nullptr, *d32 = nullptr, *p032 = nullptr, *p132 = nullptr,
        *w32 = nullptr;
  double* xalt = nullptr;  // FP64 ping-pong partner of x (mixed / FP64 line outer sweeps)
  // FP64 line form: the column factors in FP64 and the correction d
  double *dinv64 = nullptr, *l64 = nullptr, *d64 = nullptr;
  // reductions
  double* partial = nullptr;   // kPSlots x nblk
  double* cgpart = nullptr;    // 4 x cg grid
  int nblk = 0;                // grid of the reducing cell kernels
  int cg_grid = 0;             // co-resident grid of the CG kernel
  int cg_grid32 = 0;
  StepOut* out = nullptr;      // device
  StepOut* out_host = nullptr; // pinned
  std::vector<void*> allocs;   // everything to cudaFree
  char* arena = nullptr;       // the one allocation every device array slices
  size_t arena_bytes = 0, arena_off = 0;
  bool arena_plan = false;     // sizing pass of the allocation sequence
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  mutable long long launches = 0;  // kernels launched by this domain
};

// ---------------------------------------------------------------- launchers
void launch_ghosts(const Device& D, double* h, double* wc);
void launch_closure_pred(const Device& D, const double* h);
// warm: also write the mixed / FP64 line solves' starting iterate x (active
// cells): h^n, or with hprev = h^(n-1) h^n + ratio (h^n - h^(n-1)).
void launch_assemble(const Device& D, const double* hn, const double* wcn, bool warm,
                     const double* hprev = nullptr, double ratio = 0.0);
// The predictor in one fused pass (closures, faces, rows and, mixed, the
// column factors) where it applies; false: use the separate passes.
bool launch_predict(const Device& D, const double* hn, const double* wcn, bool mixed);
// The corrector (head scatter, closures, faces, fluxes, theta update) in one
// fused pass where it applies; false: use the separate passes.
bool launch_correct(const Device& D, const double* hn, const double* wcn);
void launch_closure_corr(const Device& D, const double* hn);
void launch_flux(const Device& D, const double* wcn);
void launch_update_wc(const Device& D, const double* hn, const double* wcn);
void launch_classify(const Device& D, double* wc_out, double* h_out);
void launch_walk(const Device& D, double* wc_out);
void launch_finalize(const Device& D, double* wc_out, double co_max);
void launch_step_info(const Device& D, double dq_grow, double dq_shrink, double dt_min,
                      double dt_max);
void launch_volume(const Device& D, const double* wc);
// Density coupling: the cell and face ratios from the attached scalars.
void launch_baro(const Device& D);
// Coupled top: exchange modes (before the predictor), bookkeeping (after the
// corrector's fluxes), and the coupler window's opening and seepage.
void launch_cpl_mode(const Device& D, const double* hn);
void launch_cpl_book(const Device& D, const double* wcn);
void launch_cpl_begin_window(const Device& D);
void launch_cpl_seepage(const Device& D, double dt);
// Transport window: the step's q dtg (and path records) into the window.
void launch_window_accum(const Device& D);
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
// FP64 line form (nz <= 256): FP64 column factors, then the FP64 line-PCG
// defect-correction solve (the mixed form's algorithm in FP64).
cudaError_t launch_line_factor64(Device& D);
cudaError_t launch_cg_line64(Device& D, double atol, int maxit, double outer_rtol, int max_outer);

// Raises (never lowers) a kernel's opt-in dynamic shared-memory limit to
// `bytes`.  Only raising keeps every launch recorded earlier (in a captured
// graph, or by another domain) within the limit.
cudaError_t raise_smem_limit(const void* kernel, size_t bytes);

// ---------------------------------------------------------------- batched phases
// One member's arguments for the batched non-solve phases: its geometry and
// fields, the state buffers of its current parity, its dt and controller
// constants, and its per-kernel block counts (the single-domain launch's, so
// a member's arithmetic in a batch is the single-domain step's bit for bit).
// The host refreshes the records before every batched step.
struct alignas(16) StepArgs {
  Dims d;
  Fields f;
  double *hn, *wcn, *h_out, *wc_out;
  double *hp, *wcu, *ch, *kcx, *kcy, *kcz, *kx, *ky, *kzf, *qx, *qy, *qzf;
  double *vloss, *room, *sup, *sdn;
  double *diag, *gxp, *gyp, *gzp, *rhs, *x;
  float *diag32, *gxp32, *gyp32, *gzp32, *dinv32, *l32;
  uint8_t* satf;
  int* colflag;
  double* partial;
  StepOut* out;
  double dtg, co_max, dq_grow, dq_shrink, dt_min, dt_max;
  int nblk, tc, mixed, warp_walk;
};

// Device tables of a batch's members for the batched phases.
struct PhaseTables {
  int n = 0;
  StepArgs* tab = nullptr;       // device, n records
  StepArgs* tab_host = nullptr;  // pinned, refreshed before each step
  int *first_cells = nullptr, *first_ghost = nullptr, *first_factor = nullptr;  // device, n + 1
  int grid_cells = 0, grid_ghost = 0, grid_factor = 0;
  size_t walk_smem = 0, factor_smem = 0;
  StepOut* outs = nullptr;       // device, n step records gathered
  StepOut* outs_host = nullptr;  // pinned
  int cap = 0;                   // members the buffers hold (reused while n <= cap)
};
// (Re)builds the tables for the members `ds`, reusing the buffers while they fit.
cudaError_t phase_tables_build(PhaseTables& t, const std::vector<const Device*>& ds,
                               const std::vector<int>& mixed);
void phase_tables_free(PhaseTables& t);
void fill_step_args(const Device& D, bool mixed, double dtg, double co_max, double dq_grow,
                    double dq_shrink, double dt_min, double dt_max, StepArgs& a);
// Enqueue on s: the records' upload and the predictor phases of every member
// (ghosts, closure, assembly, and the line factor of the mixed members) ...
cudaError_t batch_predictor(const PhaseTables& t, cudaStream_t s);
// ... and, after the solves, every member's corrector, post-allocation,
// clamp, audit and controller, and the read-back of the step records.
cudaError_t batch_corrector(const PhaseTables& t, cudaStream_t s);
// Launch geometry shared by the single-domain and batched launches.
int ghost_blocks(const Device& D);
int line_tile_cols(int nz);
int line_factor_blocks(const Device& D);
size_t line_factor_smem(int nz);
cudaError_t launch_line_factor_batch(const PhaseTables& t, cudaStream_t s);

// ---------------------------------------------------------------- batched solves
// Several domains' predictor solves in one cooperative launch: member i runs
// its own solve (own CG state, reductions and barrier) on the block range
// [first[i], first[i+1]); its blocks leave as soon as its solve ends.
struct SolveParams {
  double rtol, atol, outer_rtol;
  int maxit, max_outer;
};

// Kernel variant of a domain's solve: FP64 (kind 0; variant 1 = two cells a
// thread, nz even) or mixed (kind 1; variant = V * 16 + E, see gw_cg_mixed.cu).
struct SolveClass {
  int kind, variant;
  bool operator==(const SolveClass& o) const { return kind == o.kind && variant == o.variant; }
};
SolveClass solve_class(const Device& D, int precision, bool tiled_line_solve);
// Blocks of that variant one SM holds (the cooperative limit per SM).
int solve_blocks_per_sm(const SolveClass& c, size_t smem);
// Largest block count a member may take (its reduction buffer's capacity).
int solve_max_blocks(const Device& D, const SolveClass& c);

struct SolveGroup {
  SolveClass cls{0, 0};
  int n = 0, grid = 0;
  int slots = 0;                 // the members' blocks in total (first[n])
  size_t smem = 0;
  void* tab = nullptr;           // device table of per-member kernel arguments
  int* first = nullptr;          // device block offsets, n + 1
  CgState** states = nullptr;    // device array of the members' CG states
  int* queue = nullptr;          // device counter of the slots handed out
  int* order = nullptr;          // device queue order of the members, n
  int* ofirst = nullptr;         // device slot offsets in queue order, n + 1
};
// Device bytes a group of n members of class c needs for its tables.
size_t solve_group_bytes(const SolveClass& c, int n);
// Builds a group over `ds` with `nb[i]` blocks each (all of solve kind c.kind,
// member i in class variants[i]), its
// tables placed in `mem` (solve_group_bytes of device memory the caller owns).
// The launch takes min(sum nb, max_grid) co-resident blocks (max_grid at
// least every nb[i]); each block takes the members' block slots from a queue,
// so a member's slots go out together and the blocks of a converged member go
// on to the next member's.  The queue holds the members by estimated work,
// largest first (nb times the iterations of the member's previous solve),
// re-ranked on the device before every launch.
cudaError_t solve_group_build(SolveGroup& g, const SolveClass& c, const std::vector<Device*>& ds,
                              const std::vector<int>& variants, const std::vector<int>& nb,
                              const std::vector<SolveParams>& p, int max_grid, void* mem);
// Zeroes the members' CG states and the slot queue and launches the group on `s`.
cudaError_t solve_group_launch(const SolveGroup& g, cudaStream_t s);

// Per-kind pieces of the batched solves (gw_cg.cu, gw_cg_mixed.cu).
size_t cg64_args_bytes();
void cg64_fill_args(const Device& D, const SolveParams& p, int variant, void* dst);
const void* cg64_batch_kernel();
int mixed_variant(const Device& D, bool tiled);
size_t mixed_args_bytes();
void mixed_fill_args(const Device& D, const SolveParams& p, int variant, void* dst);
size_t mixed_batch_smem(const Device& D, int variant);
const void* mixed_batch_kernel();

}  // namespace fgw
