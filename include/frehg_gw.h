/* frehg_gw.h — C ABI of the B200 groundwater (3D mixed-form Richards) step.
 *
 * Drop-in for the frehg2 groundwater module's step path.  Each entry point
 * replaces one piece of the reference's C++ interface (paths are within the
 * frehg2 project):
 *
 *   frehg_gw_create        gw::RichardsSolver::RichardsSolver
 *                          (src/gw/RichardsSolver.hpp:177-178,
 *                          RichardsSolver.cpp:61-205) together with the
 *                          setup it consumes: gw::TerrainMetric
 *                          (TerrainMetric.cpp:69-430), Grid::buildGlobalIds
 *                          (Grid.cpp:160-238) and the BC markers of
 *                          RichardsSolver::buildBoundaryLists (:429-524).
 *   frehg_gw_init_state    RichardsSolver::applyInitialConditions (:331-427)
 *   frehg_gw_set_state     a restart read + RichardsSolver::refreshDerivedState
 *                          (RichardsSolver.hpp:336, RichardsSolver.cpp:880-890)
 *   frehg_gw_restore       the groundwater part of Simulation::restoreFromCheckpoint
 *                          (driver/Simulation.cpp:707-792, io/Checkpoint.hpp):
 *                          h, wc, vloss_cum and the adaptive-step scalar dtg
 *   frehg_gw_set_bc_values RichardsSolver::updateBoundaryValues (:526-566);
 *                          the caller evaluates BoundaryCondition::value(t)
 *   frehg_gw_step          RichardsSolver::step(t, dtg) (RichardsSolver.hpp:257,
 *                          RichardsSolver.cpp:729-794), including the
 *                          LinearSystem::setValues/solve KSP call it makes
 *                          (core/LinearSystem.hpp:119-133)
 *   frehg_gw_next_dt       RichardsSolver::nextDt (RichardsSolver.hpp:261)
 *   frehg_gw_get_field     head(), waterContent(), fluxXVolumetric(),
 *                          fluxYVolumetric(), fluxZFaceVolumetric(),
 *                          faceConductivityX/Y/ZFace(), waterContentStart()
 *                          (RichardsSolver.hpp:265-358)
 *   frehg_gw_owned_volume  RichardsSolver::ownedVolume (RichardsSolver.hpp:423)
 *   frehg_gw_destroy       ~RichardsSolver
 *
 * Conventions (kept from the reference): cell (j, i, k), k = 0 at the land
 * surface, k increasing downward, k unit-stride; interior host arrays are
 * indexed ((j * nx) + i) * nz + k.  x/y fluxes are positive toward -axis,
 * z fluxes positive upward, all carrying the face area [m^3/s].  z-face
 * plane k is the face above cell k; plane nz the bottom boundary face.
 *
 * Errors never cross the ABI as exceptions: every call returns a
 * frehg_gw_status; frehg_gw_last_error() describes the last failure on the
 * calling thread.  One handle may be used by one host thread at a time.
 * All device work of a handle runs on its stream (frehg_gw_set_stream).
 */
#ifndef FREHG_GW_H
#define FREHG_GW_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FREHG_GW_ABI_VERSION 1

typedef enum frehg_gw_status {
  FREHG_GW_OK = 0,
  FREHG_GW_EINVAL = 1,       /* bad argument or descriptor (reference: log::fatal) */
  FREHG_GW_EUNSUPPORTED = 2, /* a branch outside the groundwater-only step */
  FREHG_GW_ENOMEM = 3,       /* device allocation failed */
  FREHG_GW_ECUDA = 4,        /* a CUDA runtime call failed */
  FREHG_GW_ESOLVER = 5,      /* CG diverged or hit max_iterations (reference: fatal) */
  FREHG_GW_ENONFINITE = 6,   /* non-finite head or moisture after the step */
  FREHG_GW_ESTATE = 7        /* call order violated (e.g. step before init_state) */
} frehg_gw_status;

/* GwBcCode (src/gw/RichardsSolver.hpp:66-72). */
enum {
  FREHG_GW_BC_NOFLUX = 0,
  FREHG_GW_BC_HEAD = 1,
  FREHG_GW_BC_FLUX = 2,
  FREHG_GW_BC_GRAVITY = 3,
  FREHG_GW_BC_HEAD_HYDROSTATIC = 4
};

/* GroundwaterInitialConfig::Form (src/core/Config.hpp:493-498). */
enum { FREHG_GW_IC_MOISTURE = 0, FREHG_GW_IC_HEAD = 1, FREHG_GW_IC_WATER_TABLE = 2 };

/* Arithmetic of the predictor's linear solve. */
enum {
  FREHG_GW_PRECISION_FP64 = 0, /* FP64 Jacobi-PCG, PETSc KSPCG semantics */
  FREHG_GW_PRECISION_MIXED = 1, /* FP32 inner PCG inside FP64 defect correction */
  /* The mixed form's algorithm (line-preconditioned CG in defect correction,
   * started from h^n) with FP64 inner iterations, nz <= 256: the comparison
   * that isolates what FP32 buys.  Not in batches. */
  FREHG_GW_PRECISION_FP64_LINE = 2
};

/* Fields for frehg_gw_get_field. */
enum {
  FREHG_GW_FIELD_HEAD = 0,      /* (ny, nx, nz)   */
  FREHG_GW_FIELD_WC = 1,        /* (ny, nx, nz)   */
  FREHG_GW_FIELD_QX = 2,        /* (ny, nx+1, nz) faces i-1/2 .. nx-1/2 */
  FREHG_GW_FIELD_QY = 3,        /* (ny+1, nx, nz) faces j-1/2 .. ny-1/2 */
  FREHG_GW_FIELD_QZ = 4,        /* (ny, nx, nz+1) */
  FREHG_GW_FIELD_KX = 5,        /* like QX */
  FREHG_GW_FIELD_KY = 6,        /* like QY */
  FREHG_GW_FIELD_KZ = 7,        /* like QZ */
  FREHG_GW_FIELD_WC_START = 8,  /* theta^n of the last step, (ny, nx, nz) */
  FREHG_GW_FIELD_DZ = 9,        /* cell thickness (ny, nx, nz) */
  FREHG_GW_FIELD_BOT = 10,      /* cell bottom elevation, offset frame */
  FREHG_GW_FIELD_AX = 11,       /* x-face area, like QX */
  FREHG_GW_FIELD_AY = 12,       /* y-face area, like QY */
  FREHG_GW_FIELD_SINX = 13,     /* like QX */
  FREHG_GW_FIELD_COSX = 14,
  FREHG_GW_FIELD_SINY = 15,     /* like QY */
  FREHG_GW_FIELD_COSY = 16,
  FREHG_GW_FIELD_VLOSS = 17,    /* cumulative clamp volume per cell */
  /* Transport window (frehg_gw_enable_transport_window), volumes [m^3] since
   * the last reset: */
  FREHG_GW_FIELD_WINDOW_X = 18,    /* like QX */
  FREHG_GW_FIELD_WINDOW_Y = 19,    /* like QY */
  FREHG_GW_FIELD_WINDOW_Z = 20,    /* like QZ, the walks' transfers on every face they cross */
  FREHG_GW_FIELD_WINDOW_VENT = 21, /* (ny, nx): vented onto a coupled surface */
  /* density coupling (frehg_gw_attach_density): the ratios of the last step */
  FREHG_GW_FIELD_RHO = 22,      /* r_rho per cell, like HEAD */
  FREHG_GW_FIELD_VISC = 23,     /* r_visc per cell, like HEAD */
  FREHG_GW_FIELD_RHO_X = 24,    /* r_rho face means, like QX */
  FREHG_GW_FIELD_RHO_Y = 25,    /* like QY */
  FREHG_GW_FIELD_RHO_Z = 26,    /* like QZ */
  FREHG_GW_FIELD_VISC_X = 27,   /* r_visc face means, like QX */
  FREHG_GW_FIELD_VISC_Y = 28,   /* like QY */
  FREHG_GW_FIELD_VISC_Z = 29,   /* like QZ */
  /* The last step's start head h^(n-1), like HEAD: with the next dt it is
   * the state the mixed / FP64 line forms' extrapolated start needs
   * (frehg_gw_set_warm_start); ESTATE when the handle has none. */
  FREHG_GW_FIELD_HEAD_PREV = 30,
  FREHG_GW_FIELD_COUNT = 31
};

/* Static description of one domain.  Host pointers; the library copies what
 * it needs during frehg_gw_create.  Mirrors the reference's DomainConfig,
 * SoilConfig, GroundwaterConfig and SolverSystemConfig (src/core/Config.hpp:
 * 56-80, 253-260, 285-350, 673-698) after rasterization: soil and boundary
 * codes arrive per cell / per column rather than as type maps and polygons. */
typedef struct frehg_gw_desc {
  int abi_version; /* FREHG_GW_ABI_VERSION */
  int nx, ny, nz;          /* (nx+2)(ny+2)nz below 2^32 */
  double dx, dy;
  const double* dz_layers; /* nz nominal layer thicknesses (Grid::dzK) */
  double dz_stretch;       /* domain.dz_stretch (scaled terrain layer weights) */
  const double* bath;      /* ny*nx bed elevation, unshifted datum; NULL = flat 0 */
  int follow_terrain;      /* domain.follow_terrain */
  int terrain_uniform;     /* domain.terrain_layers: 1 uniform, 0 scaled */
  /* Per-cell soil, ny*nx*nz each (SoilType, Config.hpp:395-420). */
  const double *ksx, *ksy, *ksz, *vg_alpha, *vg_n, *theta_s, *theta_r, *aev;
  double specific_storage;
  /* Boundary codes (FREHG_GW_BC_*): top/bottom per column (ny*nx); side
   * codes per edge column: xm/xp indexed by j (ny), ym/yp by i (nx). */
  const int *top_code, *bot_code, *xm_code, *xp_code, *ym_code, *yp_code;
  /* Scheme switches (GroundwaterConfig). */
  int use_full3d;
  int pc_consistent;          /* predictor_corrector: 1 consistent, 0 legacy */
  int face_harmonic;          /* face_conductivity: 1 harmonic, 0 arithmetic */
  int reallocation_off;       /* reallocation: 1 disabled, 0 legacy */
  int surplus_redistribute;   /* reallocation_surplus: 1 redistribute, 0 drop */
  int saturated_contact_head; /* must be 1; the legacy in-place rule is order-dependent */
  /* Adaptive controller (GroundwaterTimestepConfig). */
  double dt_init, dt_min, dt_max, dq_grow, dq_shrink, courant_max;
  /* Predictor solve (SolverSystemConfig; the preconditioner is Jacobi). */
  double rtol, atol;
  int max_iterations;
  int precision;      /* FREHG_GW_PRECISION_* */
  double outer_rtol;  /* mixed / FP64 line: ||b - A x|| / ||b|| target of the FP64
                         outer loop (0 = 3e-12) */
  int max_outer;      /* mixed: outer-iteration cap */
} frehg_gw_desc;

/* GwStepAudit (src/gw/RichardsSolver.hpp:86-130) plus the solve statistics
 * of RichardsSolver::lastSolve (:402) and the controller output (:261). */
typedef struct frehg_gw_step_info {
  int status;
  int cg_iterations;     /* total inner iterations of the predictor solve */
  int outer_iterations;  /* mixed precision: defect-correction sweeps; fp64: 1 */
  double residual_norm;  /* final preconditioned residual norm ||D^-1 r|| */
  double boundary_in;
  double ss_storage;
  double realloc_adjust;
  double realloc_dropped;
  double vloss;
  double next_dt;
} frehg_gw_step_info;

typedef struct frehg_gw_handle frehg_gw_handle;

/* Last error message of the calling thread ("" if none). */
const char* frehg_gw_last_error(void);

/* Build geometry, masks, global ids and device state for one domain. */
int frehg_gw_create(const frehg_gw_desc* desc, frehg_gw_handle** out);
int frehg_gw_destroy(frehg_gw_handle* h);

/* Run all device work of h on this cudaStream_t (NULL = the library's own). */
int frehg_gw_set_stream(frehg_gw_handle* h, void* cuda_stream);

/* Boundary values (host arrays shaped like the codes; NULL keeps the current
 * values).  Hydrostatic stages are given in the unshifted datum.  The upload
 * (the top and bottom values, the sides' edge entries: all the step reads)
 * has landed when the call returns. */
int frehg_gw_set_bc_values(frehg_gw_handle* h, const double* top_value,
                           const double* bot_value, const double* xm_value,
                           const double* xp_value, const double* ym_value,
                           const double* yp_value);

/* Initial state from one of the three IC forms; field is ny*nx*nz (moisture,
 * head) or ny*nx (water table), NULL = the constant. */
int frehg_gw_init_state(frehg_gw_handle* h, int form, double constant, const double* field);

/* frehg_gw_init_state without any device allocation; it has no counterpart in
 * the reference.  The field is staged in one array compiled into the library
 * (FREHG_GW_STATIC_FIELD_MAX doubles, 2 MiB) instead of a buffer allocated and
 * freed per call, for callers that cannot allocate there: all free HBM already
 * given to their own pool, or other streams running that cudaFree would wait
 * for.  Larger fields return FREHG_GW_EINVAL.  All calls on a device share the
 * array: calls that overlap in time race on it and must be serialised.  The
 * first call on each device does a one-time set-up; make it before any stream
 * capture begins. */
#define FREHG_GW_STATIC_FIELD_MAX 262144
int frehg_gw_init_state_static(frehg_gw_handle* h, int form, double constant,
                               const double* field);

/* Overwrite the interior head and moisture (host, ny*nx*nz each). */
int frehg_gw_set_state(frehg_gw_handle* h, const double* head, const double* wc);

/* Restart from a checkpoint: interior head, moisture and (optionally, NULL
 * keeps it) the cumulative clamp-loss field, ny*nx*nz each, and the dt of the
 * next step.  A checkpoint is frehg_gw_get_field of HEAD, WC and VLOSS plus
 * frehg_gw_next_dt; stepping on from a restore equals the uninterrupted run. */
int frehg_gw_restore(frehg_gw_handle* h, const double* head, const double* wc,
                     const double* vloss, double dtg);

/* One groundwater step of size dtg ending at time t. */
int frehg_gw_step(frehg_gw_handle* h, double t, double dtg, frehg_gw_step_info* info);

/* The controller's next dtg (dt_init before the first step). */
int frehg_gw_next_dt(frehg_gw_handle* h, double* out);

/* Copy a field to host memory (shape per FREHG_GW_FIELD_*). */
int frehg_gw_get_field(frehg_gw_handle* h, int field, double* host_out);

/* Number of doubles frehg_gw_get_field writes for this field. */
size_t frehg_gw_field_size(const frehg_gw_handle* h, int field);

/* Sum over active cells of theta * dx * dy * dz (FP64, fixed order). */
int frehg_gw_owned_volume(frehg_gw_handle* h, double* out);

/* Number of active cells. */
long long frehg_gw_active_cells(const frehg_gw_handle* h);

/* The CUDA device ordinal the handle lives on: the calling thread's current
 * device when frehg_gw_create ran.  Every call on the handle makes that
 * device current for its duration and restores the caller's afterwards, so
 * one thread may drive handles on several GPUs.  -1 for a null handle.  (The
 * reference has one device per MPI rank, chosen by Kokkos at start-up.) */
int frehg_gw_device(const frehg_gw_handle* h);

/* Tracing (no counterpart in the reference, whose Timer sections do not
 * fence the device): with profiling on, each step records CUDA events around
 * its phases; frehg_gw_phase_times returns the last step's device times in
 * ms: [0] step-start refresh + predictor assembly (and, in the mixed form,
 * the FP32 cast and line factorization), [1] the predictor solve kernel,
 * [2] corrector, [3] post-allocation, [4] clamp, audit and controller. */
int frehg_gw_set_profiling(frehg_gw_handle* h, int on);
int frehg_gw_phase_times(frehg_gw_handle* h, double* ms5);

/* Kernel selection (no counterpart in the reference).  The fused predictor
 * (closures, faces, rows and the mixed form's column factors in one pass) and
 * fused corrector (head scatter, closures, faces, fluxes, theta update) for
 * groundwater-only domains with nz <= 256 raised a misaligned-address error
 * on the B200 whose cause is not yet found, so they are disabled: on = 1
 * returns FREHG_GW_EUNSUPPORTED, on = 0 (every phase as its separate passes,
 * the default) succeeds. */
int frehg_gw_set_fused(frehg_gw_handle* h, int on);

/* Starting iterate of the mixed and FP64 line solves (no counterpart in the
 * reference, whose KSP starts from 0): mode 1 (the default) starts a step
 * from the linear extrapolation of the last two step-start heads,
 * h^n + (dt_n / dt_(n-1)) (h^n - h^(n-1)), when the handle's previous call was
 * a step of its own from h^(n-1) (after init_state, set_state, restore or a
 * batched step it starts from h^n); mode 0 always starts from h^n.  The
 * solution's accuracy is set by the outer residual target either way; the
 * start changes the iteration count.  The FP64 Jacobi form keeps PETSc's
 * x0 = 0. */
int frehg_gw_set_warm_start(frehg_gw_handle* h, int mode);

/* The extrapolated start's history, for checkpoints that must restart bit
 * for bit (no counterpart in the reference, whose start is x0 = 0):
 * frehg_gw_prev_dt gives the last step's dt (0 when the handle has no
 * history), FREHG_GW_FIELD_HEAD_PREV its start head; after frehg_gw_restore,
 * frehg_gw_restore_prev(h, head_prev, prev_dt) puts both back (head_prev in
 * the HEAD shape). */
int frehg_gw_prev_dt(frehg_gw_handle* h, double* out);
int frehg_gw_restore_prev(frehg_gw_handle* h, const double* head_prev, double prev_dt);

/* The transport window (RichardsSolver::enableTransportWindow,
 * resetTransportWindow, windowVolumeX/Y/Z, windowVentVolume,
 * src/gw/RichardsSolver.hpp:229-248; accumulateTransportWindow,
 * RichardsSolver.cpp:826-847): once enabled, every step adds the face volumes
 * q dtg of all faces into the window fields (FREHG_GW_FIELD_WINDOW_*), and the
 * post-allocation walks record each transfer on every face it crosses in the z
 * window (the step's QZ keeps the reference's receiver-face mirror).  The
 * window stays on the device for a transport consumer; reset zeroes it.  The
 * ET vapour and root-sink windows are outside this drop-in. */
int frehg_gw_enable_transport_window(frehg_gw_handle* h);
int frehg_gw_reset_transport_window(frehg_gw_handle* h);

/* Density coupling: the baroclinic ratios of a transported salinity and/or
 * temperature (RichardsSolver::attachScalar with baroclinic on,
 * attachTemperature and setDensityCoefficients, src/gw/RichardsSolver.hpp:
 * 191-225; updateBaroclinicFaces, src/gw/Baroclinic.cpp:46-186).  At the start
 * of every step, from the scalars' current values,
 *   r_rho  = 1 + beta_saline s - thermal_expansion (T - T0)
 *   r_visc = 1 / (1 + beta_saline_visc s)
 * per cell (ghosts included), and their face means between active flanks with
 * the reference's edge rules; the legs carry r v, the z gravity terms r^2 v
 * (the consistent form's along-layer terms too), prescribed boundary fluxes r,
 * the theta update weighs each face flux by its r and the storage by the
 * cell's, and hydrostatic edge ghosts scale by the face r.  Without an
 * attached scalar every ratio is exactly 1. */
typedef struct frehg_gw_density {
  double beta_saline;           /* r_rho slope per unit s (DensityCouplingConfig: 0.000744) */
  double beta_saline_visc;      /* r_visc slope (0.0022) */
  double thermal_expansion;     /* beta_T per unit T (0 = no thermal term) */
  double reference_temperature; /* T0 (20) */
  int reallocation_gradient;    /* 1: the post-allocation split measures the vertical
                                   gradient against the face r_rho instead of 1
                                   (densityReallocationGradient) */
} frehg_gw_density;

enum {
  FREHG_GW_SCALAR_SALINE = 0,      /* s per cell, (ny+2)*(nx+2)*nz halo layout: the
                                      ghosts carry the side values the transport
                                      module enforces */
  FREHG_GW_SCALAR_SALINE_SURF = 1, /* surface s above the top faces of coupled
                                      columns, (ny+2)*(nx+2) */
  FREHG_GW_SCALAR_TEMP = 2,        /* T per cell, like SALINE */
  FREHG_GW_SCALAR_TEMP_SURF = 3    /* like SALINE_SURF */
};

/* Attach the scalars (saline and/or thermal, at least one) with the density
 * coefficients; allocates their device fields, zeroed, and the ratio fields.
 * Once only; a handle in a batch refuses it (FREHG_GW_EUNSUPPORTED). */
int frehg_gw_attach_density(frehg_gw_handle* h, int saline, int thermal,
                            const frehg_gw_density* coeffs);
/* Copy a scalar from host memory (layout per FREHG_GW_SCALAR_*), or read it
 * back (out); either pointer may be NULL.  A device-resident producer writes
 * frehg_gw_scalar_ptr's field on the handle's stream instead. */
int frehg_gw_set_scalar(frehg_gw_handle* h, int which, const double* values);
int frehg_gw_get_scalar(frehg_gw_handle* h, int which, double* out);
double* frehg_gw_scalar_ptr(frehg_gw_handle* h, int which);

/* Kernels this handle has launched since creation. */
long long frehg_gw_kernel_launches(const frehg_gw_handle* h);

/* ---------------------------------------------------------------- batches
 * Many independent domains stepped together: ensemble members, soil-parameter
 * sweeps, hillslopes of uneven size.  No counterpart in the reference, whose
 * driver steps one domain per rank; each member's step is exactly
 * frehg_gw_step's, with the member's own dt.
 *
 * A batch is a view over existing handles (it neither owns nor destroys
 * them).  One batch step runs the non-solve phases of all members on
 * concurrent streams and their predictor solves in one cooperative launch per
 * kernel class, each member on its own block range with its own CG state and
 * barrier (a member's blocks leave when its solve converges).  The step is
 * captured once as a CUDA graph per pattern of the members' state parities
 * and replayed.  A member's block counts depend on its own size and the
 * options only, so its results do not depend on the other members.  Member
 * handles stay usable between batch steps (boundary values, fields, state);
 * a batch must not step while its members are stepped on their own. */
typedef struct frehg_gw_batch frehg_gw_batch;

typedef struct {
  int cells_per_block;  /* active cells per solve block of a member; 0 = 16384 */
  int tiled_line_solve; /* mixed form: 1 = shared-memory tiled line solve at every depth */
  int use_graph;        /* 1 = replay each step as a CUDA graph, 0 = launch directly */
  int streams;          /* per_member_phases: concurrent member streams; 0 = 32 */
  int per_member_phases;/* 1 = launch each member's non-solve kernels on its own (streams);
                           0 = one launch per phase for all members (default) */
} frehg_gw_batch_opts;

typedef struct {
  int members;
  int solve_launches;       /* cooperative solve launches per step */
  int solve_blocks;         /* their blocks in total */
  int graphs;               /* captured step graphs */
  int uses_graph;           /* 0 once a capture failed (steps then launch directly) */
  long long steps;          /* batch steps since creation or the last autotune */
  long long kernel_launches;/* kernels those steps ran */
  long long kernels_per_step;
  int cells_per_block;
  int tiled_line_solve;
  double phase_ms[3];       /* last directly launched step (batched phases, use_graph = 0):
                               predictor, solves, corrector ms */
} frehg_gw_batch_stats_t;

/* Batch over n members (each initialised); opts may be NULL (defaults,
 * graphs on). */
int frehg_gw_batch_create(frehg_gw_handle* const* members, int n,
                          const frehg_gw_batch_opts* opts, frehg_gw_batch** out);
int frehg_gw_batch_destroy(frehg_gw_batch* b);
/* Rebinds the batch to a new member list (same options), reusing its streams
 * and buffers while they fit; for callers whose set of domains changes often
 * (continuous batching).  Captured graphs are dropped. */
int frehg_gw_batch_set_members(frehg_gw_batch* b, frehg_gw_handle* const* members, int n);
/* One step of every member with its own next dt (frehg_gw_next_dt, or the
 * value set by frehg_gw_batch_set_dt); infos receives n step records.  A
 * failing member does not advance; the first failure is returned. */
int frehg_gw_batch_step(frehg_gw_batch* b, frehg_gw_step_info* infos);
/* Overrides member i's dt for the next batch step (e.g. to end on a time). */
int frehg_gw_batch_set_dt(frehg_gw_batch* b, int i, double dtg);
/* Times candidate decompositions (solve blocks per member, and for the mixed
 * form the column or tiled line solve) on trial steps from a snapshot of the
 * members' state, restores that state and keeps the fastest; results are
 * cached per batch shape for the process.  best_ms is -1 on a cache hit.
 * Candidates: 4096..131072 cells per block. */
int frehg_gw_batch_autotune(frehg_gw_batch* b, int trials, frehg_gw_batch_opts* chosen,
                            double* best_ms);
int frehg_gw_batch_stats(const frehg_gw_batch* b, frehg_gw_batch_stats_t* out);
/* Solve blocks of each member (n ints). */
int frehg_gw_batch_solve_blocks(const frehg_gw_batch* b, int* nb);

/* Device memory frehg_gw_create allocates for this descriptor (an upper
 * estimate including allocation rounding); no counterpart in the reference.
 * It reads the soil arrays: a soil field uniform over the domain is kept as
 * one value and one equal byte for byte to an earlier field (ksx = ksy = ksz
 * of an isotropic soil) shares that field's array, so neither takes a cell
 * array of device memory. */
size_t frehg_gw_device_bytes(const frehg_gw_desc* desc);

/* ---------------------------------------------------------------- serving
 * A request loop for Richards solves of mixed sizes (no counterpart in the
 * reference).  Requests are copied at submission and queued; each tick
 * admits queued requests in arrival order while the device-memory budget and
 * the slot count allow (their fields and solver state then stay on the
 * device), steps every admitted request once as one batch (each with its own
 * adaptive dt; their work overlaps on the device), and retires finished
 * requests (head and theta kept on the host, device state freed).  A
 * request's result depends on its own inputs and the server options only, so
 * it is the same alone and among others.  One host thread drives a server. */
typedef struct frehg_gw_server frehg_gw_server;

typedef struct {
  size_t hbm_budget_bytes; /* device memory the server may hold; 0 = 90% of free memory */
  int max_active;          /* slots: requests stepping at once; 0 = 64 */
  int cells_per_block;     /* batch option (frehg_gw_batch_opts) */
  int use_graph;           /* batch option; graphs are re-captured when the set changes */
  int streams;             /* batch option */
} frehg_gw_server_opts;

typedef struct {
  const frehg_gw_desc* desc;   /* the domain, as for frehg_gw_create */
  int ic_form;                 /* FREHG_GW_IC_* */
  double ic_constant;
  const double* ic_field;      /* as for frehg_gw_init_state; NULL = the constant */
  const double *bc_top, *bc_bottom, *bc_xm, *bc_xp, *bc_ym, *bc_yp; /* NULL = 0 */
  int steps;                   /* adaptive steps to run */
} frehg_gw_request;

enum {
  FREHG_GW_REQ_QUEUED = 0,
  FREHG_GW_REQ_RUNNING = 1,
  FREHG_GW_REQ_DONE = 2,
  FREHG_GW_REQ_FAILED = 3
};

typedef struct {
  int state;               /* FREHG_GW_REQ_* */
  int status;              /* frehg_gw_status of a finished request */
  int steps, steps_done;
  long long cells;         /* active cells (0 until admitted) */
  double sim_time;         /* simulated time reached */
  double submit_s;         /* submission time, s since the server's creation */
  double queue_s;          /* submission to admission, -1 while queued */
  double latency_s;        /* submission to completion, -1 until finished */
  frehg_gw_step_info last; /* the request's last step record */
} frehg_gw_request_status;

typedef struct {
  int active;  /* requests in the running batch */
  int queued;  /* waiting, or in the worker's hands being admitted or retired */
  long long completed, ticks, cell_steps;
  size_t device_bytes_used, device_bytes_budget;
  double busy_s;           /* time spent inside frehg_gw_server_tick */
  double now_s;            /* time since the server's creation */
  double admit_s, rebatch_s, step_s, retire_s; /* busy_s by part: admission (device
                              state creation), batch rebuilds, batch steps, retirement */
} frehg_gw_server_stats_t;

int frehg_gw_server_create(const frehg_gw_server_opts* opts, frehg_gw_server** out);
int frehg_gw_server_destroy(frehg_gw_server* s);
/* Copies the request and queues it; *id identifies it from then on.
 * FREHG_GW_ENOMEM when it can never fit the budget. */
int frehg_gw_server_submit(frehg_gw_server* s, const frehg_gw_request* req, long long* id);
/* Admit, step, retire (see above); returns the counts left running/queued. */
int frehg_gw_server_tick(frehg_gw_server* s, int* active, int* queued);
int frehg_gw_server_poll(frehg_gw_server* s, long long id, frehg_gw_request_status* st);
/* A finished request's head or water content (FREHG_GW_FIELD_HEAD / _WC). */
int frehg_gw_server_fetch(frehg_gw_server* s, long long id, int field, double* host_out);
/* Forgets a finished request. */
int frehg_gw_server_release(frehg_gw_server* s, long long id);
int frehg_gw_server_stats(const frehg_gw_server* s, frehg_gw_server_stats_t* st);

/* ---------------------------------------------------------------- coupled top
 * The surface-subsurface exchange of coupled runs.
 *
 *   frehg_gw_attach_coupling  RichardsSolver::attachCoupling with the
 *                             GwCoupling views (src/gw/RichardsSolver.hpp:
 *                             132-186); the step then runs the coupled
 *                             branches of classifyCoupledTop (Corrector.cpp:
 *                             47-115), the top face K (Predictor.cpp:278-310),
 *                             assembly (:527-547, :627-674), the top flux
 *                             (Corrector.cpp:388-465),
 *                             applyCoupledTopBookkeeping (:539-627), the
 *                             reallocation's wet-top contact and surface vent
 *                             (Reallocate.cpp:323-333, :463-490) and the
 *                             hydrostatic edge ghost (Predictor.cpp:66-87)
 *   frehg_gw_coupled_audit    the GwStepAudit cpl* terms and pcClampVolume
 *                             (RichardsSolver.hpp:96-128, :384)
 *   frehg_gw_coupler_*        coupling::Coupler (src/coupling/Coupler.hpp,
 *                             Coupler.cpp:13-131, Exchange.cpp:21-127): the
 *                             sync / subcycled substep window, the seepage
 *                             application and the coupled audit
 *
 * Surface fields are (ny+2)*(nx+2) doubles in the halo layout (index
 * j * (nx+2) + i), elevations in the mesh's offset frame
 * (frehg_gw_elevation_offset).  The groundwater step reads the depth, debits
 * the window's infiltration budget and deposits bounce-backs and vents onto
 * eta and depth exactly where the reference does; the surface solve itself
 * (its free-surface and velocity phases and the depth refresh) stays with the
 * caller.  Evapotranspiration, the transport window and the paired salt
 * store are outside this drop-in. */
enum {
  FREHG_GW_SURF_ETA = 0,        /* free surface, offset frame */
  FREHG_GW_SURF_DEPTH = 1,      /* surface depth */
  FREHG_GW_SURF_SEEP_ACCUM = 2, /* exchanged, not yet applied depth */
  FREHG_GW_SURF_AVAIL = 3,      /* the window's remaining infiltrable depth */
  FREHG_GW_SURF_GAIN = 4,       /* this surface step's coupled deposits */
  FREHG_GW_SURF_BOUNCE = 5,     /* the bounce-back share of gain (when booked) */
  FREHG_GW_SURF_QSS = 6,        /* applied seepage rate of the last window */
  FREHG_GW_SURF_BOTTOM = 7,     /* surface bed elevation, offset frame */
  FREHG_GW_SURF_MODE = 8,       /* exchange mode of the last step (read only) */
  FREHG_GW_SURF_COUNT = 9
};

typedef struct frehg_gw_coupling {
  double min_depth;  /* surfaceWater.min_depth */
  int vent_all;      /* every vent deposits (the paired store's rule) */
  int book_bounce;   /* keep the bounce-back share of gain */
  /* Device arrays, (ny+2)*(nx+2) each, indexed by FREHG_GW_SURF_* (MODE
   * excluded); NULL = the handle allocates and zeroes its own. */
  double* field[8];
} frehg_gw_coupling;

/* The cpl* terms of the last step [m^3] and the cumulative clamp volume of
 * the consistent form's pressurized seepage faces. */
typedef struct frehg_gw_coupled_audit {
  double exchanged; /* net upward volume through the coupled top faces */
  double bounce;    /* returned to a dry surface by a full top cell */
  double vent;      /* vented onto the surface by the send walk */
  double vent_thin; /* the part of vent the legacy rule would have discarded */
  double evap;      /* evaporative top flux taken off the seepage accumulator */
  double pc_clamp_volume;
} frehg_gw_coupled_audit;

int frehg_gw_attach_coupling(frehg_gw_handle* h, const frehg_gw_coupling* c);
/* Host copies of a surface field (FREHG_GW_SURF_*). */
int frehg_gw_get_surface(frehg_gw_handle* h, int which, double* host_out);
int frehg_gw_set_surface(frehg_gw_handle* h, int which, const double* host_in);
/* Device address of a surface field (for a caller's own surface kernels). */
int frehg_gw_surface_ptr(frehg_gw_handle* h, int which, double** dev_out);
int frehg_gw_coupled_audit_get(frehg_gw_handle* h, frehg_gw_coupled_audit* out);
/* Mesh elevation offset: offset-frame elevation = datum elevation + offset. */
double frehg_gw_elevation_offset(const frehg_gw_handle* h);

typedef struct frehg_gw_coupler_opts {
  int sync;       /* coupling.mode: 1 sync (lockstep), 0 subcycled */
  double dt;      /* time.dt, the surface step */
  double dt_init; /* groundwater dt_init (subcycled start) */
  double t_start; /* time.t_start */
} frehg_gw_coupler_opts;

/* One surface step's coupled budget (CouplingAudit, Coupler.hpp:59-66). */
typedef struct frehg_gw_window_audit {
  frehg_gw_step_info gw;      /* audit terms and CG iterations summed over the
                                 substeps; next_dt = the subsurface dtg after */
  frehg_gw_coupled_audit cpl; /* summed; pc_clamp_volume cumulative */
  double applied;      /* net volume the seepage application added to eta */
  double discarded;    /* infiltration remainder cut by the eta >= bottom clamp */
  double surface_gain; /* all coupled surface deposits of the step */
  double accum_volume; /* held seepage at the end of the step */
  long substeps;
} frehg_gw_window_audit;

int frehg_gw_coupler_init(frehg_gw_handle* h, const frehg_gw_coupler_opts* o);
/* The subsurface part of Coupler::step(t, dt) on a surface the caller has
 * already advanced to t (depth refreshed): open the window, take the sync
 * step or the subcycled steps that fit, apply the seepage, reduce the audit. */
int frehg_gw_coupler_step(frehg_gw_handle* h, double t, double dt, frehg_gw_window_audit* out);
/* Coupler::nextDt, currentDtg, gwLag(t). */
int frehg_gw_coupler_state(frehg_gw_handle* h, double t, double* next_dt, double* dtg,
                           double* lag);
/* Coupler::restore(t, dtg, lag) after a checkpoint read. */
int frehg_gw_coupler_restore(frehg_gw_handle* h, double t, double dtg, double lag);

#ifdef __cplusplus
}
#endif

#endif /* FREHG_GW_H */
