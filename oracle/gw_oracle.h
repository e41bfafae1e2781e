/* gw_oracle.h — CPU restatement of the frehg2 groundwater step.
 *
 * TEST INFRASTRUCTURE.  This is the parity oracle for the B200 step, not a
 * product path: only tests, the smoke check and the CPU-baseline leg of
 * bench.py load it.  It restates, serially and in FP64, the reference's
 * gw::RichardsSolver::step (src/gw/RichardsSolver.cpp:729-794) with its
 * TerrainMetric setup and PETSc KSPCG (Jacobi lane) solve, behind the same
 * descriptor as the product ABI (include/frehg_gw.h).  Each function in
 * gw_oracle.c cites the reference file:line it follows.
 *
 * Pinning: the restatement is checked against the reference's own golden
 * values (tests/unit/test_vangenuchten.cpp, the test_gw.cpp invariants) and
 * against the reference's own sources compiled on host shims (oracle/_ref).
 */
#ifndef FREHG_GW_ORACLE_H
#define FREHG_GW_ORACLE_H

#include "../include/frehg_gw.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_gw oracle_gw;

const char* oracle_gw_last_error(void);
oracle_gw* oracle_gw_create(const frehg_gw_desc* desc);
void oracle_gw_destroy(oracle_gw* s);
int oracle_gw_set_bc_values(oracle_gw* s, const double* top, const double* bot, const double* xm,
                            const double* xp, const double* ym, const double* yp);
int oracle_gw_init_state(oracle_gw* s, int form, double constant, const double* field);
int oracle_gw_set_state(oracle_gw* s, const double* head, const double* wc);
int oracle_gw_step(oracle_gw* s, double t, double dtg, frehg_gw_step_info* info);
double oracle_gw_next_dt(const oracle_gw* s);
long oracle_gw_last_system(const oracle_gw* s, double* vals7, long* cols7, double* rhs);
/* Fields in the ABI shapes (include/frehg_gw.h, FREHG_GW_FIELD_*). */
int oracle_gw_get_field(const oracle_gw* s, int field, double* out);
double oracle_gw_owned_volume(const oracle_gw* s);
long long oracle_gw_active_cells(const oracle_gw* s);
double oracle_gw_elevation_offset(const oracle_gw* s);
/* ktop per column (ny*nx) and gids in the halo layout ((ny+2)*(nx+2)*nz). */
void oracle_gw_gid(const oracle_gw* s, int* gid, int* ktop);

/* Coupled top (RichardsSolver::attachCoupling, src/gw/RichardsSolver.hpp:
 * 132-186) with surface fields owned by the oracle, and the subsurface part
 * of coupling::Coupler::step (src/coupling/Coupler.cpp:69-131). */
int oracle_gw_attach_coupling(oracle_gw* s, double min_depth, int vent_all, int book_bounce);
int oracle_gw_surface(oracle_gw* s, int which, double* out, const double* in);
void oracle_gw_coupled_audit(const oracle_gw* s, frehg_gw_coupled_audit* out);
int oracle_gw_coupler_init(oracle_gw* s, const frehg_gw_coupler_opts* o);
int oracle_gw_coupler_step(oracle_gw* s, double t, double dt, const double* bottom,
                           frehg_gw_window_audit* out);
void oracle_gw_coupler_state(const oracle_gw* s, double t, double* next_dt, double* dtg,
                             double* lag);
void oracle_gw_coupler_restore(oracle_gw* s, double t, double dtg, double lag);
/* The mesh bed, offset frame, (ny+2)*(nx+2) with the mirrored halo. */
void oracle_gw_bath(const oracle_gw* s, double* out);

/* Transport window (RichardsSolver::enableTransportWindow / reset /
 * windowVolumeX/Y/Z / windowVentVolume, RichardsSolver.hpp:229-248). */
int oracle_gw_enable_transport_window(oracle_gw* s);
void oracle_gw_reset_transport_window(oracle_gw* s);
int oracle_gw_window(const oracle_gw* s, int which, double* out);

/* Density coupling (RichardsSolver::attachScalar / attachTemperature /
 * setDensityCoefficients, RichardsSolver.hpp:191-225; Baroclinic.cpp) with the
 * scalars owned by the oracle (halo layouts, FREHG_GW_SCALAR_*); the ratios
 * come back through oracle_gw_get_field (FREHG_GW_FIELD_RHO .. VISC_Z). */
int oracle_gw_attach_density(oracle_gw* s, int saline, int thermal, const frehg_gw_density* dc);
int oracle_gw_scalar(oracle_gw* s, int which, double* out, const double* in);

/* Pointwise closures (src/gw/VanGenuchten.hpp:45-128), exported for the
 * golden-value tests. */
double oracle_vg_theta(double vga, double vgn, double ts, double tr, double aev, double h);
double oracle_vg_head(double vga, double vgn, double ts, double tr, double aev, double wc);
double oracle_vg_capacity(double vga, double vgn, double ts, double tr, double aev, double h);
double oracle_vg_conductivity(double vga, double vgn, double ts, double tr, double aev, double h,
                              double ks);
double oracle_vg_dkdtheta(double vga, double vgn, double ts, double tr, double aev, double wc,
                          double ks);

/* Standalone Jacobi-PCG on a 7-point system given per-row legs
 * [diag, xm, xp, ym, yp, zm, zp] and neighbor rows (-1 = none), PETSc KSPCG
 * semantics (used by the solver parity test).  Returns iterations, or a
 * negative KSP divergence reason. */
int oracle_cg7(long n, const double* vals7, const long* cols7, const double* b, double* x,
               double rtol, double atol, int maxit, double* resid);

#ifdef __cplusplus
}
#endif

#endif /* FREHG_GW_ORACLE_H */
