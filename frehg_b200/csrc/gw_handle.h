// Internal: the handle behind the C ABI and the step phases shared by the
// single-domain step (gw_api.cu) and the batched step (gw_batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/frehg_gw.h"
#include "gw_internal.h"

struct frehg_gw_handle {
  fgw::Device D;
  int device = 0;  // the CUDA device the handle's memory and stream live on
  double offset = 0.0;
  long long nactive = 0;
  double* bath_dev = nullptr;
  std::vector<int> codes;      // host copy, 6 x ncol
  std::vector<double> values;  // host staging, 6 x ncol
  bool values_pinned = false;  // staging page-locked with cudaHostRegister
  double rtol = 1e-8, atol = 1e-14, outer_rtol = 1e-11;
  int maxit = 1000, max_outer = 30, precision = 0;
  double dt_min = 0, dt_max = 0, dq_grow = 0.01, dq_shrink = 0.02, co_max = 2.0;
  double next_dt = 0.0;
  bool have_state = false;
  int start_buf = 0;  // ping-pong index of the last step's theta^n
  bool profiling = false;
  bool fused = false;  // fused phase kernels where they apply (frehg_gw_set_fused)
  // Starting iterate of the mixed / FP64 line solves (frehg_gw_set_warm_start):
  // extrapolated from the previous step's start state when it is at hand
  // (have_prev: the last call stepped this handle alone from that state).
  bool extrapolate = true;
  bool have_prev = false;
  double prev_dtg = 0.0;
  cudaEvent_t ev[6] = {};
  double phase_ms[5] = {0, 0, 0, 0, 0};
  // coupled top: the last step's books and the cumulative mode-3 clamp
  frehg_gw_coupled_audit cpl_last{};
  double pc_clamp_total = 0.0;
  // coupler (coupling::Coupler state): sync flag, surface dt, subsurface dt
  // and clock
  bool coupler = false;
  int csync = 1;
  double cdt = 0.0, cdtg = 0.0, ctsub = 0.0;
};

namespace fgw_api {

// Makes `dev` the calling thread's current device for the scope of one ABI
// call and gives the caller's own back at the end, so that a thread driving
// handles on several GPUs reaches each handle's memory and stream whatever
// device it had selected.
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      ok = false;
      return;
    }
    if (prev != dev) {
      ok = cudaSetDevice(dev) == cudaSuccess;
      switched = ok;
    }
  }
  ~DeviceGuard() {
    if (switched) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Records `msg` as the calling thread's last error and returns `status`.
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

// The kernels of one step before and after the predictor solve, on the
// handle's stream; every kernel reads the step's dtg from the device step
// record.
// dtg: the step's dt, for the extrapolated starting iterate of a single
// step (0: start from h^n, as the batched steps do).
cudaError_t enqueue_predictor(frehg_gw_handle* h, double dtg = 0.0);
void enqueue_corrector(frehg_gw_handle* h);
// Interprets the step record read back into D.out_host: fills *info (may be
// null) and, on success, flips the state buffers and takes the next dt.
int finish_step(frehg_gw_handle* h, frehg_gw_step_info* info);
// Writes the host's next dt into the device step record.
cudaError_t upload_next_dt(frehg_gw_handle* h);

}  // namespace fgw_api

// Every ABI call on a handle runs on the handle's device (first statement
// after the handle's null check).
#define FGW_ON_DEVICE(h)                                 \
  fgw_api::DeviceGuard fgw_device_guard_((h)->device);   \
  if (!fgw_device_guard_.ok)                             \
  return fgw_api::fail(FREHG_GW_ECUDA, "cannot make the handle's device current")
