// Serving loop for Richards solves of mixed sizes (frehg_gw_server_*).
//
// Requests arrive with their whole input (domain, soil, boundary codes and
// values, initial state, step count) and are copied at submission, so the
// caller's buffers can be reused at once.  A worker thread admits queued
// requests in arrival order while the device-memory budget and the slot count
// allow (it builds each request's handle and state on the device, where the
// state stays until the request finishes) and retires finished ones (head and
// theta copied to host memory, device state freed, latency recorded), so that
// host-side set-up and read-back overlap the device work.  Each tick of the
// caller's thread:
//
//   1. takes the requests the worker has made ready into the running set;
//   2. steps every running request once, each with its own adaptive dt, as one
//      batch (frehg_gw_batch_*): the requests' work overlaps on the device and
//      their solves share cooperative launches;
//   3. hands the requests that have taken all their steps to the worker.
//
// A request's arithmetic depends on its own inputs and the server options
// only: its solve's block count comes from its own size, and its dt sequence
// from its own controller, so its result is the same whether it ran alone or
// among others.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gw_handle.h"
#include "gw_setup.h"

using fgw_api::cuda_fail;
using fgw_api::fail;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  long long id = 0;
  frehg_gw_desc desc{};
  std::vector<double> dz, bath, soil[8], bc[6], ic_field;
  std::vector<int> codes[6];
  bool has_bc[6] = {false, false, false, false, false, false};
  bool has_bath = false, has_field = false;
  int ic_form = 0;
  double ic_constant = 0.0;
  int steps = 0;
  size_t bytes = 0;
  double t_submit = 0.0, t_admit = -1.0, t_done = -1.0;
  // running
  frehg_gw_handle* h = nullptr;
  int done_steps = 0;
  double sim_t = 0.0;
  long long cells = 0;
  // finished
  int state = FREHG_GW_REQ_QUEUED;
  int status = FREHG_GW_OK;
  std::string error;
  std::vector<double> head, wc;
  frehg_gw_step_info last{};
};

template <class T>
void copy_in(std::vector<T>& dst, const T* src, size_t n) {
  if (src) dst.assign(src, src + n);
  else dst.clear();
}

}  // namespace

struct frehg_gw_server {
  frehg_gw_server_opts opts{};
  size_t budget = 0;
  int slots = 64;
  int device = 0;
  Clock::time_point t0;
  // Shared with the worker (under mu).
  std::mutex mu;
  std::condition_variable cv;   // wakes the worker
  std::condition_variable done; // wakes a tick waiting for the worker
  bool stop = false;
  long long next_id = 1;
  size_t used = 0;              // device memory held by admitted requests
  int held = 0;                 // requests being admitted, ready or running
  int busy = 0;                 // requests the worker is admitting or retiring
  std::deque<std::unique_ptr<Request>> queue, retiring;
  std::vector<std::unique_ptr<Request>> ready;
  std::map<long long, std::unique_ptr<Request>> finished;
  long long completed = 0;
  double admit_s = 0.0, retire_s = 0.0;
  // The ticking thread's own.
  std::vector<std::unique_ptr<Request>> active;
  frehg_gw_batch* batch = nullptr;
  bool dirty = true;
  long long ticks = 0, cell_steps = 0;
  double busy_s = 0.0, rebatch_s = 0.0, step_s = 0.0;
  std::thread worker;
};

namespace {

double now_s(const frehg_gw_server* s) {
  return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

// Finishes request r (success or failure): keeps head and theta on the host,
// frees its device state.  Worker thread, outside the lock.
void finish(Request* r, int status, const std::string& err) {
  r->status = status;
  r->error = err;
  if (status == FREHG_GW_OK && r->h) {
    r->head.resize(frehg_gw_field_size(r->h, FREHG_GW_FIELD_HEAD));
    r->wc.resize(frehg_gw_field_size(r->h, FREHG_GW_FIELD_WC));
    int rc = frehg_gw_get_field(r->h, FREHG_GW_FIELD_HEAD, r->head.data());
    if (rc == FREHG_GW_OK) rc = frehg_gw_get_field(r->h, FREHG_GW_FIELD_WC, r->wc.data());
    if (rc != FREHG_GW_OK) {
      r->status = rc;
      r->error = frehg_gw_last_error();
    }
  }
  if (r->h) {
    frehg_gw_destroy(r->h);
    r->h = nullptr;
  }
  r->state = (r->status == FREHG_GW_OK) ? FREHG_GW_REQ_DONE : FREHG_GW_REQ_FAILED;
}

// Creates the device state of a queued request; returns a status.  Worker
// thread, outside the lock.
int admit(Request* r) {
  frehg_gw_handle* h = nullptr;
  int rc = frehg_gw_create(&r->desc, &h);
  if (rc != FREHG_GW_OK) return rc;
  const double* bc[6];
  for (int k = 0; k < 6; ++k) bc[k] = r->has_bc[k] ? r->bc[k].data() : nullptr;
  rc = frehg_gw_set_bc_values(h, bc[0], bc[1], bc[2], bc[3], bc[4], bc[5]);
  if (rc == FREHG_GW_OK)
    rc = frehg_gw_init_state(h, r->ic_form, r->ic_constant,
                             r->has_field ? r->ic_field.data() : nullptr);
  if (rc != FREHG_GW_OK) {
    frehg_gw_destroy(h);
    return rc;
  }
  r->h = h;
  r->cells = frehg_gw_active_cells(h);
  return FREHG_GW_OK;
}

// The worker: retirements first (they free memory and slots), then
// admissions in arrival order while the budget and the slots allow.
void worker_loop(frehg_gw_server* s) {
  cudaSetDevice(s->device);  // the device of the thread that created the server
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    if (!s->retiring.empty()) {
      std::unique_ptr<Request> r = std::move(s->retiring.front());
      s->retiring.pop_front();
      ++s->busy;
      lk.unlock();
      const auto t = Clock::now();
      finish(r.get(), r->status, r->error);
      const double dt = std::chrono::duration<double>(Clock::now() - t).count();
      lk.lock();
      --s->busy;
      s->retire_s += dt;
      s->used -= std::min(s->used, r->bytes);
      r->t_done = now_s(s);
      ++s->completed;
      const long long id = r->id;
      s->finished[id] = std::move(r);
      s->done.notify_all();
      continue;
    }
    if (!s->queue.empty() && s->held < s->slots && s->used + s->queue.front()->bytes <= s->budget) {
      std::unique_ptr<Request> r = std::move(s->queue.front());
      s->queue.pop_front();
      s->used += r->bytes;
      ++s->held;
      ++s->busy;
      lk.unlock();
      const auto t = Clock::now();
      const int rc = admit(r.get());
      const std::string err = rc == FREHG_GW_OK ? "" : frehg_gw_last_error();
      const double dt = std::chrono::duration<double>(Clock::now() - t).count();
      lk.lock();
      --s->busy;
      s->admit_s += dt;
      if (rc == FREHG_GW_ENOMEM && s->held > 1) {
        // Out of device memory despite the budget: wait for a retirement.
        s->used -= std::min(s->used, r->bytes);
        --s->held;
        s->queue.push_front(std::move(r));
        s->cv.wait(lk, [&] { return s->stop || !s->retiring.empty(); });
        continue;
      }
      r->t_admit = now_s(s);
      if (rc != FREHG_GW_OK) {
        s->used -= std::min(s->used, r->bytes);
        --s->held;
        r->status = rc;
        r->error = err;
        r->state = FREHG_GW_REQ_FAILED;
        r->t_done = r->t_admit;
        ++s->completed;
        const long long id = r->id;
        s->finished[id] = std::move(r);
      } else {
        s->ready.push_back(std::move(r));
      }
      s->done.notify_all();
      continue;
    }
    s->cv.wait(lk);
  }
}

Request* find(frehg_gw_server* s, long long id) {
  auto it = s->finished.find(id);
  if (it != s->finished.end()) return it->second.get();
  for (auto& r : s->active)
    if (r->id == id) return r.get();
  for (auto& r : s->ready)
    if (r->id == id) return r.get();
  for (auto& r : s->queue)
    if (r->id == id) return r.get();
  for (auto& r : s->retiring)
    if (r->id == id) return r.get();
  return nullptr;
}

}  // namespace

extern "C" {

size_t frehg_gw_device_bytes(const frehg_gw_desc* d) {
  if (!d || d->nx < 1 || d->ny < 1 || d->nz < 1) return 0;
  // The arena frehg_gw_create allocates: each array rounded to 256 bytes,
  // the arena to the 2 MiB page.  Reduction buffers are sized for up to 512
  // SMs, so the figure holds for any device.
  const size_t ncol = static_cast<size_t>(d->nx + 2) * (d->ny + 2);
  const size_t n3 = ncol * d->nz, nf = ncol * (d->nz + 1);
  const size_t m = static_cast<size_t>(d->nx + 2) * d->nz, ns = n3 + 2 * m;
  auto r = [](size_t bytes) { return (bytes + 255) & ~static_cast<size_t>(255); };
  int arrays = 8, ones = 0;  // geometry; soil by fgw::soil_storage
  for (int f = 0; f < 8; ++f) {
    const int k = fgw::soil_storage(*d, f, nullptr);
    arrays += k == fgw::kSoilOwn;
    ones += k == fgw::kSoilUniform;
  }
  size_t b = arrays * r(8 * n3) + ones * r(8);  // soil and geometry
  b += r(8 * ncol);                         // bed raster
  b += r(n3) + r(n3);                       // activity mask, saturation flags
  b += r(4 * 6 * ncol) + r(8 * 6 * ncol);   // BC codes and values
  b += 4 * r(8 * n3);                       // head and theta, two buffers each
  b += 14 * r(8 * n3);                      // closures, fluxes, walk scratch
  b += 2 * r(8 * nf);                       // z-face conductivity and flux
  b += r(4 * ncol);                         // column flags
  b += 11 * r(8 * ns);                      // FP64 solver vectors with margins
  if (d->precision == FREHG_GW_PRECISION_MIXED) b += 12 * r(4 * ns) + r(8 * ns);
  if (d->precision == FREHG_GW_PRECISION_FP64_LINE) b += 4 * r(8 * ns);
  const size_t nblk = std::min<size_t>((n3 + 255) / 256, 512 * 8);
  const size_t cg = std::max<size_t>((n3 + 255) / 256, 512 * 4);
  b += r(8 * fgw::kPSlots * nblk) + r(8 * 4 * cg) + r(sizeof(fgw::StepOut));
  const size_t page = 2u << 20;
  return (b + page - 1) / page * page;
}

int frehg_gw_server_create(const frehg_gw_server_opts* opts, frehg_gw_server** out) {
  if (!out) return fail(FREHG_GW_EINVAL, "server: null argument");
  *out = nullptr;
  auto* s = new frehg_gw_server;
  if (opts) s->opts = *opts;
  s->budget = s->opts.hbm_budget_bytes;
  s->slots = s->opts.max_active > 0 ? s->opts.max_active : 64;
  if (s->budget == 0) {
    size_t free_b = 0, total_b = 0;
    const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) {
      delete s;
      return cuda_fail(e, "server: device memory");
    }
    s->budget = free_b / 10 * 9;
  }
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    // No device to query (submission and queueing still work; admission
    // reports the device error per request).
    s->device = 0;
    cudaGetLastError();
  }
  s->t0 = Clock::now();
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return FREHG_GW_OK;
}

int frehg_gw_server_destroy(frehg_gw_server* s) {
  if (!s) return FREHG_GW_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->batch) frehg_gw_batch_destroy(s->batch);
  for (auto& r : s->active)
    if (r->h) frehg_gw_destroy(r->h);
  for (auto& r : s->ready)
    if (r->h) frehg_gw_destroy(r->h);
  for (auto& r : s->retiring)
    if (r->h) frehg_gw_destroy(r->h);
  delete s;
  return FREHG_GW_OK;
}

int frehg_gw_server_submit(frehg_gw_server* s, const frehg_gw_request* q, long long* id) {
  if (!s || !q || !q->desc || !id) return fail(FREHG_GW_EINVAL, "server: null argument");
  const frehg_gw_desc& d = *q->desc;
  if (d.nx < 1 || d.ny < 1 || d.nz < 1 || q->steps < 1)
    return fail(FREHG_GW_EINVAL, "server: empty domain or no steps");
  if (!d.ksx || !d.ksy || !d.ksz || !d.vg_alpha || !d.vg_n || !d.theta_s || !d.theta_r ||
      !d.aev || !d.top_code || !d.bot_code || !d.xm_code || !d.xp_code || !d.ym_code ||
      !d.yp_code)
    return fail(FREHG_GW_EINVAL, "server: descriptor arrays missing");
  auto r = std::make_unique<Request>();
  const size_t nx = d.nx, ny = d.ny, nz = d.nz, n2 = nx * ny, n3 = n2 * nz;
  r->desc = d;
  copy_in(r->dz, d.dz_layers, nz);
  r->has_bath = d.bath != nullptr;
  copy_in(r->bath, d.bath, n2);
  const double* soil[8] = {d.ksx, d.ksy, d.ksz, d.vg_alpha, d.vg_n, d.theta_s, d.theta_r, d.aev};
  for (int k = 0; k < 8; ++k) copy_in(r->soil[k], soil[k], n3);
  const int* codes[6] = {d.top_code, d.bot_code, d.xm_code, d.xp_code, d.ym_code, d.yp_code};
  const size_t csz[6] = {n2, n2, ny, ny, nx, nx};
  for (int k = 0; k < 6; ++k) copy_in(r->codes[k], codes[k], csz[k]);
  const double* bc[6] = {q->bc_top, q->bc_bottom, q->bc_xm, q->bc_xp, q->bc_ym, q->bc_yp};
  for (int k = 0; k < 6; ++k) {
    r->has_bc[k] = bc[k] != nullptr;
    copy_in(r->bc[k], bc[k], csz[k]);
  }
  r->ic_form = q->ic_form;
  r->ic_constant = q->ic_constant;
  r->has_field = q->ic_field != nullptr;
  copy_in(r->ic_field, q->ic_field, q->ic_form == FREHG_GW_IC_WATER_TABLE ? n2 : n3);
  r->desc.dz_layers = r->dz.empty() ? nullptr : r->dz.data();
  r->desc.bath = r->has_bath ? r->bath.data() : nullptr;
  r->desc.ksx = r->soil[0].data();
  r->desc.ksy = r->soil[1].data();
  r->desc.ksz = r->soil[2].data();
  r->desc.vg_alpha = r->soil[3].data();
  r->desc.vg_n = r->soil[4].data();
  r->desc.theta_s = r->soil[5].data();
  r->desc.theta_r = r->soil[6].data();
  r->desc.aev = r->soil[7].data();
  r->desc.top_code = r->codes[0].data();
  r->desc.bot_code = r->codes[1].data();
  r->desc.xm_code = r->codes[2].data();
  r->desc.xp_code = r->codes[3].data();
  r->desc.ym_code = r->codes[4].data();
  r->desc.yp_code = r->codes[5].data();
  r->steps = q->steps;
  r->bytes = frehg_gw_device_bytes(&r->desc);
  if (r->bytes > s->budget)
    return fail(FREHG_GW_ENOMEM, "server: request needs " + std::to_string(r->bytes) +
                                     " bytes of device memory; the budget is " +
                                     std::to_string(s->budget));
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    r->t_submit = now_s(s);
    *id = r->id;
    s->queue.push_back(std::move(r));
  }
  s->cv.notify_all();
  return FREHG_GW_OK;
}

int frehg_gw_server_tick(frehg_gw_server* s, int* active, int* queued) {
  if (!s) return fail(FREHG_GW_EINVAL, "null server");
  const auto tick0 = Clock::now();
  auto lap = [](Clock::time_point& t) {
    const auto now = Clock::now();
    const double d = std::chrono::duration<double>(now - t).count();
    t = now;
    return d;
  };
  auto t = tick0;
  // 1. Take in what the worker has made ready; with nothing to step, wait
  // briefly for the worker instead of spinning.
  {
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->active.empty() && s->ready.empty() && (s->busy > 0 || !s->queue.empty()))
      s->done.wait_for(lk, std::chrono::milliseconds(2));
    for (auto& r : s->ready) {
      r->state = FREHG_GW_REQ_RUNNING;
      s->active.push_back(std::move(r));
      s->dirty = true;
    }
    s->ready.clear();
  }
  // 2. One step of every running request, as one batch.
  int status = FREHG_GW_OK;
  if (!s->active.empty()) {
    if (s->dirty) {
      std::vector<frehg_gw_handle*> hs;
      for (auto& r : s->active) hs.push_back(r->h);
      int rc;
      if (s->batch) {
        rc = frehg_gw_batch_set_members(s->batch, hs.data(), static_cast<int>(hs.size()));
      } else {
        frehg_gw_batch_opts bo{};
        bo.cells_per_block = s->opts.cells_per_block;
        bo.use_graph = s->opts.use_graph;
        bo.streams = s->opts.streams;
        rc = frehg_gw_batch_create(hs.data(), static_cast<int>(hs.size()), &bo, &s->batch);
      }
      if (rc != FREHG_GW_OK) return rc;
      s->dirty = false;
    }
    s->rebatch_s += lap(t);
    std::vector<frehg_gw_step_info> infos(s->active.size());
    std::vector<double> dts(s->active.size());
    for (size_t i = 0; i < s->active.size(); ++i) dts[i] = s->active[i]->h->next_dt;
    const int rc = frehg_gw_batch_step(s->batch, infos.data());
    if (rc == FREHG_GW_ECUDA) status = rc;  // device trouble: report, keep state
    s->step_s += lap(t);
    // 3. Progress; requests done (or failed) go to the worker for retirement.
    std::vector<std::unique_ptr<Request>> keep, out;
    for (size_t i = 0; i < s->active.size(); ++i) {
      std::unique_ptr<Request>& r = s->active[i];
      if (infos[i].status == FREHG_GW_OK) {
        ++r->done_steps;
        r->sim_t += dts[i];
        r->last = infos[i];
        s->cell_steps += r->cells;
      }
      if (infos[i].status != FREHG_GW_OK || r->done_steps >= r->steps) {
        r->status = infos[i].status;
        if (r->status != FREHG_GW_OK)
          r->error = "step failed (status " + std::to_string(r->status) + ")";
        out.push_back(std::move(r));
      } else {
        keep.push_back(std::move(r));
      }
    }
    s->active.swap(keep);
    if (!out.empty()) {
      s->dirty = true;
      std::lock_guard<std::mutex> lk(s->mu);
      for (auto& r : out) {
        s->retiring.push_back(std::move(r));
        --s->held;
      }
    }
    s->cv.notify_all();
    ++s->ticks;
  }
  s->busy_s += std::chrono::duration<double>(Clock::now() - tick0).count();
  std::lock_guard<std::mutex> lk(s->mu);
  if (active) *active = static_cast<int>(s->active.size() + s->ready.size());
  if (queued)
    *queued = static_cast<int>(s->queue.size() + s->retiring.size()) + s->busy;
  return status;
}

int frehg_gw_server_poll(frehg_gw_server* s, long long id, frehg_gw_request_status* st) {
  if (!s || !st) return fail(FREHG_GW_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  Request* r = find(s, id);
  if (!r) return fail(FREHG_GW_EINVAL, "server: unknown or released request");
  st->state = r->state;
  st->status = r->status;
  st->steps = r->steps;
  st->steps_done = r->done_steps;
  st->cells = r->cells;
  st->sim_time = r->sim_t;
  st->submit_s = r->t_submit;
  st->queue_s = r->t_admit >= 0.0 ? r->t_admit - r->t_submit : -1.0;
  st->latency_s = r->t_done >= 0.0 ? r->t_done - r->t_submit : -1.0;
  st->last = r->last;
  return FREHG_GW_OK;
}

int frehg_gw_server_fetch(frehg_gw_server* s, long long id, int field, double* out) {
  if (!s || !out) return fail(FREHG_GW_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  Request* r = find(s, id);
  if (!r || r->state != FREHG_GW_REQ_DONE)
    return fail(FREHG_GW_ESTATE, "server: request not finished");
  const std::vector<double>* v = field == FREHG_GW_FIELD_HEAD ? &r->head
                                 : field == FREHG_GW_FIELD_WC ? &r->wc
                                                              : nullptr;
  if (!v) return fail(FREHG_GW_EINVAL, "server: only head and water content are kept");
  std::copy(v->begin(), v->end(), out);
  return FREHG_GW_OK;
}

int frehg_gw_server_release(frehg_gw_server* s, long long id) {
  if (!s) return fail(FREHG_GW_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->finished.find(id);
  if (it == s->finished.end()) return fail(FREHG_GW_ESTATE, "server: request not finished");
  s->finished.erase(it);
  return FREHG_GW_OK;
}

int frehg_gw_server_stats(const frehg_gw_server* s, frehg_gw_server_stats_t* st) {
  if (!s || !st) return fail(FREHG_GW_EINVAL, "null argument");
  auto* m = const_cast<frehg_gw_server*>(s);
  std::lock_guard<std::mutex> lk(m->mu);
  st->active = static_cast<int>(s->active.size() + s->ready.size());
  // As frehg_gw_server_tick counts them: waiting, being admitted or retired by
  // the worker (a request in the worker's hands is in no container).
  st->queued = static_cast<int>(s->queue.size() + s->retiring.size()) + s->busy;
  st->completed = s->completed;
  st->ticks = s->ticks;
  st->cell_steps = s->cell_steps;
  st->device_bytes_used = s->used;
  st->device_bytes_budget = s->budget;
  st->busy_s = s->busy_s;
  st->admit_s = s->admit_s;
  st->rebatch_s = s->rebatch_s;
  st->step_s = s->step_s;
  st->retire_s = s->retire_s;
  st->now_s = now_s(s);
  return FREHG_GW_OK;
}

}  // extern "C"
