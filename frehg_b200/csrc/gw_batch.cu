// Batched stepping of many independent domains (frehg_gw_batch_*).
//
// A batch is a view over existing handles.  One batch step runs every
// member's step with the member's own dt:
//
//   1.     the predictor phases of all members -- step-start ghost refresh,
//          closure, assembly (and the mixed form's FP32 cast and line
//          factorisation) -- one launch per phase, each member on its
//          single-domain block count

//   2.     the predictor solves of all members in one cooperative launch per
//          solve kind (FP64, mixed) of at most the device's co-resident
//          blocks, each member in its own class's form (column layout, vector
//          width) on its own block count with its own CG state, reductions
//          and barrier; the blocks take the members' block slots from a queue
//          ordered by estimated work, so the blocks of a member whose solve
//          has converged go straight on to the next waiting member's slots
//   3.     corrector, post-allocation, clamp, audit and controller of all
//          members, one launch per phase, and one read-back of all step
//          records; one synchronisation for the whole batch
//
// Each phase launch reads every member's arguments (state buffers of its
// current parity, dt) from a table the host refreshes in pinned memory before
// the step, so the whole step is captured once as a CUDA graph and replayed.
// With per_member_phases the non-solve kernels are instead launched member by
// member on a pool of streams (the members' dt then travels through their
// device step records, and one graph is captured per pattern of parities).
//
// A member's block counts depend on its own size and the batch options only,
// never on the other members, so a member's arithmetic (including the order
// of every reduction) is the same alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gw_coop.cuh"
#include "gw_handle.h"

using fgw_api::cuda_fail;
using fgw_api::fail;

namespace fgw {

namespace {

// Before a group's solve launch, one block: ranks the members by estimated
// work, nb (iterations of the previous solve + 4), largest first, ties by
// table index (up to kRankMax members; beyond, table order), writes the queue
// order and its slot offsets, then zeroes the members' CG states and the
// slot counter.  The order only decides which member's slots go out first;
// a member's arithmetic depends on its own block count alone.
constexpr int kRankMax = 1024;

__global__ void k_queue_setup(CgState** st, const int* __restrict__ first, int n, int* queue,
                              int* order, int* ofirst) {
  __shared__ int part[256];
  const int t = threadIdx.x;
  if (n <= kRankMax) {
    for (int i = t; i < n; i += blockDim.x) {
      const long long wi = static_cast<long long>(first[i + 1] - first[i]) * (st[i]->its + 4);
      int rank = 0;
      for (int j = 0; j < n; ++j) {
        const long long wj = static_cast<long long>(first[j + 1] - first[j]) * (st[j]->its + 4);
        rank += (wj > wi || (wj == wi && j < i)) ? 1 : 0;
      }
      order[rank] = i;
    }
  } else {
    for (int i = t; i < n; i += blockDim.x) order[i] = i;
  }
  __syncthreads();
  // ofirst: exclusive prefix of the block counts in queue order, by chunks
  // of blockDim.x members (a thread sums its chunk, the block scans the sums).
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int lo = t * per, hi = min(n, lo + per);
  int sum = 0;
  for (int q = lo; q < hi; ++q) sum += first[order[q] + 1] - first[order[q]];
  part[t] = sum;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int u = 0; u < static_cast<int>(blockDim.x); ++u) {
      const int v = part[u];
      part[u] = run;
      run += v;
    }
    ofirst[n] = run;
  }
  __syncthreads();
  int run = part[t];
  for (int q = lo; q < hi; ++q) {
    ofirst[q] = run;
    run += first[order[q] + 1] - first[order[q]];
  }
  __syncthreads();
  for (int i = t; i < n; i += blockDim.x) {
    CgState* s = st[i];
    s->dp = 0.0;
    s->rnorm0 = 0.0;
    s->its = 0;
    s->reason = 0;
    s->outer = 0;
    s->err = 0;
    s->bar_count = 0u;
    s->bar_gen = 0u;
  }
  if (t == 0) *queue = 0;
}

size_t args_bytes(const SolveClass& c) {
  return c.kind == 0 ? cg64_args_bytes() : mixed_args_bytes();
}

const void* batch_kernel(const SolveClass& c) {
  return c.kind == 0 ? cg64_batch_kernel() : mixed_batch_kernel();
}

}  // namespace

SolveClass solve_class(const Device& D, int precision, bool tiled_line_solve) {
  if (precision == FREHG_GW_PRECISION_MIXED) return SolveClass{1, mixed_variant(D, tiled_line_solve)};
  return SolveClass{0, (D.d.nz % 2 == 0) ? 1 : 0};
}

int solve_blocks_per_sm(const SolveClass& c, size_t smem) {
  const void* k = batch_kernel(c);
  if (smem > 0) raise_smem_limit(k, smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, coop::kCgBlock, smem) !=
      cudaSuccess)
    per_sm = 0;
  return per_sm;
}

int solve_max_blocks(const Device& D, const SolveClass& c) {
  // The member's reduction buffer holds 4 max(cg_grid, cg_grid32) doubles;
  // a solve on G blocks uses 3 G of them (FP64) or 4 G (mixed).
  const int cap = (4 * std::max(D.cg_grid, D.cg_grid32)) / (c.kind == 1 ? 4 : 3);
  return std::max(1, cap);
}

size_t solve_group_bytes(const SolveClass& c, int n) {
  auto r = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  return r(args_bytes(c) * n) + r(sizeof(int) * (n + 1)) + r(sizeof(CgState*) * n) +
         r(sizeof(int)) + r(sizeof(int) * n) + r(sizeof(int) * (n + 1));
}

cudaError_t solve_group_build(SolveGroup& g, const SolveClass& c, const std::vector<Device*>& ds,
                              const std::vector<int>& variants, const std::vector<int>& nb,
                              const std::vector<SolveParams>& p, int max_grid, void* mem) {
  g.cls = c;
  g.n = static_cast<int>(ds.size());
  const size_t ab = args_bytes(c);
  std::vector<unsigned char> tab(ab * ds.size());
  std::vector<int> first(ds.size() + 1, 0);
  std::vector<CgState*> st(ds.size());
  g.smem = 0;
  for (size_t i = 0; i < ds.size(); ++i) {
    if (c.kind == 0) cg64_fill_args(*ds[i], p[i], variants[i], tab.data() + i * ab);
    else mixed_fill_args(*ds[i], p[i], variants[i], tab.data() + i * ab);
    first[i + 1] = first[i] + nb[i];
    st[i] = &ds[i]->out->cg;
    if (c.kind == 1) g.smem = std::max(g.smem, mixed_batch_smem(*ds[i], variants[i]));
  }
  g.slots = first.back();
  g.grid = std::min(g.slots, max_grid);
  auto r = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  char* base = static_cast<char*>(mem);
  g.tab = base;
  g.first = reinterpret_cast<int*>(base + r(tab.size()));
  g.states = reinterpret_cast<CgState**>(base + r(tab.size()) + r(first.size() * sizeof(int)));
  char* q = base + r(tab.size()) + r(first.size() * sizeof(int)) +
            r(st.size() * sizeof(CgState*));
  g.queue = reinterpret_cast<int*>(q);
  g.order = reinterpret_cast<int*>(q + r(sizeof(int)));
  g.ofirst = reinterpret_cast<int*>(q + r(sizeof(int)) + r(sizeof(int) * ds.size()));
  cudaError_t e = cudaMemcpy(g.tab, tab.data(), tab.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(g.first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(g.states, st.data(), st.size() * sizeof(CgState*), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && g.smem > 0)
    e = raise_smem_limit(batch_kernel(c), g.smem);
  return e;
}

cudaError_t solve_group_launch(const SolveGroup& g, cudaStream_t s) {
  k_queue_setup<<<1, 256, 0, s>>>(g.states, g.first, g.n, g.queue, g.order, g.ofirst);
  void* tab = g.tab;
  int* first = g.first;
  int n = g.n;
  int* queue = g.queue;
  int* order = g.order;
  int* ofirst = g.ofirst;
  void* args[] = {&tab, &first, &n, &queue, &order, &ofirst};
  return cudaLaunchCooperativeKernel(batch_kernel(g.cls), dim3(g.grid), dim3(coop::kCgBlock), args,
                                     g.smem, s);
}


}  // namespace fgw

// ---------------------------------------------------------------- the batch
struct frehg_gw_batch {
  std::vector<frehg_gw_handle*> m;
  int device = 0;                   // the members' device
  frehg_gw_batch_opts opts{};
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> pool;
  cudaEvent_t fork1 = nullptr, fork2 = nullptr;
  std::vector<cudaEvent_t> join1, join2;
  std::vector<fgw::SolveGroup> groups;
  std::vector<int> nb;              // solve blocks per member
  std::map<std::vector<unsigned char>, cudaGraphExec_t> graphs;  // by member parities
  long long launches = 0;           // kernels launched by batch steps
  long long launches_per_step = 0;  // of the last step
  long long steps = 0;
  std::string graph_error;          // why graphs were given up, if they were
  fgw::PhaseTables phases;          // batched non-solve phases
  void* group_mem = nullptr;        // the solve groups' tables
  size_t group_cap = 0;
  cudaEvent_t ev[4] = {};           // step start, after predictor, after solves, end
  double phase_ms[3] = {0, 0, 0};   // of the last step
};

namespace {

constexpr int kDefaultCellsPerBlock = 16384;
constexpr int kDefaultStreams = 32;

void free_groups(frehg_gw_batch* b) { b->groups.clear(); }

void drop_graphs(frehg_gw_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
}

// Block counts and cooperative launch groups for the current options.
int build_groups(frehg_gw_batch* b) {
  free_groups(b);
  drop_graphs(b);
  const int n = static_cast<int>(b->m.size());
  const long long cpb = b->opts.cells_per_block > 0 ? b->opts.cells_per_block
                                                    : kDefaultCellsPerBlock;
  const bool tiled = b->opts.tiled_line_solve != 0;
  std::vector<fgw::SolveClass> cls(n);
  b->nb.assign(n, 1);
  for (int i = 0; i < n; ++i) {
    frehg_gw_handle* h = b->m[i];
    cls[i] = fgw::solve_class(h->D, h->precision, tiled);
    const long long want = (h->nactive + cpb - 1) / cpb;
    b->nb[i] = static_cast<int>(std::max(1LL, std::min<long long>(
                                                  want, fgw::solve_max_blocks(h->D, cls[i]))));
  }
  // The members of one solve kind (FP64, mixed) share one launch of at most
  // the device's co-resident blocks, each in its own class's form; they
  // queue for those blocks, largest estimated work first (k_queue_setup), so
  // the longest solves start first and the small ones fill the tail.
  struct Spec {
    fgw::SolveClass c;
    int cap = 0;
    std::vector<fgw::Device*> ds;
    std::vector<int> variants;
    std::vector<int> nbs;
    std::vector<fgw::SolveParams> ps;
  };
  std::vector<Spec> specs;
  for (int kind = 0; kind < 2; ++kind) {
    size_t smem = 0;
    bool any = false;
    for (int j = 0; j < n; ++j) {
      if (cls[j].kind != kind) continue;
      any = true;
      if (kind == 1) smem = std::max(smem, fgw::mixed_batch_smem(b->m[j]->D, cls[j].variant));
    }
    if (!any) continue;
    const fgw::SolveClass c{kind, 0};
    const int per_sm = fgw::solve_blocks_per_sm(c, smem);
    if (per_sm < 1) return fail(FREHG_GW_ECUDA, "batch: solve kernel cannot be resident");
    Spec cur{c, 0, {}, {}, {}, {}};
    for (int j = 0; j < n; ++j) {
      if (cls[j].kind != kind) continue;
      frehg_gw_handle* h = b->m[j];
      cur.cap = per_sm * h->D.sm_count;
      b->nb[j] = std::min(b->nb[j], cur.cap);
      cur.ds.push_back(&h->D);
      cur.variants.push_back(cls[j].variant);
      cur.nbs.push_back(b->nb[j]);
      cur.ps.push_back(fgw::SolveParams{h->rtol, h->atol, h->outer_rtol, h->maxit, h->max_outer});
    }
    specs.push_back(cur);
  }
  // One device allocation for every group's tables, kept while it fits.
  size_t need = 0;
  for (const auto& sp : specs) need += fgw::solve_group_bytes(sp.c, static_cast<int>(sp.ds.size()));
  if (need > b->group_cap) {
    const size_t cap = std::max(need, 2 * b->group_cap);
    if (b->group_mem) cudaFree(b->group_mem);
    b->group_mem = nullptr;
    b->group_cap = 0;
    const cudaError_t e = cudaMalloc(&b->group_mem, cap);
    if (e != cudaSuccess) return cuda_fail(e, "batch: solve tables");
    b->group_cap = cap;
  }
  size_t off = 0;
  for (const auto& sp : specs) {
    fgw::SolveGroup g;
    const cudaError_t e = fgw::solve_group_build(g, sp.c, sp.ds, sp.variants, sp.nbs, sp.ps,
                                                 sp.cap, static_cast<char*>(b->group_mem) + off);
    if (e != cudaSuccess) return cuda_fail(e, "batch: solve group");
    off += fgw::solve_group_bytes(sp.c, static_cast<int>(sp.ds.size()));
    b->groups.push_back(g);
  }
  return FREHG_GW_OK;
}

// Enqueues one batch step with batched phases on b->stream (under capture
// or not); the member records must be filled.  Counts kernels into *kernels.
cudaError_t enqueue_batched_phases(frehg_gw_batch* b, long long* kernels) {
  const fgw::PhaseTables& t = b->phases;
  // Phase timing events only on direct launches (a graph replay does not
  // time captured events).
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(b->stream, &cap);
  const bool timed = cap == cudaStreamCaptureStatusNone;
  auto mark = [&](int k) { return timed ? cudaEventRecord(b->ev[k], b->stream) : cudaSuccess; };
  cudaError_t e = mark(0);
  if (e == cudaSuccess) e = fgw::batch_predictor(t, b->stream);
  if (e == cudaSuccess) e = mark(1);
  long long k = 4 + (t.grid_factor > 0 ? 1 : 0);
  for (const auto& g : b->groups) {
    if (e != cudaSuccess) break;
    e = fgw::solve_group_launch(g, b->stream);
    k += 2;
  }
  if (e == cudaSuccess) e = mark(2);
  if (e == cudaSuccess) e = fgw::batch_corrector(t, b->stream);
  if (e == cudaSuccess) e = mark(3);
  *kernels = k + 8;
  return e;
}

// Enqueues one batch step, member by member, on b->stream and its pool
// (under capture or not).  Counts the kernels it launches into *kernels.
cudaError_t enqueue_member_phases(frehg_gw_batch* b, long long* kernels) {
  const int n = static_cast<int>(b->m.size());
  const int P = static_cast<int>(b->pool.size());
  long long before = 0;
  for (auto* h : b->m) before += h->D.launches;
  std::vector<cudaStream_t> own(n);
  cudaError_t e = cudaEventRecord(b->fork1, b->stream);
  for (int p = 0; p < P && e == cudaSuccess; ++p) e = cudaStreamWaitEvent(b->pool[p], b->fork1, 0);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    frehg_gw_handle* h = b->m[i];
    own[i] = h->D.stream;
    h->D.stream = b->pool[i % P];
    e = cudaMemcpyAsync(&h->D.out->next_dt, &h->D.out_host->next_dt, sizeof(double),
                        cudaMemcpyHostToDevice, h->D.stream);
    if (e == cudaSuccess) e = fgw_api::enqueue_predictor(h);
  }
  for (int p = 0; p < P && e == cudaSuccess; ++p) {
    e = cudaEventRecord(b->join1[p], b->pool[p]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join1[p], 0);
  }
  long long solves = 0;
  for (const auto& g : b->groups) {
    if (e != cudaSuccess) break;
    e = fgw::solve_group_launch(g, b->stream);
    solves += 2;
  }
  if (e == cudaSuccess) e = cudaEventRecord(b->fork2, b->stream);
  for (int p = 0; p < P && e == cudaSuccess; ++p) e = cudaStreamWaitEvent(b->pool[p], b->fork2, 0);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    frehg_gw_handle* h = b->m[i];
    fgw_api::enqueue_corrector(h);
    e = cudaMemcpyAsync(h->D.out_host, h->D.out, sizeof(fgw::StepOut), cudaMemcpyDeviceToHost,
                        h->D.stream);
  }
  for (int p = 0; p < P && e == cudaSuccess; ++p) {
    e = cudaEventRecord(b->join2[p], b->pool[p]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join2[p], 0);
  }
  for (int i = 0; i < n; ++i)
    if (own[i]) b->m[i]->D.stream = own[i];
  long long after = 0;
  for (auto* h : b->m) after += h->D.launches;
  *kernels = (after - before) + solves;
  return e;
}

// The solve groups and the phase tables of the current members.
int build_member_tables(frehg_gw_batch* b) {
  int rc = build_groups(b);
  if (rc != FREHG_GW_OK) return rc;
  std::vector<const fgw::Device*> ds;
  std::vector<int> mixed;
  for (auto* h : b->m) {
    ds.push_back(&h->D);
    mixed.push_back(h->precision == FREHG_GW_PRECISION_MIXED ? 1 : 0);
  }
  const cudaError_t ep = fgw::phase_tables_build(b->phases, ds, mixed);
  return ep == cudaSuccess ? FREHG_GW_OK : cuda_fail(ep, "batch: phase tables");
}

std::vector<unsigned char> parities(const frehg_gw_batch* b) {
  if (!b->opts.per_member_phases) return {};  // one graph serves every parity pattern
  std::vector<unsigned char> k(b->m.size());
  for (size_t i = 0; i < b->m.size(); ++i) k[i] = static_cast<unsigned char>(b->m[i]->D.cur);
  return k;
}

// Runs one batch step (graph replay when possible) and waits for it.
int run_step(frehg_gw_batch* b) {
  const bool batched = !b->opts.per_member_phases;
  auto enqueue = batched ? enqueue_batched_phases : enqueue_member_phases;
  if (batched) {
    for (size_t i = 0; i < b->m.size(); ++i) {
      const frehg_gw_handle* h = b->m[i];
      fgw::fill_step_args(h->D, h->precision == FREHG_GW_PRECISION_MIXED, h->next_dt, h->co_max,
                          h->dq_grow, h->dq_shrink, h->dt_min, h->dt_max, b->phases.tab_host[i]);
    }
  } else {
    for (auto* h : b->m) h->D.out_host->next_dt = h->next_dt;
  }
  long long kernels = 0;
  cudaError_t e = cudaSuccess;
  bool ran = false;
  if (b->opts.use_graph && b->graph_error.empty()) {
    const auto key = parities(b);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const cudaError_t ee = enqueue(b, &kernels);
        e = cudaStreamEndCapture(b->stream, &graph);
        if (ee != cudaSuccess) e = ee;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        // Give up graphs for this batch and launch directly from now on.
        b->graph_error = cudaGetErrorString(e);
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
      } else {
        it = b->graphs.emplace(key, exec).first;
        b->launches_per_step = kernels;
      }
    }
    if (b->graph_error.empty()) {
      e = cudaGraphLaunch(it->second, b->stream);
      if (e != cudaSuccess) return cuda_fail(e, "batch step (graph)");
      ran = true;
      kernels = b->launches_per_step;
    }
  }
  if (!ran) {
    e = enqueue(b, &kernels);
    if (e != cudaSuccess) return cuda_fail(e, "batch step");
    b->launches_per_step = kernels;
  }
  e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch step");
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "batch step kernels");
  if (batched) {
    for (size_t i = 0; i < b->m.size(); ++i) *b->m[i]->D.out_host = b->phases.outs_host[i];
    if (!ran) {
      for (int p = 0; p < 3; ++p) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, b->ev[p], b->ev[p + 1]) == cudaSuccess) b->phase_ms[p] = ms;
        else cudaGetLastError();
      }
    }
  }
  b->launches += kernels;
  ++b->steps;
  return FREHG_GW_OK;
}

// Member state a step changes (for the autotuner's trial steps).
struct Snapshot {
  std::vector<double*> h, wc, vloss;
  std::vector<double> next_dt;
  std::vector<int> cur, start_buf;
};

int snapshot_take(frehg_gw_batch* b, Snapshot& s) {
  for (auto* hd : b->m) {
    const size_t bytes = hd->D.d.ncell * sizeof(double);
    double *a = nullptr, *c = nullptr, *v = nullptr;
    cudaError_t e = cudaMalloc(&a, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&v, bytes);
    s.h.push_back(a);
    s.wc.push_back(c);
    s.vloss.push_back(v);
    if (e != cudaSuccess) return cuda_fail(e, "autotune snapshot");
    cudaMemcpyAsync(a, hd->D.h[hd->D.cur], bytes, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(c, hd->D.wc[hd->D.cur], bytes, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(v, hd->D.vloss, bytes, cudaMemcpyDeviceToDevice, b->stream);
    s.next_dt.push_back(hd->next_dt);
    s.cur.push_back(hd->D.cur);
    s.start_buf.push_back(hd->start_buf);
  }
  const cudaError_t e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? FREHG_GW_OK : cuda_fail(e, "autotune snapshot");
}

int snapshot_restore(frehg_gw_batch* b, const Snapshot& s) {
  for (size_t i = 0; i < b->m.size(); ++i) {
    frehg_gw_handle* hd = b->m[i];
    const size_t bytes = hd->D.d.ncell * sizeof(double);
    hd->D.cur = s.cur[i];
    hd->start_buf = s.start_buf[i];
    hd->next_dt = s.next_dt[i];
    cudaMemcpyAsync(hd->D.h[hd->D.cur], s.h[i], bytes, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(hd->D.wc[hd->D.cur], s.wc[i], bytes, cudaMemcpyDeviceToDevice, b->stream);
    cudaMemcpyAsync(hd->D.vloss, s.vloss[i], bytes, cudaMemcpyDeviceToDevice, b->stream);
  }
  const cudaError_t e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? FREHG_GW_OK : cuda_fail(e, "autotune restore");
}

void snapshot_free(Snapshot& s) {
  for (auto* p : s.h) if (p) cudaFree(p);
  for (auto* p : s.wc) if (p) cudaFree(p);
  for (auto* p : s.vloss) if (p) cudaFree(p);
  s = Snapshot{};
}

std::mutex g_tune_mu;
std::map<std::string, frehg_gw_batch_opts> g_tune_cache;

std::string tune_key(const frehg_gw_batch* b) {
  std::string k = std::to_string(b->m.size());
  for (auto* h : b->m) {
    k += ':' + std::to_string(h->D.d.nx) + 'x' + std::to_string(h->D.d.ny) + 'x' +
         std::to_string(h->D.d.nz) + (h->precision == FREHG_GW_PRECISION_MIXED ? 'm' : 'd');
  }
  return k;
}

}  // namespace

extern "C" {

int frehg_gw_batch_create(frehg_gw_handle* const* members, int n,
                          const frehg_gw_batch_opts* opts, frehg_gw_batch** out) {
  if (!members || !out || n < 1) return fail(FREHG_GW_EINVAL, "batch: null argument or n < 1");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return fail(FREHG_GW_EINVAL, "batch: null member");
    if (!members[i]->have_state) return fail(FREHG_GW_ESTATE, "batch: member without state");
    if (members[i]->device != members[0]->device)
      return fail(FREHG_GW_EINVAL, "batch: members on different devices");
    if (members[i]->precision == FREHG_GW_PRECISION_FP64_LINE)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: the FP64 line form steps on its own");
    if (members[i]->D.f.cpl)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: a coupled-top member steps on its own");
    if (members[i]->D.win_x)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: a member with a transport window steps on its own");
    if (members[i]->D.f.baro)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: a member with density coupling steps on its own");
    for (int j = 0; j < i; ++j)
      if (members[j] == members[i]) return fail(FREHG_GW_EINVAL, "batch: member given twice");
  }
  FGW_ON_DEVICE(members[0]);
  auto* b = new frehg_gw_batch;
  b->device = members[0]->device;
  b->m.assign(members, members + n);
  if (opts) b->opts = *opts;
  else b->opts.use_graph = 1;
  // The stream pool serves the member-by-member path only.
  const int P = b->opts.per_member_phases
                    ? std::max(1, std::min(n, b->opts.streams > 0 ? b->opts.streams
                                                                  : kDefaultStreams))
                    : 0;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  b->pool.resize(P, nullptr);
  b->join1.resize(P, nullptr);
  b->join2.resize(P, nullptr);
  for (int p = 0; p < P && e == cudaSuccess; ++p) {
    e = cudaStreamCreateWithFlags(&b->pool[p], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join1[p], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join2[p], cudaEventDisableTiming);
  }
  for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = cudaEventCreate(&b->ev[k]);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork1, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork2, cudaEventDisableTiming);
  int rc = (e == cudaSuccess) ? FREHG_GW_OK : cuda_fail(e, "batch: streams");
  if (rc == FREHG_GW_OK) rc = build_member_tables(b);
  if (rc != FREHG_GW_OK) {
    frehg_gw_batch_destroy(b);
    return rc;
  }
  *out = b;
  return FREHG_GW_OK;
}

int frehg_gw_batch_set_members(frehg_gw_batch* b, frehg_gw_handle* const* members, int n) {
  if (!b || !members || n < 1) return fail(FREHG_GW_EINVAL, "batch: null argument or n < 1");
  FGW_ON_DEVICE(b);
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return fail(FREHG_GW_EINVAL, "batch: null member");
    if (!members[i]->have_state) return fail(FREHG_GW_ESTATE, "batch: member without state");
    if (members[i]->device != b->device)
      return fail(FREHG_GW_EINVAL, "batch: members on different devices");
    if (members[i]->precision == FREHG_GW_PRECISION_FP64_LINE)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: the FP64 line form steps on its own");
    if (members[i]->D.f.cpl)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: a coupled-top member steps on its own");
    if (members[i]->D.win_x)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: a member with a transport window steps on its own");
    if (members[i]->D.f.baro)
      return fail(FREHG_GW_EUNSUPPORTED, "batch: a member with density coupling steps on its own");
  }
  const cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch: set members");
  b->m.assign(members, members + n);
  return build_member_tables(b);
}

int frehg_gw_batch_destroy(frehg_gw_batch* b) {
  if (!b) return FREHG_GW_OK;
  FGW_ON_DEVICE(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  free_groups(b);
  if (b->group_mem) cudaFree(b->group_mem);
  fgw::phase_tables_free(b->phases);
  for (auto s : b->pool) if (s) cudaStreamDestroy(s);
  for (auto ev : b->join1) if (ev) cudaEventDestroy(ev);
  for (auto ev : b->join2) if (ev) cudaEventDestroy(ev);
  for (auto ev : b->ev) if (ev) cudaEventDestroy(ev);
  if (b->fork1) cudaEventDestroy(b->fork1);
  if (b->fork2) cudaEventDestroy(b->fork2);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FREHG_GW_OK;
}

int frehg_gw_batch_step(frehg_gw_batch* b, frehg_gw_step_info* infos) {
  if (!b) return fail(FREHG_GW_EINVAL, "null batch");
  FGW_ON_DEVICE(b);
  for (auto* h : b->m)
    if (!(h->next_dt > 0.0) || !std::isfinite(h->next_dt))
      return fail(FREHG_GW_EINVAL, "batch: member dt must be positive");
  const int rc = run_step(b);
  if (rc != FREHG_GW_OK) return rc;
  int first_bad = FREHG_GW_OK;
  std::string msg;
  for (size_t i = 0; i < b->m.size(); ++i) {
    const int s = fgw_api::finish_step(b->m[i], infos ? &infos[i] : nullptr);
    b->m[i]->have_prev = false;  // batched steps start from h^n
    if (s != FREHG_GW_OK && first_bad == FREHG_GW_OK) {
      first_bad = s;
      msg = "batch member " + std::to_string(i) + ": " + frehg_gw_last_error();
    }
  }
  if (first_bad != FREHG_GW_OK) return fail(first_bad, msg);
  return FREHG_GW_OK;
}

int frehg_gw_batch_set_dt(frehg_gw_batch* b, int i, double dtg) {
  if (!b || i < 0 || i >= static_cast<int>(b->m.size()))
    return fail(FREHG_GW_EINVAL, "batch: bad member index");
  if (!(dtg > 0.0) || !std::isfinite(dtg)) return fail(FREHG_GW_EINVAL, "dtg must be positive");
  b->m[i]->next_dt = dtg;
  return FREHG_GW_OK;
}

int frehg_gw_batch_autotune(frehg_gw_batch* b, int trials, frehg_gw_batch_opts* chosen,
                            double* best_ms) {
  if (!b) return fail(FREHG_GW_EINVAL, "null batch");
  FGW_ON_DEVICE(b);
  if (trials < 1) trials = 1;
  const std::string key = tune_key(b);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      b->opts.cells_per_block = it->second.cells_per_block;
      b->opts.tiled_line_solve = it->second.tiled_line_solve;
      const int rc = build_groups(b);
      if (chosen) *chosen = b->opts;
      if (best_ms) *best_ms = -1.0;
      return rc;
    }
  }
  bool any_mixed_columns = false;
  for (auto* h : b->m)
    if (h->precision == FREHG_GW_PRECISION_MIXED && h->D.d.nz <= 256) any_mixed_columns = true;
  const int cpbs[] = {4096, 8192, 16384, 32768, 65536, 131072};
  Snapshot snap;
  int rc = snapshot_take(b, snap);
  const frehg_gw_batch_opts start = b->opts;
  frehg_gw_batch_opts best = start;
  double best_t = 1e300;
  for (int tiled = 0; tiled <= (any_mixed_columns ? 1 : 0) && rc == FREHG_GW_OK; ++tiled) {
    for (int cpb : cpbs) {
      b->opts.cells_per_block = cpb;
      b->opts.tiled_line_solve = tiled;
      rc = build_groups(b);
      if (rc != FREHG_GW_OK) break;
      double t = 1e300;
      for (int k = 0; k <= trials && rc == FREHG_GW_OK; ++k) {
        rc = snapshot_restore(b, snap);
        if (rc != FREHG_GW_OK) break;
        const auto t0 = std::chrono::steady_clock::now();
        rc = run_step(b);
        const auto t1 = std::chrono::steady_clock::now();
        // k = 0 captures the graph; the later trials are timed.
        if (k > 0) t = std::min(t, std::chrono::duration<double, std::milli>(t1 - t0).count());
      }
      if (rc == FREHG_GW_OK && t < best_t) {
        best_t = t;
        best = b->opts;
      }
    }
  }
  if (rc == FREHG_GW_OK) rc = snapshot_restore(b, snap);
  snapshot_free(snap);
  b->opts.cells_per_block = best.cells_per_block;
  b->opts.tiled_line_solve = best.tiled_line_solve;
  const int rb = build_groups(b);
  if (rc == FREHG_GW_OK) rc = rb;
  b->steps = 0;
  b->launches = 0;
  if (rc != FREHG_GW_OK) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = b->opts;
  }
  if (chosen) *chosen = b->opts;
  if (best_ms) *best_ms = best_t;
  return FREHG_GW_OK;
}

int frehg_gw_batch_stats(const frehg_gw_batch* b, frehg_gw_batch_stats_t* out) {
  if (!b || !out) return fail(FREHG_GW_EINVAL, "null argument");
  out->members = static_cast<int>(b->m.size());
  out->solve_launches = static_cast<int>(b->groups.size());
  out->solve_blocks = 0;
  for (const auto& g : b->groups) out->solve_blocks += g.grid;
  out->graphs = static_cast<int>(b->graphs.size());
  out->uses_graph = (b->opts.use_graph && b->graph_error.empty()) ? 1 : 0;
  out->steps = b->steps;
  out->kernel_launches = b->launches;
  out->kernels_per_step = b->launches_per_step;
  out->cells_per_block = b->opts.cells_per_block > 0 ? b->opts.cells_per_block
                                                     : kDefaultCellsPerBlock;
  out->tiled_line_solve = b->opts.tiled_line_solve;
  for (int p = 0; p < 3; ++p) out->phase_ms[p] = b->phase_ms[p];
  return FREHG_GW_OK;
}

int frehg_gw_batch_solve_blocks(const frehg_gw_batch* b, int* nb) {
  if (!b || !nb) return fail(FREHG_GW_EINVAL, "null argument");
  for (size_t i = 0; i < b->nb.size(); ++i) nb[i] = b->nb[i];
  return FREHG_GW_OK;
}

}  // extern "C"
