// C ABI entry points (include/openjij_b200.h): context, graph upload, the SA
// and SQA runs with their planner, FP64 energies.  No exception crosses the
// ABI; every CUDA error becomes a status with a message in the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "oj_internal.h"

namespace oj {
oj_status finish_graph(oj_ctx* ctx, oj_graph* g);
cudaError_t ensure_dense(oj_graph* g);
}  // namespace oj

using namespace oj;

namespace {

constexpr const char* kVersion = "openjij_b200 0.1.0 (sm_100a)";

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

oj_status cuda_fail(oj_ctx* ctx, cudaError_t e, const char* where) {
  if (ctx) ctx->last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? OJ_ERR_OOM : OJ_ERR_CUDA;
}

#define OJ_CK(call, where)                              \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, where); \
  } while (0)

// A kernel's host preparation failed: a stated reason means the kernel cannot
// run this graph; otherwise a CUDA error (out of memory included).
oj_status prep_fail(oj_ctx* ctx, cudaError_t e, const std::string& why) {
  if (!why.empty()) {
    ctx->last_error = why;
    return OJ_ERR_UNSUPPORTED;
  }
  return cuda_fail(ctx, e, "kernel preparation");
}

oj_status arg_fail(oj_ctx* ctx, const char* msg) {
  if (ctx) ctx->last_error = msg;
  return OJ_ERR_ARG;
}

// Expands (param_k, mcs_k) into one entry per sweep, as Algorithm::run does
// (include/openjij/algorithm/algorithm.hpp:47-54).
template <class T>
oj_status expand(oj_ctx* ctx, const T* params, const int32_t* mcs, int32_t num_sched, std::vector<T>& out) {
  out.clear();
  for (int32_t k = 0; k < num_sched; ++k) {
    if (mcs[k] < 0) return arg_fail(ctx, "one_mc_step must be non-negative");
    for (int32_t m = 0; m < mcs[k]; ++m) out.push_back(params[k]);
  }
  return OJ_OK;
}

oj_status rng_base(oj_ctx* ctx, uint64_t seed, int64_t first_sweep, int64_t replica_offset, RngBase* rb) {
  if (first_sweep < 0 || first_sweep > 0xFFFFFFFFll) return arg_fail(ctx, "first_sweep out of range");
  if (replica_offset < 0 || replica_offset > 0xFFFFFFFFll || (replica_offset & 31) != 0)
    return arg_fail(ctx, "replica_offset must be a non-negative multiple of 32");
  rb->k0 = (uint32_t)seed;
  rb->k1 = (uint32_t)(seed >> 32);
  rb->sweep0 = (uint32_t)first_sweep;
  rb->rep0 = (uint32_t)replica_offset;
  return OJ_OK;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Thresholds of the bit-packed kernel: thr[k][m] = floor(exp(-beta_k*2c*m)*2^32),
// m = 1..D (dE = 2c*m); always[k] bit m when the probability is 1.
void msc_thresholds(const std::vector<float>& betas, double c, int D, std::vector<uint32_t>& thr,
                    std::vector<uint32_t>& always) {
  const size_t S = betas.size();
  thr.assign(S * (D + 1), 0u);
  always.assign(S, 0u);
  for (size_t k = 0; k < S; ++k)
    for (int m = 1; m <= D; ++m) {
      const double p = std::exp(-(double)betas[k] * 2.0 * c * (double)m);
      const double t = std::floor(std::ldexp(p, 32));
      uint32_t v;
      if (p >= 1.0) {
        always[k] |= 1u << m;
        v = 0xFFFFFFFFu;
      } else {
        v = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
      }
      thr[k * (D + 1) + m] = v;
    }
}

// Thresholds of the bit-packed SQA kernel, class m = u*3 + k (u unsatisfied
// spatial bonds of D, k aligned Trotter neighbours):
//   dE = a*float(2c(D-2u)) + B*float(4-4k) in FP32 (each product and the sum rounded once);
//   dE <= 0 -> always (mode[2s] bit m); NaN or exp(-dE) == 0 -> never;
//   else thr[s][m] = min(2^32-1, floor(exp(-dE)*2^32)) and mode[2s+1] bit m.
void sqa_msc_thresholds(const std::vector<float2>& coef, double c, int D, std::vector<uint32_t>& thr,
                        std::vector<uint32_t>& mode) {
  const int NC = (D + 1) * 3;
  const size_t S = coef.size();
  thr.assign(S * NC, 0u);
  mode.assign(S * 2, 0u);
  for (size_t k = 0; k < S; ++k) {
    uint32_t always = 0, live = 0;
    for (int u = 0; u <= D; ++u)
      for (int kk = 0; kk < 3; ++kk) {
        const int m = u * 3 + kk;
        const float dEsp = (float)(2.0 * c * (double)(D - 2 * u));
        const float dEtrot = (float)(4 - 4 * kk);
        const float p1 = coef[k].x * dEsp;
        const float p2 = coef[k].y * dEtrot;
        const float dE = p1 + p2;
        uint32_t v = 0;
        if (std::isnan(dE)) {
          v = 0;
        } else if (dE <= 0.0f) {
          always |= 1u << m;
        } else {
          const double t = std::floor(std::ldexp(std::exp(-(double)dE), 32));
          v = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
          if (v) live |= 1u << m;
        }
        thr[k * NC + m] = v;
      }
    mode[2 * k] = always;
    mode[2 * k + 1] = live;
  }
}

oj_status build_batch(oj_ctx* ctx, int32_t count, const int32_t* n, const int64_t* offset, const double* J_aug,
                      oj_batch** out, bool checked = false);

// The graph's augmented matrix as a one-instance batch: FP32 padded rows for
// the dense jump kernel and the FP64 matrix for the replica-parallel energies.
oj_status ensure_single(oj_ctx* ctx, oj_graph* g) {
  if (g->single) return OJ_OK;
  const int n = g->n;
  const int64_t n1 = (int64_t)n + 1;
  std::vector<double> A;
  try {
    A.assign((size_t)(n1 * n1), 0.0);
  } catch (...) {
    return OJ_ERR_OOM;
  }
  for (int64_t i = 0; i < n1; ++i)
    for (int64_t q = g->aug_indptr[i]; q < g->aug_indptr[i + 1]; ++q)
      A[(size_t)(i * n1 + g->aug_indices[q])] = g->aug_data[q];
  const int32_t nn = n;
  const int64_t off = 0;
  oj_batch* b1 = nullptr;
  if (oj_status bs = build_batch(ctx, 1, &nn, &off, A.data(), &b1, true)) return bs;  // the graph is validated
  g->single.reset(b1);
  return OJ_OK;
}

// FP64 energies of R replicas of a dense graph with the batched energy kernel
// (the coupling matrix is read once per 32 replicas).
cudaError_t single_energy(oj_ctx* ctx, oj_graph* g, int R, const int8_t* spins, double* out, cudaStream_t st) {
  struct Tab {
    int32_t reads, order;
    int64_t soff, eoff;
  } h{R, 0, 0, 0};
  cudaError_t e = g->single_tab.ensure(sizeof(Tab));
  if (e != cudaSuccess) return e;
  Tab* d = g->single_tab.as<Tab>();
  if ((e = cudaMemcpyAsync(d, &h, sizeof(Tab), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  const int ns = batch_energy_splits(g->single.get(), R, ctx->sm_count);
  if (ns > 1 && (e = ctx->eparts.ensure((size_t)ns * R * 8)) != cudaSuccess) return e;
  return launch_batch_energy(g->single.get(), &d->reads, &d->soff, &d->eoff, &d->order, R, spins, out, st, ns,
                             ctx->eparts.as<double>(), R);
}

// Device counters of a run, zeroed on the stream before its launches:
// [0] accepted flips (u64), [8] largest field drift (float bits), [12] status
// of the bounded device waits.  The main annealing launch gets rb with the
// flip counter when statistics are asked for (tuning launches never do).
oj_status arm_counters(oj_ctx* ctx, oj_run_stats* stats, RngBase* rb) {
  cudaError_t e = ctx->counters.ensure(32);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->counters.ptr, 0, 32, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "run counters");
  if (stats) rb->flips = ctx->counters.as<unsigned long long>();
  return OJ_OK;
}

struct RunCounters {
  double flips = -1.0;
  float drift = -1.0f;
  int status = 0;
};

// The counters after the stream has drained.
RunCounters read_counters(oj_ctx* ctx) {
  RunCounters rc;
  unsigned char buf[16];
  if (cudaMemcpyAsync(buf, ctx->counters.ptr, 16, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    return rc;
  }
  unsigned long long f;
  std::memcpy(&f, buf, 8);
  std::memcpy(&rc.drift, buf + 8, 4);
  std::memcpy(&rc.status, buf + 12, 4);
  rc.flips = (double)f;
  return rc;
}

// Work items of the tensor-core field kernel for a batch call, uploaded to the
// context; drift and status go to the run counters (armed before).
oj_status field_call(oj_ctx* ctx, const oj_batch* b, const int32_t* reads, const std::vector<int>& order,
                     int max_reads, FieldCall* fc) {
  fc->NT = field_tc_tile_replicas(b, max_reads);
  std::vector<int32_t> it, hot;
  field_tc_items(b, reads, order, fc->NT, it);
  fc->nitems = (int)(it.size() / 3);
  if (hot_tc_applies(b)) hot_tc_items(b, reads, order, hot);
  fc->hot_nitems = (int)(hot.size() / 2);
  const size_t nf = it.size();
  it.insert(it.end(), hot.begin(), hot.end());  // field items, then hot-sweep items
  cudaError_t e = ctx->fitems.ensure(std::max<size_t>(it.size() * 4, 16));
  if (e == cudaSuccess && !it.empty())
    e = cudaMemcpyAsync(ctx->fitems.ptr, it.data(), it.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "field items");
  fc->items = ctx->fitems.as<int32_t>();
  fc->hot_items = fc->items + nf;
  fc->nrep = 0;
  for (int m = 0; m < b->count; ++m) fc->nrep += (size_t)reads[m];
  if (fc->hot_nitems > 0) {
    e = ctx->kstart.ensure(std::max<size_t>(fc->nrep * 4, 16));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "hot-sweep table");
    fc->kstart = ctx->kstart.as<int32_t>();
  }
  char* cb = ctx->counters.as<char>();
  fc->drift = reinterpret_cast<unsigned int*>(cb + 8);
  fc->status = reinterpret_cast<int*>(cb + 12);
  fc->wait_limit = ctx->wait_limit;
  return OJ_OK;
}

// Sweep-kernel arguments of a batched run besides the sweep range.
struct SweepPlan {
  const oj_batch* b;
  const int32_t* d_reads;
  const int64_t* d_soff;
  const int32_t* d_items;
  int nitems;
  int* d_counter;
  int8_t* spins;
  const float* d_betas;  // one per sweep
  uint32_t inst0;
  int variant;
  float* d_fields;
  const int64_t* d_foff;
  double* d_energies;
  const int64_t* d_eoff;
};

// A batched (or dense-jump) run of S sweeps: the fields of the initial spins on
// the tensor cores, then the sweeps.  When the batch's FP32 field sums are not
// exact, the run is cut at every multiple of ctx->recompute global sweeps and
// the fields are computed anew there from the spins (the same cut points for a
// run split over calls at such multiples); with `measure`, the sweep kernel
// stores its incremental fields before each recompute and after the last
// sweep, and the field kernel records their largest deviation (the drift).
cudaError_t run_batch_enqueue(oj_ctx* ctx, cudaStream_t st, const SweepPlan& p, int64_t S, RngBase rb,
                              const FieldCall& fc, bool measure, int* launches) {
  const bool exact = p.b->exact_fields;
  const bool wf = measure && !exact;
  cudaError_t e = launch_field_tc(p.b, p.d_reads, p.d_soff, p.spins, p.d_fields, p.d_foff, fc.items, fc.nitems, fc.NT,
                                  false, fc.drift, fc.status, fc.wait_limit, st);
  if (e != cudaSuccess) return e;
  ++*launches;
  const int64_t K = exact ? 0 : ctx->recompute;
  // exact one-digit batches: the flip-heavy first sweeps on the tensor cores;
  // each replica tile continues in the sweep kernel at the sweep it stopped at
  const int32_t* kstart = nullptr;
  if (exact && fc.hot_nitems > 0 && S > 0) {
    e = cudaMemsetAsync(fc.kstart, 0, fc.nrep * 4, st);
    if (e != cudaSuccess) return e;
    e = launch_hot_tc(p.b, p.d_reads, p.d_soff, p.spins, p.d_fields, p.d_foff, p.d_eoff, fc.hot_items,
                      fc.hot_nitems, p.d_betas, S, rb, p.inst0, fc.kstart, fc.status, fc.wait_limit, st);
    if (e != cudaSuccess) return e;
    ++*launches;
    kstart = fc.kstart;
  }
  if (K > 0 && p.b->max_n <= 128 && p.b->d_q32.ptr) {
    // one-chunk instances: the sweep kernel sets the fields anew itself at the
    // same global sweeps (and checks the drift after the last one), in one launch
    return launch_batch_sweeps(p.b, p.d_reads, p.d_soff, p.d_items, p.nitems, p.d_counter, p.spins, p.d_betas, S, rb,
                               p.inst0, ctx->sm_count, st, launches, p.variant, p.d_fields, p.d_foff, p.d_energies,
                               p.d_eoff, wf, fc.status, fc.wait_limit, nullptr, (int)K, wf ? fc.drift : nullptr);
  }
  int64_t k = 0;
  while (k < S) {
    const uint64_t g = (uint64_t)rb.sweep0 + (uint64_t)k;
    int64_t len = S - k;
    if (K > 0) len = std::min<int64_t>(len, K - (int64_t)(g % (uint64_t)K));
    RngBase rs = rb;
    rs.sweep0 = (uint32_t)g;
    e = launch_batch_sweeps(p.b, p.d_reads, p.d_soff, p.d_items, p.nitems, p.d_counter, p.spins, p.d_betas + k, len,
                            rs, p.inst0, ctx->sm_count, st, launches, p.variant, p.d_fields, p.d_foff, p.d_energies,
                            p.d_eoff, wf, fc.status, fc.wait_limit, kstart);
    if (e != cudaSuccess) return e;
    k += len;
    if (k < S || wf) {
      e = launch_field_tc(p.b, p.d_reads, p.d_soff, p.spins, p.d_fields, p.d_foff, fc.items, fc.nitems, fc.NT, wf,
                          fc.drift, fc.status, fc.wait_limit, st);
      if (e != cudaSuccess) return e;
      ++*launches;
    }
  }
  return cudaSuccess;
}

// A batched / dense-jump run as one CUDA graph: the launches are captured on
// the context's graph stream (after the work already queued on its stream),
// the kept executable graph is updated to the capture (or instantiated anew
// when the launch sequence changed), replayed, and the context's stream waits
// for it.  OJ_GRAPH=0 in the environment enqueues the launches directly.  A
// capture that fails is not retried as direct launches: the error is the
// run's.
cudaError_t run_batch(oj_ctx* ctx, const SweepPlan& p, int64_t S, RngBase rb, const FieldCall& fc, bool measure,
                      int* launches) {
  const char* env = std::getenv("OJ_GRAPH");
  if (env && env[0] == '0') return run_batch_enqueue(ctx, ctx->stream, p, S, rb, fc, measure, launches);
  cudaError_t e = cudaSuccess;
  if (!ctx->gstream && (e = cudaStreamCreateWithFlags(&ctx->gstream, cudaStreamNonBlocking)) != cudaSuccess)
    return e;
  for (auto& ev : ctx->gev)
    if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
  const cudaStream_t gs = ctx->gstream;
  if ((e = cudaEventRecord(ctx->gev[0], ctx->stream)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(gs, ctx->gev[0], 0)) != cudaSuccess)
    return e;
  if ((e = cudaStreamBeginCapture(gs, cudaStreamCaptureModeRelaxed)) != cudaSuccess) return e;
  int nl = 0;
  const cudaError_t re = run_batch_enqueue(ctx, gs, p, S, rb, fc, measure, &nl);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(gs, &graph);
  if (re != cudaSuccess || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return re != cudaSuccess ? re : ce;
  }
  if (ctx->gexec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(ctx->gexec, graph, &info) != cudaSuccess) {
      cudaGetLastError();  // another launch sequence: instantiate anew
      cudaGraphExecDestroy(ctx->gexec);
      ctx->gexec = nullptr;
    }
  }
  if (!ctx->gexec) e = cudaGraphInstantiate(&ctx->gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    ctx->gexec = nullptr;
    return e;
  }
  if ((e = cudaGraphLaunch(ctx->gexec, gs)) != cudaSuccess) return e;
  if ((e = cudaEventRecord(ctx->gev[1], gs)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(ctx->stream, ctx->gev[1], 0)) != cudaSuccess)
    return e;
  *launches += nl;
  return cudaSuccess;
}

// OJ_AUTOTUNE=1 in the environment tunes every call's first use of a shape,
// OJ_AUTOTUNE=0 none (not even on request: fixed shapes for profiling).
bool autotune_requested(uint32_t flags) {
  const char* e = std::getenv("OJ_AUTOTUNE");
  if (e && e[0] == '0') return false;
  return (flags & OJ_AUTOTUNE) || (e && e[0] == '1');
}

// Autotuner core: for each candidate, restore() puts the call's own initial
// state into a scratch copy and enqueue(i) runs candidate i on it for a few
// sweeps; each candidate runs twice and the faster run counts.  Returns the
// fastest candidate (the default one, def, unless another is 3 % faster),
// -1 when none launched, or -2 on a device error (which the caller reports).
// Candidates that cannot launch (cluster or shared-memory limits) are skipped.
template <class Restore, class Enqueue>
int time_candidates(cudaStream_t st, int count, Restore restore, Enqueue enqueue, cudaError_t* err, int def = -1) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if ((*err = cudaEventCreate(&e0)) != cudaSuccess) return -2;
  if ((*err = cudaEventCreate(&e1)) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -2;
  }
  float best = 0.0f, def_ms = -1.0f;
  int bi = -1;
  for (int i = 0; i < count && *err == cudaSuccess; ++i) {
    float ms = 0.0f;
    bool ok = true;
    for (int rep = 0; rep < 2 && ok; ++rep) {
      if ((*err = restore()) != cudaSuccess) break;
      cudaEventRecord(e0, st);
      const cudaError_t le = enqueue(i);
      cudaEventRecord(e1, st);
      if (le != cudaSuccess) {
        cudaGetLastError();  // launch-configuration errors are not sticky
        ok = false;
        break;
      }
      if ((*err = cudaStreamSynchronize(st)) != cudaSuccess) break;
      float t = 0.0f;
      cudaEventElapsedTime(&t, e0, e1);
      ms = rep == 0 ? t : std::min(ms, t);
    }
    if (*err != cudaSuccess) break;
    if (ok && i == def) def_ms = ms;
    if (ok && (bi < 0 || ms < best)) {
      best = ms;
      bi = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (*err != cudaSuccess) return -2;
  // the default shape stays unless another is clearly (3 %) faster: short
  // timings of a few sweeps carry that much noise
  if (def_ms > 0.0f && best > 0.97f * def_ms) return def;
  return bi;
}

}  // namespace

extern "C" {

const char* oj_version(void) { return kVersion; }

const char* oj_status_string(oj_status s) {
  switch (s) {
    case OJ_OK: return "ok";
    case OJ_ERR_ARG: return "invalid argument";
    case OJ_ERR_OOM: return "out of memory";
    case OJ_ERR_CUDA: return "CUDA error";
    case OJ_ERR_TIMEOUT: return "device wait timed out";
    case OJ_ERR_BOUNDS: return "device bounds check failed";
    case OJ_ERR_UNSUPPORTED: return "unsupported by the selected kernel";
    case OJ_ERR_NODEVICE: return "no usable CUDA device";
    default: return "unknown status";
  }
}

oj_status oj_ctx_create(int32_t device, oj_ctx** out) {
  if (!out) return OJ_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return OJ_ERR_NODEVICE;
  }
  if (device < 0 || device >= count) return OJ_ERR_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return OJ_ERR_CUDA;
  if (prop.major < 10) return OJ_ERR_NODEVICE;  // the kernels are built for sm_100a only
  oj_ctx* ctx = new (std::nothrow) oj_ctx();
  if (!ctx) return OJ_ERR_OOM;
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  DeviceGuard dg(device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return OJ_ERR_CUDA;
  }
  ctx->own_stream = true;
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  // set-up of oj_sa_run_bitpacked_noalloc on this device, so that its calls
  // allocate nothing; a failure only disables that entry point
  const cudaError_t pe = noalloc_prepare(device);
  if (pe != cudaSuccess) {
    cudaGetLastError();
    ctx->noalloc_error = std::string("set-up of the allocation-free entry point failed: ") + cudaGetErrorString(pe);
  }
  host_pin_device(device);
  *out = ctx;
  return OJ_OK;
}

oj_status oj_ctx_destroy(oj_ctx* ctx) {
  if (!ctx) return OJ_OK;
  {
    DeviceGuard dg(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->spins.release();
    ctx->words.release();
    ctx->params.release();
    ctx->energies.release();
    ctx->best.release();
    ctx->aux.release();
    ctx->batch.release();
    ctx->fields.release();
    ctx->eparts.release();
    ctx->counters.release();
    for (auto& e : ctx->ev)
      if (e) cudaEventDestroy(e);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    for (auto& e : ctx->gev)
      if (e) cudaEventDestroy(e);
    for (auto& e : ctx->pev)
      if (e) cudaEventDestroy(e);
    if (ctx->gstream) cudaStreamDestroy(ctx->gstream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return OJ_OK;
}

oj_status oj_ctx_set_stream(oj_ctx* ctx, void* stream) {
  if (!ctx) return OJ_ERR_ARG;
  DeviceGuard dg(ctx->device);
  if (ctx->own_stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  ctx->stream = static_cast<cudaStream_t>(stream);
  ctx->own_stream = false;
  return OJ_OK;
}

oj_status oj_ctx_synchronize(oj_ctx* ctx) {
  if (!ctx) return OJ_ERR_ARG;
  DeviceGuard dg(ctx->device);
  OJ_CK(cudaStreamSynchronize(ctx->stream), "synchronize");
  return OJ_OK;
}

const char* oj_ctx_last_error(const oj_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

oj_status oj_ctx_set_field_recompute(oj_ctx* ctx, int32_t sweeps) {
  if (!ctx || sweeps < 0) return arg_fail(ctx, "the recompute interval must be >= 0");
  ctx->recompute = sweeps;
  return OJ_OK;
}

oj_status oj_ctx_inject_fault(oj_ctx* ctx, int32_t kind, int64_t after) {
  if (!ctx) return OJ_ERR_ARG;
  if (kind == OJ_FAULT_NONE) {
    alloc_fail_countdown().store(-1);
    return OJ_OK;
  }
  if (kind != OJ_FAULT_ALLOC || after < 0) return arg_fail(ctx, "unknown fault kind or negative count");
  alloc_fail_countdown().store((long long)after);
  return OJ_OK;
}

oj_status oj_ctx_set_wait_limit(oj_ctx* ctx, int64_t iterations) {
  if (!ctx) return OJ_ERR_ARG;
  ctx->wait_limit = iterations < 0 ? -1 : (long long)iterations;
  return OJ_OK;
}

oj_status oj_graph_create_csr(oj_ctx* ctx, int32_t n, const int64_t* indptr, const int32_t* indices,
                              const double* data, oj_graph** out) {
  if (!ctx || !out || n < 0 || !indptr) return arg_fail(ctx, "null argument or negative size");
  *out = nullptr;
  if (indptr[0] != 0 || indptr[n + 1] < indptr[0]) return arg_fail(ctx, "invalid indptr");
  const int64_t nnz = indptr[n + 1];
  if (nnz > 0 && (!indices || !data)) return arg_fail(ctx, "null indices/data");
  DeviceGuard dg(ctx->device);
  oj_graph* g = new (std::nothrow) oj_graph();
  if (!g) return OJ_ERR_OOM;
  g->device = ctx->device;
  g->n = n;
  try {
    g->aug_indptr.assign(indptr, indptr + n + 2);
    g->aug_indices.assign(indices, indices + nnz);
    g->aug_data.assign(data, data + nnz);
  } catch (...) {
    delete g;
    return OJ_ERR_OOM;
  }
  for (int i = 0; i <= n; ++i)
    if (indptr[i + 1] < indptr[i]) {
      delete g;
      return arg_fail(ctx, "indptr must be non-decreasing");
    }
  oj_status s;
  try {
    s = finish_graph(ctx, g);
  } catch (...) {
    s = OJ_ERR_OOM;
  }
  if (s != OJ_OK) {
    delete g;
    return s;
  }
  *out = g;
  return OJ_OK;
}

oj_status oj_graph_create_dense(oj_ctx* ctx, int32_t n, const double* J, oj_graph** out) {
  if (!ctx || !out || n < 0 || !J) return arg_fail(ctx, "null argument or negative size");
  const int64_t n1 = (int64_t)n + 1;
  std::vector<int64_t> ip;
  std::vector<int32_t> ix;
  std::vector<double> dv;
  try {
    ip.reserve(n1 + 1);
    ip.push_back(0);
    for (int64_t i = 0; i < n1; ++i) {
      for (int64_t j = 0; j < n1; ++j) {
        const double v = J[i * n1 + j];
        if (v != 0.0 || i == j) {
          ix.push_back((int32_t)j);
          dv.push_back(v);
        }
      }
      ip.push_back((int64_t)ix.size());
    }
  } catch (...) {
    return OJ_ERR_OOM;
  }
  return oj_graph_create_csr(ctx, n, ip.data(), ix.data(), dv.data(), out);
}

oj_status oj_graph_destroy(oj_graph* g) {
  delete g;
  return OJ_OK;
}

oj_status oj_graph_query(const oj_graph* g, oj_graph_info* out) {
  if (!g || !out) return OJ_ERR_ARG;
  *out = g->info;
  return OJ_OK;
}

// FP64 energies of a graph's spin vectors, the sites split over enough CTAs to
// cover the SMs (partial sums in the context's buffer, added in order).
cudaError_t graph_energy(oj_ctx* ctx, const oj_graph* g, int count, const int8_t* d_spins, double* d_e,
                         cudaStream_t st, int* launches) {
  const int ns = energy_splits(g, count, ctx->sm_count);
  if (ns > 1) {
    const cudaError_t e = ctx->eparts.ensure((size_t)ns * count * 8);
    if (e != cudaSuccess) return e;
  }
  if (launches) *launches += ns > 1 ? 2 : 1;
  return launch_energy(g, count, d_spins, d_e, st, ns, ns > 1 ? ctx->eparts.as<double>() : nullptr);
}

oj_status oj_sa_run(oj_ctx* ctx, const oj_graph* gc, int32_t R, int8_t* spins, const double* betas,
                    const int32_t* mcs, int32_t num_sched, uint64_t seed, int64_t first_sweep,
                    int64_t replica_offset, uint32_t flags, double* energies, oj_run_stats* stats) {
  if (!ctx || !gc || R < 0 || num_sched < 0) return arg_fail(ctx, "null argument or negative size");
  if (num_sched > 0 && (!betas || !mcs)) return arg_fail(ctx, "null schedule");
  oj_graph* g = const_cast<oj_graph*>(gc);
  if (g->device != ctx->device) return arg_fail(ctx, "graph belongs to another device");
  const int n = g->n;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (R == 0 || n == 0) return OJ_OK;
  if (!spins) return arg_fail(ctx, "null spins");
  for (int32_t k = 0; k < num_sched; ++k)
    if (!(betas[k] >= 0.0) || std::isinf(betas[k])) return arg_fail(ctx, "beta must be finite and >= 0");
  RngBase rb;
  if (oj_status s = rng_base(ctx, seed, first_sweep, replica_offset, &rb)) return s;
  DeviceGuard dg(ctx->device);
  std::vector<double> bexp;
  if (oj_status s = expand(ctx, betas, mcs, num_sched, bexp)) return s;
  const int64_t S = (int64_t)bexp.size();
  std::vector<float> bf(bexp.begin(), bexp.end());
  const bool devp = (flags & OJ_DEVICE_POINTERS) != 0;
  uint32_t kernel = flags & OJ_KERNEL_MASK;
  const oj_graph_info& inf = g->info;
  if (kernel == OJ_KERNEL_AUTO) {
    if (inf.bimodal && g->regular && inf.max_degree <= msc_max_degree() && inf.max_degree >= 1) {
      kernel = OJ_KERNEL_BITPACKED;
    } else if (inf.num_colours > 64 && (int64_t)n * n * 4 <= ((int64_t)8 << 30)) {
      // dense: one warp per replica jumping between accepted flips (fastest
      // measured on dense QUBOs) up to its size limit, else the plain kernel
      kernel = n <= batch_max_sites() ? OJ_KERNEL_DENSE_JUMP : OJ_KERNEL_DENSE_PLAIN;
    } else {
      kernel = OJ_KERNEL_COLOUR;
    }
  }
  if (kernel == OJ_KERNEL_BITPACKED &&
      !(inf.bimodal && g->regular && inf.max_degree <= msc_max_degree() && inf.max_degree >= 1)) {
    ctx->last_error = "bit-packed kernel needs a regular graph with couplings +-c (degree <= 8) and h = 0";
    return OJ_ERR_UNSUPPORTED;
  }
  if (kernel > OJ_KERNEL_DENSE_JUMP) return arg_fail(ctx, "unknown kernel");
  if (kernel == OJ_KERNEL_DENSE_JUMP && n > batch_max_sites()) {
    ctx->last_error = "dense jump kernel supports n <= 4096";
    return OJ_ERR_UNSUPPORTED;
  }
  if (kernel == OJ_KERNEL_DENSE_TC) {
    std::string why;
    cudaError_t pe = dense_tc_prepare(g, &why);
    if (pe != cudaSuccess) {
      return prep_fail(ctx, pe, why);
    }
  }
  cudaStream_t st = ctx->stream;
  const size_t spin_bytes = (size_t)R * n;
  int8_t* d_spins = spins;
  if (!devp) {
    OJ_CK(ctx->spins.ensure(spin_bytes), "alloc spins");
    d_spins = ctx->spins.as<int8_t>();
  } else if (!is_device_ptr(spins)) {
    return arg_fail(ctx, "OJ_DEVICE_POINTERS set but spins is not device memory");
  }
  int launches = 0;
  int P_used = 0, threads_used = 0, variant_used = 0;
  bool tuned_now = false;
  bool energies_in_kernel = false;  // the dense jump kernel wrote them (exact fields)
  RngBase rbm = rb;                 // rb of the main annealing launch (counts accepted flips)
  if (oj_status cs = arm_counters(ctx, stats, &rbm)) return cs;
  bool field_run = false;           // the tensor-core field kernel ran (drift and status to read)
  OJ_CK(cudaEventRecord(ctx->ev[0], st), "event");
  if (!devp) OJ_CK(cudaMemcpyAsync(d_spins, spins, spin_bytes, cudaMemcpyHostToDevice, st), "H2D spins");
  if (kernel == OJ_KERNEL_BITPACKED) {
    const int D = inf.max_degree;
    const int G = (R + 31) / 32;
    std::string why;
    // the cached shape's cluster when there is one, so the plan is built once
    const uint64_t key = ((uint64_t)OJ_KERNEL_BITPACKED << 40) | (uint64_t)R;
    const auto cached = g->tuned.find(key);
    const int P = (cached != g->tuned.end() && cached->second.cluster) ? cached->second.cluster
                                                                       : msc_choose_cluster(g, G, ctx->sm_count);
    cudaError_t pe = msc_prepare(g, P, &why);
    if (pe != cudaSuccess) {
      return prep_fail(ctx, pe, why);
    }
    std::vector<uint32_t> thr, alw;
    msc_thresholds(bf, inf.coupling_abs, D, thr, alw);
    const size_t pbytes = (thr.size() + alw.size()) * 4;
    OJ_CK(ctx->params.ensure(std::max<size_t>(pbytes, 16)), "alloc params");
    uint32_t* d_thr = ctx->params.as<uint32_t>();
    uint32_t* d_alw = d_thr + thr.size();
    if (S > 0) {
      OJ_CK(cudaMemcpyAsync(d_thr, thr.data(), thr.size() * 4, cudaMemcpyHostToDevice, st), "H2D thr");
      OJ_CK(cudaMemcpyAsync(d_alw, alw.data(), alw.size() * 4, cudaMemcpyHostToDevice, st), "H2D always");
    }
    OJ_CK(ctx->words.ensure((size_t)G * n * 4), "alloc words");
    uint32_t* d_words = ctx->words.as<uint32_t>();
    OJ_CK(launch_pack(d_spins, R, n, d_words, st), "pack");
    ++launches;
    // launch shape: cached, autotuned now, or the default heuristic
    Shape shp;
    auto it = g->tuned.find(key);
    if (it != g->tuned.end()) {
      shp = it->second;
    } else if (autotune_requested(flags) && S > 0) {
      std::vector<Shape> cand;
      for (int Pc : {1, 2, 4, 8, 16})
        if (Pc == 1 || n / Pc >= 64)
          for (int th : {256, 512, 1024}) cand.push_back(Shape{Pc, th, 0});
      int def_msc = -1;  // the heuristic shape
      for (size_t q = 0; q < cand.size(); ++q)
        if (cand[q].cluster == msc_choose_cluster(g, G, ctx->sm_count) && cand[q].threads == msc_default_threads())
          def_msc = (int)q;
      OJ_CK(ctx->aux.ensure((size_t)G * n * 4), "alloc tuning scratch");
      uint32_t* scratch = ctx->aux.as<uint32_t>();
      const int64_t Ssub = std::min<int64_t>(S, 16);
      cudaError_t terr = cudaSuccess;
      const int bi = time_candidates(
          st, (int)cand.size(),
          [&] { return cudaMemcpyAsync(scratch, d_words, (size_t)G * n * 4, cudaMemcpyDeviceToDevice, st); },
          [&](int i) {
            std::string w;
            const cudaError_t e = msc_prepare(g, cand[i].cluster, &w);
            if (e != cudaSuccess) return e;
            return launch_sa_msc(g, G, scratch, d_thr, d_alw, Ssub, rb, st, nullptr, cand[i].threads);
          },
          &terr, def_msc);
      if (bi == -2) return cuda_fail(ctx, terr, "autotune");
      if (bi >= 0) shp = cand[bi];
      g->tuned[key] = shp;
      tuned_now = true;
    }
    P_used = shp.cluster ? shp.cluster : msc_choose_cluster(g, G, ctx->sm_count);
    threads_used = shp.threads ? shp.threads : msc_default_threads();
    pe = msc_prepare(g, P_used, &why);
    if (pe != cudaSuccess) {
      return prep_fail(ctx, pe, why);
    }
    OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
    if (S > 0)
      OJ_CK(launch_sa_msc(g, G, d_words, d_thr, d_alw, S, rbm, st, &launches, threads_used), "sa bit-packed kernel");
    OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
    OJ_CK(launch_unpack(d_words, R, n, d_spins, st), "unpack");
    ++launches;
  } else if (kernel == OJ_KERNEL_DENSE_JUMP) {
    if (oj_status bs = ensure_single(ctx, g)) return bs;
    auto make_items = [&](int W) {
      std::vector<int32_t> it;
      for (int gq = 0; gq * W < R; ++gq) {
        it.push_back(0);
        it.push_back(gq);
      }
      return it;
    };
    const uint64_t key = ((uint64_t)OJ_KERNEL_DENSE_JUMP << 40) | (uint64_t)R;
    auto tit = g->tuned.find(key);
    int variant = tit != g->tuned.end() ? tit->second.variant : batch_default_variant();
    if (n > batch_variant_max_n(variant)) variant = 83;
    std::vector<int32_t> items = make_items(batch_variant_warps(variant));
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t b_hdr = al(8 + 8 + 8), b_items = al(make_items(batch_min_warps()).size() * 4 + 4), b_cnt = al(4),
                 b_beta = al(bf.size() * 4 + 4);
    OJ_CK(ctx->batch.ensure(b_hdr + b_items + b_cnt + b_beta), "alloc tables");
    char* base = ctx->batch.as<char>();
    int32_t* d_reads = reinterpret_cast<int32_t*>(base);
    int64_t* d_soff = reinterpret_cast<int64_t*>(base + 8);
    int64_t* d_foff = reinterpret_cast<int64_t*>(base + 16);
    int32_t* d_items = reinterpret_cast<int32_t*>(base + b_hdr);
    int* d_counter = reinterpret_cast<int*>(base + b_hdr + b_items);
    float* d_beta = reinterpret_cast<float*>(base + b_hdr + b_items + b_cnt);
    const int32_t hreads = R;
    const int64_t hsoff = 0;
    OJ_CK(cudaMemcpyAsync(d_reads, &hreads, 4, cudaMemcpyHostToDevice, st), "H2D reads");
    OJ_CK(cudaMemcpyAsync(d_soff, &hsoff, 8, cudaMemcpyHostToDevice, st), "H2D offsets");
    OJ_CK(cudaMemcpyAsync(d_foff, &hsoff, 8, cudaMemcpyHostToDevice, st), "H2D offsets");
    // initial fields of every replica, [R][n rounded up to 128] floats
    OJ_CK(ctx->fields.ensure(std::max<size_t>((size_t)R * (((size_t)n + 127) / 128 * 128) * 4, 16)), "alloc fields");
    float* d_fields = ctx->fields.as<float>();
    if (S > 0) OJ_CK(cudaMemcpyAsync(d_beta, bf.data(), bf.size() * 4, cudaMemcpyHostToDevice, st), "H2D betas");
    FieldCall fc;
    if (oj_status fs = field_call(ctx, g->single.get(), &hreads, std::vector<int>{0}, R, &fc)) return fs;
    if (tit == g->tuned.end() && autotune_requested(flags) && S > 0) {
      // candidates run 16 sweeps with betas spread over the schedule on a copy of the spins
      std::vector<int> cand;
      for (int v : {45, 82, 83, 84, 162, 321})
        if (n <= batch_variant_max_n(v)) cand.push_back(v);
      const int64_t Ssub = std::min<int64_t>(S, 32);
      std::vector<float> tb(Ssub);
      for (int64_t q = 0; q < Ssub; ++q) tb[q] = bf[(size_t)((q * S) / Ssub)];
      const size_t sb_al = al(spin_bytes);
      OJ_CK(ctx->aux.ensure(sb_al + tb.size() * 4), "alloc tuning scratch");
      int8_t* scratch = ctx->aux.as<int8_t>();
      float* d_tb = reinterpret_cast<float*>(ctx->aux.as<char>() + sb_al);
      OJ_CK(cudaMemcpyAsync(d_tb, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice, st), "H2D tuning betas");
      cudaError_t terr = cudaSuccess;
      std::vector<int32_t> it;
      int loaded = -1;
      const int bi = time_candidates(
          st, (int)cand.size(),
          [&] { return cudaMemcpyAsync(scratch, d_spins, spin_bytes, cudaMemcpyDeviceToDevice, st); },
          [&](int i) {
            if (loaded != i) {
              it = make_items(batch_variant_warps(cand[i]));
              if (it.size() * 4 > b_items) return cudaErrorInvalidValue;  // never past the table
              const cudaError_t e = cudaMemcpyAsync(d_items, it.data(), it.size() * 4, cudaMemcpyHostToDevice, st);
              if (e != cudaSuccess) return e;
              loaded = i;
            }
            return launch_sa_batch(g->single.get(), d_reads, d_soff, d_items, (int)(it.size() / 2), d_counter,
                                   scratch, d_tb, Ssub, rb, 0, ctx->sm_count, st, nullptr, cand[i], d_fields, d_foff,
                                   fc);
          },
          &terr, (int)(std::find(cand.begin(), cand.end(), variant) - cand.begin()));
      if (bi == -2) return cuda_fail(ctx, terr, "autotune");
      variant = bi >= 0 ? cand[bi] : 83;
      g->tuned[key] = Shape{0, 0, variant};
      tuned_now = true;
      items = make_items(batch_variant_warps(variant));
    }
    OJ_CK(cudaMemcpyAsync(d_items, items.data(), items.size() * 4, cudaMemcpyHostToDevice, st), "H2D items");
    // exact FP32 fields: the sweep kernel writes the energies (its eoff table is d_soff, zero)
    double* d_ek = nullptr;
    if (energies && S > 0 && g->single->exact_fields) {
      d_ek = energies;
      if (!devp) {
        OJ_CK(ctx->energies.ensure((size_t)R * 8), "alloc energies");
        d_ek = ctx->energies.as<double>();
      }
      energies_in_kernel = true;
    }
    OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
    if (S > 0) {
      const SweepPlan sp{g->single.get(), d_reads, d_soff, d_items, (int)(items.size() / 2), d_counter, d_spins,
                         d_beta, 0, variant, d_fields, d_foff, d_ek, d_soff};
      OJ_CK(run_batch(ctx, sp, S, rbm, fc, stats != nullptr, &launches), "sa dense jump kernel");
      field_run = true;
    }
    OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
    threads_used = batch_variant_warps(variant) * 32;
    variant_used = variant;
  } else {
    OJ_CK(ctx->params.ensure(std::max<size_t>(bf.size() * 4, 16)), "alloc params");
    float* d_beta = ctx->params.as<float>();
    if (S > 0) OJ_CK(cudaMemcpyAsync(d_beta, bf.data(), bf.size() * 4, cudaMemcpyHostToDevice, st), "H2D betas");
    if (kernel == OJ_KERNEL_DENSE_PLAIN) OJ_CK(ensure_dense(g), "dense J upload");
    OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
    if (S > 0) {
      if (kernel == OJ_KERNEL_DENSE_TC) {
        OJ_CK(cudaMemsetAsync(g->tc->status.ptr, 0, sizeof(int), st), "status reset");
        OJ_CK(launch_sa_dense_tc(g, R, d_spins, d_beta, S, rbm, 16, st, &launches), "sa dense tensor-core kernel");
      } else if (kernel == OJ_KERNEL_DENSE_PLAIN)
        OJ_CK(launch_sa_dense_plain(g, R, d_spins, d_beta, S, rbm, st, &launches), "sa dense kernel");
      else
        OJ_CK(launch_sa_colour(g, R, d_spins, d_beta, S, rbm, st, &launches), "sa colour kernel");
    }
    OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
  }
  if (energies && energies_in_kernel) {
    if (!devp)
      OJ_CK(cudaMemcpyAsync(energies, ctx->energies.as<double>(), (size_t)R * 8, cudaMemcpyDeviceToHost, st),
            "D2H energies");
  } else if (energies) {
    double* d_e = energies;
    if (!devp) {
      OJ_CK(ctx->energies.ensure((size_t)R * 8), "alloc energies");
      d_e = ctx->energies.as<double>();
    }
    const bool dense = kernel == OJ_KERNEL_DENSE_PLAIN || kernel == OJ_KERNEL_DENSE_TC || kernel == OJ_KERNEL_DENSE_JUMP;
    if (dense && n <= batch_max_sites() && ensure_single(ctx, g) == OJ_OK) {
      OJ_CK(single_energy(ctx, g, R, d_spins, d_e, st), "energy kernel");
      if (batch_energy_splits(g->single.get(), R, ctx->sm_count) > 1) ++launches;  // the parts' sum
    } else {
      OJ_CK(graph_energy(ctx, g, R, d_spins, d_e, st, nullptr), "energy kernel");
      if (energy_splits(g, R, ctx->sm_count) > 1) ++launches;  // the parts' sum
    }
    ++launches;
    if (!devp) OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)R * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
  }
  if (!devp) OJ_CK(cudaMemcpyAsync(spins, d_spins, spin_bytes, cudaMemcpyDeviceToHost, st), "D2H spins");
  OJ_CK(cudaEventRecord(ctx->ev[3], st), "event");
  if (!devp || stats || kernel == OJ_KERNEL_DENSE_TC || field_run) OJ_CK(cudaStreamSynchronize(st), "run");
  RunCounters rc;
  if (stats || field_run) rc = read_counters(ctx);
  if (field_run && rc.status) {
    ctx->last_error = "tensor-core field kernel: a bounded device wait ran out";
    return OJ_ERR_TIMEOUT;
  }
  if (kernel == OJ_KERNEL_DENSE_TC && S > 0) {
    int flag = 0;
    OJ_CK(cudaMemcpy(&flag, g->tc->status.ptr, sizeof(int), cudaMemcpyDeviceToHost), "status read");
    if (flag) {
      ctx->last_error = "tensor-core dense kernel: a bounded device wait timed out";
      return OJ_ERR_TIMEOUT;
    }
  }
  if (stats) {
    stats->kernel = (int32_t)(kernel >> OJ_KERNEL_SHIFT);
    stats->launches = launches;
    stats->sweeps = S;
    stats->attempts = (double)R * n * (double)S;
    stats->cluster = P_used;
    stats->threads = threads_used;
    stats->variant = variant_used;
    stats->tuned = tuned_now ? 1 : 0;
    cudaEventElapsedTime(&stats->anneal_ms, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&stats->total_ms, ctx->ev[0], ctx->ev[3]);
    stats->accepted = rc.flips;
    stats->field_drift = !field_run ? -1.0 : (g->single->exact_fields ? 0.0 : (double)rc.drift);
  }
  return OJ_OK;
}

// The second stream and the events of a two-half run (made once).
static cudaError_t pipe_streams(oj_ctx* ctx) {
  cudaError_t e = cudaSuccess;
  if (!ctx->gstream && (e = cudaStreamCreateWithFlags(&ctx->gstream, cudaStreamNonBlocking)) != cudaSuccess)
    return e;
  for (auto& ev : ctx->pev)
    if (!ev && (e = cudaEventCreate(&ev)) != cudaSuccess) return e;
  return cudaSuccess;
}

oj_status oj_sqa_run(oj_ctx* ctx, const oj_graph* gc, int32_t R, int32_t T, int8_t* spins, double gamma,
                     const double* betas, const double* s, const int32_t* mcs, int32_t num_sched,
                     uint64_t seed, int64_t first_sweep, int64_t replica_offset, uint32_t flags,
                     double* energies, int32_t* best_slice, oj_run_stats* stats) {
  if (!ctx || !gc || R < 0 || num_sched < 0) return arg_fail(ctx, "null argument or negative size");
  if (T < 2) return arg_fail(ctx, "trotter slices must be equal or larger than 2.");
  if (num_sched > 0 && (!betas || !s || !mcs)) return arg_fail(ctx, "null schedule");
  oj_graph* g = const_cast<oj_graph*>(gc);
  if (g->device != ctx->device) return arg_fail(ctx, "graph belongs to another device");
  const int n = g->n;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (R == 0 || n == 0) return OJ_OK;
  if (!spins) return arg_fail(ctx, "null spins");
  uint32_t kernel = flags & OJ_KERNEL_MASK;
  const bool split_ok = sqa_split_applies(g, T);
  const bool msc_ok = g->info.bimodal && g->regular && T <= 32 && sqa_msc_fits(g);
  if (kernel == OJ_KERNEL_AUTO) kernel = (split_ok || msc_ok) ? OJ_KERNEL_BITPACKED : OJ_KERNEL_COLOUR;
  if (kernel != OJ_KERNEL_COLOUR && kernel != OJ_KERNEL_BITPACKED) {
    ctx->last_error = "SQA runs on the colour-class or the bit-packed kernel";
    return OJ_ERR_UNSUPPORTED;
  }
  if (kernel == OJ_KERNEL_BITPACKED && !split_ok && !msc_ok) {
    ctx->last_error =
        "bit-packed SQA needs a regular graph with couplings +-c (degree <= 8), h = 0 and an even T <= 64 "
        "(or T <= 32 and n <= 65535)";
    return OJ_ERR_UNSUPPORTED;
  }
  RngBase rb;
  if (oj_status st_ = rng_base(ctx, seed, first_sweep, replica_offset, &rb)) return st_;
  DeviceGuard dg(ctx->device);
  // per-schedule-entry coefficients (single_spin_flip.hpp:147-148, 215-217)
  std::vector<float2> coef_sched(num_sched);
  for (int32_t k = 0; k < num_sched; ++k) {
    const double beta = betas[k], sk = s[k];
    const double a = sk * (beta / (double)(size_t)T);
    const double B = (1 / 2.) * std::log(std::tanh(beta * gamma * (1.0 - sk) / (double)(size_t)T));
    coef_sched[k] = make_float2((float)a, (float)B);
  }
  std::vector<float2> coef;
  if (oj_status st_ = expand(ctx, coef_sched.data(), mcs, num_sched, coef)) return st_;
  const int64_t S = (int64_t)coef.size();
  const bool devp = (flags & OJ_DEVICE_POINTERS) != 0;
  cudaStream_t st = ctx->stream;
  const size_t spin_bytes = (size_t)R * T * n;
  int8_t* d_spins = spins;
  if (!devp) {
    OJ_CK(ctx->spins.ensure(spin_bytes), "alloc spins");
    d_spins = ctx->spins.as<int8_t>();
  } else if (!is_device_ptr(spins)) {
    return arg_fail(ctx, "OJ_DEVICE_POINTERS set but spins is not device memory");
  }
  int launches = 0;
  int P_used = 0, threads_used = 0;
  bool tuned_now = false;
  RngBase rbm = rb;  // rb of the main annealing launch (counts accepted flips)
  if (oj_status cs = arm_counters(ctx, stats, &rbm)) return cs;
  // slice-split runs from host buffers with a known launch shape go in two
  // halves of replica groups on two streams (the copies of one half overlap
  // the other's kernel); OJ_PIPE=0 in the environment runs them whole
  const int Psplit = sqa_split_replicas_per_group(T);
  const uint64_t split_key = ((uint64_t)0x80 << 40) | ((uint64_t)T << 32) | (uint64_t)R;
  const char* pipe_env = std::getenv("OJ_PIPE");
  const bool pipe = !devp && kernel == OJ_KERNEL_BITPACKED && split_ok && S > 0 && R > Psplit &&
                    (g->tuned.count(split_key) > 0 || !autotune_requested(flags)) &&
                    !(pipe_env && pipe_env[0] == '0');
  OJ_CK(cudaEventRecord(ctx->ev[0], st), "event");
  if (!devp && !pipe) OJ_CK(cudaMemcpyAsync(d_spins, spins, spin_bytes, cudaMemcpyHostToDevice, st), "H2D spins");
  if (kernel == OJ_KERNEL_BITPACKED && split_ok) {
    const int P = sqa_split_replicas_per_group(T);
    const int G = (R + P - 1) / P;
    std::string why;
    // the cached shape's cluster when there is one, so the plan is built once
    const uint64_t key = ((uint64_t)0x80 << 40) | ((uint64_t)T << 32) | (uint64_t)R;
    const auto cached = g->tuned.find(key);
    const cudaError_t pe =
        sqa_split_prepare(g, G, ctx->sm_count, &why, cached != g->tuned.end() ? cached->second.cluster : 0);
    if (pe != cudaSuccess) {
      return prep_fail(ctx, pe, why);
    }
    std::vector<uint32_t> thr, mode;
    sqa_msc_thresholds(coef, g->info.coupling_abs, g->info.max_degree, thr, mode);
    OJ_CK(ctx->params.ensure(std::max<size_t>((thr.size() + mode.size()) * 4, 16)), "alloc params");
    uint32_t* d_thr = ctx->params.as<uint32_t>();
    uint32_t* d_mode = d_thr + thr.size();
    if (S > 0) {
      OJ_CK(cudaMemcpyAsync(d_thr, thr.data(), thr.size() * 4, cudaMemcpyHostToDevice, st), "H2D thr");
      OJ_CK(cudaMemcpyAsync(d_mode, mode.data(), mode.size() * 4, cudaMemcpyHostToDevice, st), "H2D mode");
    }
    OJ_CK(ctx->words.ensure((size_t)G * 2 * n * 4), "alloc words");
    uint32_t* d_words = ctx->words.as<uint32_t>();
    if (!pipe) {
      OJ_CK(launch_sqa_split_pack(d_spins, R, T, n, G, d_words, st), "pack");
      ++launches;
    }
    Shape shp;
    auto it = g->tuned.find(key);
    if (it != g->tuned.end()) {
      shp = it->second;
    } else if (autotune_requested(flags) && S > 0) {
      std::vector<Shape> cand;
      for (int Pc : {1, 2, 4})
        if (Pc == 1 || n / Pc >= 64)
          for (int th : {256, 512}) cand.push_back(Shape{Pc, th, 0});
      int def_split = -1;  // the heuristic shape (the plan prepared above)
      for (size_t q = 0; q < cand.size(); ++q)
        if (cand[q].cluster == g->msc->P && cand[q].threads == split_default_threads()) def_split = (int)q;
      OJ_CK(ctx->aux.ensure((size_t)G * 2 * n * 4), "alloc tuning scratch");
      uint32_t* scratch = ctx->aux.as<uint32_t>();
      const int64_t Ssub = std::min<int64_t>(S, 16);
      cudaError_t terr = cudaSuccess;
      const int bi = time_candidates(
          st, (int)cand.size(),
          [&] { return cudaMemcpyAsync(scratch, d_words, (size_t)G * 2 * n * 4, cudaMemcpyDeviceToDevice, st); },
          [&](int i) {
            std::string w;
            const cudaError_t e = sqa_split_prepare(g, G, ctx->sm_count, &w, cand[i].cluster);
            if (e != cudaSuccess || g->msc->P != cand[i].cluster) return e != cudaSuccess ? e : cudaErrorInvalidValue;
            return launch_sqa_split(g, G, T, scratch, d_thr, d_mode, Ssub, rb, st, nullptr, cand[i].threads);
          },
          &terr, def_split);
      if (bi == -2) return cuda_fail(ctx, terr, "autotune");
      if (bi >= 0) shp = cand[bi];
      g->tuned[key] = shp;
      tuned_now = true;
    }
    {
      const cudaError_t pe2 = sqa_split_prepare(g, G, ctx->sm_count, &why, shp.cluster);
      if (pe2 != cudaSuccess) {
        return prep_fail(ctx, pe2, why);
      }
    }
    P_used = g->msc->P;
    threads_used = shp.threads ? shp.threads : split_default_threads();
    if (!pipe) {
      OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
      if (S > 0)
        OJ_CK(launch_sqa_split(g, G, T, d_words, d_thr, d_mode, S, rbm, st, &launches, threads_used),
              "sqa slice-split kernel");
      OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
      OJ_CK(launch_sqa_split_unpack(d_words, R, T, n, G, d_spins, st), "unpack");
      ++launches;
    } else {
      // halves: groups [0, GA) on the context stream, [GA, G) on the second
      // stream, each copied in, packed, annealed (at its global group index,
      // so with the same draws), unpacked, its energies and best slices
      // computed and all of it copied out; every buffer is sized before the
      // first launch
      OJ_CK(pipe_streams(ctx), "pipeline streams");
      const cudaStream_t s2 = ctx->gstream;
      // a call that fails part way waits for the second stream's work before
      // it returns, so that no copy of it still runs into the buffers
      struct JoinOnError {
        cudaStream_t s;
        bool armed = true;
        ~JoinOnError() {
          if (armed) cudaStreamSynchronize(s);
        }
      } join{s2};
      const int GA = (G + 1) / 2, RA = GA * P, RB = R - RA;
      const size_t offB = (size_t)RA * T * n;
      uint32_t* wB = d_words + (size_t)GA * 2 * n;
      double* d_e = nullptr;
      int32_t* d_b = nullptr;
      double *partsA = nullptr, *partsB = nullptr;
      const int nsA = energy_splits(g, RA * T, ctx->sm_count), nsB = energy_splits(g, RB * T, ctx->sm_count);
      if (energies || best_slice) {
        OJ_CK(ctx->energies.ensure((size_t)R * T * 8), "alloc energies");
        d_e = ctx->energies.as<double>();
        const size_t pa = nsA > 1 ? (size_t)nsA * RA * T : 0, pb = nsB > 1 ? (size_t)nsB * RB * T : 0;
        if (pa + pb > 0) {
          OJ_CK(ctx->eparts.ensure((pa + pb) * 8), "alloc energy parts");
          partsA = nsA > 1 ? ctx->eparts.as<double>() : nullptr;
          partsB = nsB > 1 ? ctx->eparts.as<double>() + pa : nullptr;
        }
      }
      if (best_slice) {
        OJ_CK(ctx->best.ensure((size_t)R * 4), "alloc best");
        d_b = ctx->best.as<int32_t>();
      }
      OJ_CK(cudaEventRecord(ctx->pev[0], st), "event");
      OJ_CK(cudaStreamWaitEvent(s2, ctx->pev[0], 0), "event wait");
      RngBase rbB = rbm;
      rbB.rep0 += (uint32_t)RA;
      OJ_CK(cudaMemcpyAsync(d_spins, spins, offB, cudaMemcpyHostToDevice, st), "H2D spins");
      OJ_CK(launch_sqa_split_pack(d_spins, RA, T, n, GA, d_words, st), "pack");
      OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
      OJ_CK(launch_sqa_split(g, GA, T, d_words, d_thr, d_mode, S, rbm, st, &launches, threads_used),
            "sqa slice-split kernel");
      OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
      OJ_CK(cudaMemcpyAsync(d_spins + offB, spins + offB, spin_bytes - offB, cudaMemcpyHostToDevice, s2),
            "H2D spins");
      OJ_CK(launch_sqa_split_pack(d_spins + offB, RB, T, n, G - GA, wB, s2), "pack");
      OJ_CK(launch_sqa_split(g, G - GA, T, wB, d_thr, d_mode, S, rbB, s2, &launches, threads_used),
            "sqa slice-split kernel");
      OJ_CK(cudaEventRecord(ctx->pev[1], s2), "event");
      OJ_CK(launch_sqa_split_unpack(d_words, RA, T, n, GA, d_spins, st), "unpack");
      OJ_CK(launch_sqa_split_unpack(wB, RB, T, n, G - GA, d_spins + offB, s2), "unpack");
      launches += 4;  // packs and unpacks
      if (d_e) {
        double* eB = d_e + (size_t)RA * T;
        OJ_CK(launch_energy(g, RA * T, d_spins, d_e, st, nsA, partsA), "energy kernel");
        OJ_CK(launch_energy(g, RB * T, d_spins + offB, eB, s2, nsB, partsB), "energy kernel");
        launches += (nsA > 1 ? 2 : 1) + (nsB > 1 ? 2 : 1);
        if (energies) {
          OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)RA * T * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
          OJ_CK(cudaMemcpyAsync(energies + (size_t)RA * T, eB, (size_t)RB * T * 8, cudaMemcpyDeviceToHost, s2),
                "D2H energies");
        }
        if (d_b) {
          OJ_CK(launch_best_slice(d_e, RA, T, d_b, st), "best slice");
          OJ_CK(launch_best_slice(eB, RB, T, d_b + RA, s2), "best slice");
          launches += 2;
          OJ_CK(cudaMemcpyAsync(best_slice, d_b, (size_t)RA * 4, cudaMemcpyDeviceToHost, st), "D2H best");
          OJ_CK(cudaMemcpyAsync(best_slice + RA, d_b + RA, (size_t)RB * 4, cudaMemcpyDeviceToHost, s2),
                "D2H best");
        }
      }
      OJ_CK(cudaMemcpyAsync(spins, d_spins, offB, cudaMemcpyDeviceToHost, st), "D2H spins");
      OJ_CK(cudaMemcpyAsync(spins + offB, d_spins + offB, spin_bytes - offB, cudaMemcpyDeviceToHost, s2),
            "D2H spins");
      OJ_CK(cudaEventRecord(ctx->pev[2], s2), "event");
      OJ_CK(cudaStreamWaitEvent(st, ctx->pev[2], 0), "event wait");
      join.armed = false;
    }
  } else if (kernel == OJ_KERNEL_BITPACKED) {
    OJ_CK(sqa_msc_prepare(g), "bit-packed SQA tables");
    std::vector<uint32_t> thr, mode;
    sqa_msc_thresholds(coef, g->info.coupling_abs, g->info.max_degree, thr, mode);
    OJ_CK(ctx->params.ensure(std::max<size_t>((thr.size() + mode.size()) * 4, 16)), "alloc params");
    uint32_t* d_thr = ctx->params.as<uint32_t>();
    uint32_t* d_mode = d_thr + thr.size();
    if (S > 0) {
      OJ_CK(cudaMemcpyAsync(d_thr, thr.data(), thr.size() * 4, cudaMemcpyHostToDevice, st), "H2D thr");
      OJ_CK(cudaMemcpyAsync(d_mode, mode.data(), mode.size() * 4, cudaMemcpyHostToDevice, st), "H2D mode");
    }
    OJ_CK(ctx->words.ensure((size_t)R * n * 4), "alloc words");
    uint32_t* d_words = ctx->words.as<uint32_t>();
    OJ_CK(launch_sqa_pack(d_spins, R, T, n, d_words, st), "pack");
    ++launches;
    OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
    if (S > 0) OJ_CK(launch_sqa_msc(g, R, T, d_words, d_thr, d_mode, S, rbm, st, &launches), "sqa bit-packed kernel");
    OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
    OJ_CK(launch_sqa_unpack(d_words, R, T, n, d_spins, st), "unpack");
    ++launches;
  } else {
    OJ_CK(ctx->params.ensure(std::max<size_t>(coef.size() * sizeof(float2), 16)), "alloc params");
    float2* d_coef = ctx->params.as<float2>();
    if (S > 0)
      OJ_CK(cudaMemcpyAsync(d_coef, coef.data(), coef.size() * sizeof(float2), cudaMemcpyHostToDevice, st),
            "H2D coef");
    OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
    if (S > 0) OJ_CK(launch_sqa_colour(g, R, T, d_spins, d_coef, S, rbm, st, &launches), "sqa kernel");
    OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
  }
  if (pipe) {
    // the halves computed and copied out their energies, best slices and spins
  } else if (energies || best_slice) {
    double* d_e = (devp && energies) ? energies : nullptr;
    if (!d_e) {
      OJ_CK(ctx->energies.ensure((size_t)R * T * 8), "alloc energies");
      d_e = ctx->energies.as<double>();
    }
    OJ_CK(graph_energy(ctx, g, R * T, d_spins, d_e, st, &launches), "energy kernel");
    if (energies && !devp)
      OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)R * T * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
    if (best_slice) {
      int32_t* d_b = devp ? best_slice : nullptr;
      if (!d_b) {
        OJ_CK(ctx->best.ensure((size_t)R * 4), "alloc best");
        d_b = ctx->best.as<int32_t>();
      }
      OJ_CK(launch_best_slice(d_e, R, T, d_b, st), "best slice");
      ++launches;
      if (!devp) OJ_CK(cudaMemcpyAsync(best_slice, d_b, (size_t)R * 4, cudaMemcpyDeviceToHost, st), "D2H best");
    }
  }
  if (!devp && !pipe) OJ_CK(cudaMemcpyAsync(spins, d_spins, spin_bytes, cudaMemcpyDeviceToHost, st), "D2H spins");
  OJ_CK(cudaEventRecord(ctx->ev[3], st), "event");
  if (!devp || stats) OJ_CK(cudaStreamSynchronize(st), "run");
  if (stats) {
    stats->kernel = (int32_t)(kernel >> OJ_KERNEL_SHIFT);
    stats->launches = launches;
    stats->sweeps = S;
    stats->attempts = (double)R * T * n * (double)S;
    stats->cluster = P_used;
    stats->threads = threads_used;
    stats->tuned = tuned_now ? 1 : 0;
    cudaEventElapsedTime(&stats->anneal_ms, ctx->ev[1], ctx->ev[2]);
    if (pipe) {
      // from the first half's kernel start to the later of the two ends
      float tb = 0.0f;
      cudaEventElapsedTime(&tb, ctx->ev[1], ctx->pev[1]);
      stats->anneal_ms = std::max(stats->anneal_ms, tb);
    }
    cudaEventElapsedTime(&stats->total_ms, ctx->ev[0], ctx->ev[3]);
    stats->accepted = read_counters(ctx).flips;
    stats->field_drift = -1.0;
  }
  return OJ_OK;
}

oj_status oj_energy(oj_ctx* ctx, const oj_graph* g, int32_t R, const int8_t* spins, uint32_t flags,
                    double* energies) {
  if (!ctx || !g || R < 0 || (R > 0 && (!spins || !energies))) return arg_fail(ctx, "null argument");
  if (R == 0) return OJ_OK;
  if (g->n == 0) {
    for (int32_t r = 0; r < R; ++r) energies[r] = 0.0;
    return OJ_OK;
  }
  DeviceGuard dg(ctx->device);
  const bool devp = (flags & OJ_DEVICE_POINTERS) != 0;
  cudaStream_t st = ctx->stream;
  const int8_t* d_spins = spins;
  double* d_e = energies;
  if (!devp) {
    OJ_CK(ctx->aux.ensure((size_t)R * g->n), "alloc spins");
    OJ_CK(cudaMemcpyAsync(ctx->aux.ptr, spins, (size_t)R * g->n, cudaMemcpyHostToDevice, st), "H2D spins");
    d_spins = ctx->aux.as<int8_t>();
    OJ_CK(ctx->energies.ensure((size_t)R * 8), "alloc energies");
    d_e = ctx->energies.as<double>();
  }
  OJ_CK(graph_energy(ctx, g, R, d_spins, d_e, st, nullptr), "energy kernel");
  if (!devp) {
    OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)R * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
    OJ_CK(cudaStreamSynchronize(st), "energy");
  }
  return OJ_OK;
}

oj_status oj_graph_flip_stats(oj_ctx* ctx, const oj_graph* g, int32_t K, const int8_t* spins, double threshold,
                              double* dE_quad, double* dE_lin, double* abs_min) {
  if (!ctx || !g || !abs_min || K < 1 || K > flip_stats_max_k() || (g->n > 0 && (!spins || !dE_quad || !dE_lin)))
    return arg_fail(ctx, "null argument or K outside 1..8");
  const int n = g->n;
  for (size_t q = 0; q < (size_t)n * K; ++q)
    if (spins[q] != 1 && spins[q] != -1) return arg_fail(ctx, "spins must be +1 or -1");
  // the corner (n, n) of the augmented matrix is part of the reference's minimum
  double amin = INFINITY;
  for (int64_t p = g->aug_indptr[n]; p < g->aug_indptr[n + 1]; ++p)
    if (g->aug_indices[p] == n && std::fabs(g->aug_data[p]) > threshold) amin = std::fabs(g->aug_data[p]);
  if (n == 0) {
    *abs_min = amin;
    return OJ_OK;
  }
  DeviceGuard dg(ctx->device);
  cudaStream_t st = ctx->stream;
  const size_t nk = (size_t)n * K;
  OJ_CK(ctx->aux.ensure(nk), "alloc spins");
  OJ_CK(ctx->energies.ensure(nk * 16 + 8), "alloc statistics");
  double* d_quad = ctx->energies.as<double>();
  double* d_lin = d_quad + nk;
  unsigned long long* d_min = reinterpret_cast<unsigned long long*>(d_lin + nk);
  unsigned long long m0;
  std::memcpy(&m0, &amin, 8);
  OJ_CK(cudaMemcpyAsync(ctx->aux.ptr, spins, nk, cudaMemcpyHostToDevice, st), "H2D spins");
  OJ_CK(cudaMemcpyAsync(d_min, &m0, 8, cudaMemcpyHostToDevice, st), "H2D minimum");
  OJ_CK(launch_flip_stats(g, K, ctx->aux.as<int8_t>(), threshold, d_quad, d_lin, d_min, st), "flip statistics kernel");
  OJ_CK(cudaMemcpyAsync(dE_quad, d_quad, nk * 8, cudaMemcpyDeviceToHost, st), "D2H quad");
  OJ_CK(cudaMemcpyAsync(dE_lin, d_lin, nk * 8, cudaMemcpyDeviceToHost, st), "D2H lin");
  OJ_CK(cudaMemcpyAsync(&m0, d_min, 8, cudaMemcpyDeviceToHost, st), "D2H minimum");
  OJ_CK(cudaStreamSynchronize(st), "flip statistics");
  std::memcpy(abs_min, &m0, 8);
  return OJ_OK;
}

oj_status oj_batch_flip_stats(oj_ctx* ctx, const oj_batch* b, int32_t K, const int8_t* spins, double threshold,
                              double* dE_quad, double* dE_lin, double* abs_min) {
  if (!ctx || !b || K < 1 || K > flip_stats_max_k() || (b->count > 0 && !abs_min))
    return arg_fail(ctx, "null argument or K outside 1..8");
  std::vector<int64_t> soff(b->count + 1, 0);
  for (int k = 0; k < b->count; ++k) soff[k + 1] = soff[k] + b->n[k];
  const size_t nk = (size_t)soff[b->count] * K;
  if (nk > 0 && (!spins || !dE_quad || !dE_lin)) return arg_fail(ctx, "null argument");
  for (size_t q = 0; q < nk; ++q)
    if (spins[q] != 1 && spins[q] != -1) return arg_fail(ctx, "spins must be +1 or -1");
  if (b->count == 0) return OJ_OK;
  DeviceGuard dg(ctx->device);
  cudaStream_t st = ctx->stream;
  const size_t soff_bytes = (size_t)b->count * 8, spin_at = (soff_bytes + 255) & ~(size_t)255;
  OJ_CK(ctx->aux.ensure(spin_at + std::max<size_t>(nk, 1)), "alloc spins");
  OJ_CK(ctx->energies.ensure(nk * 16 + (size_t)b->count * 8), "alloc statistics");
  double* d_quad = ctx->energies.as<double>();
  double* d_lin = d_quad + nk;
  unsigned long long* d_min = reinterpret_cast<unsigned long long*>(d_lin + nk);
  const double inf = INFINITY;
  unsigned long long inf_bits;
  std::memcpy(&inf_bits, &inf, 8);
  std::vector<unsigned long long> m(b->count, inf_bits);
  char* aux = ctx->aux.as<char>();
  OJ_CK(cudaMemcpyAsync(aux, soff.data(), soff_bytes, cudaMemcpyHostToDevice, st), "H2D offsets");
  if (nk) OJ_CK(cudaMemcpyAsync(aux + spin_at, spins, nk, cudaMemcpyHostToDevice, st), "H2D spins");
  OJ_CK(cudaMemcpyAsync(d_min, m.data(), m.size() * 8, cudaMemcpyHostToDevice, st), "H2D minima");
  OJ_CK(launch_batch_flip_stats(b, K, reinterpret_cast<int8_t*>(aux + spin_at), reinterpret_cast<int64_t*>(aux),
                                threshold, d_quad, d_lin, d_min, st),
        "batch flip statistics kernel");
  if (nk) {
    OJ_CK(cudaMemcpyAsync(dE_quad, d_quad, nk * 8, cudaMemcpyDeviceToHost, st), "D2H quad");
    OJ_CK(cudaMemcpyAsync(dE_lin, d_lin, nk * 8, cudaMemcpyDeviceToHost, st), "D2H lin");
  }
  OJ_CK(cudaMemcpyAsync(m.data(), d_min, m.size() * 8, cudaMemcpyDeviceToHost, st), "D2H minima");
  OJ_CK(cudaStreamSynchronize(st), "batch flip statistics");
  std::memcpy(abs_min, m.data(), m.size() * 8);
  return OJ_OK;
}

oj_status oj_batch_create_dense(oj_ctx* ctx, int32_t count, const int32_t* n, const int64_t* offset,
                                const double* J_aug, oj_batch** out) {
  return build_batch(ctx, count, n, offset, J_aug, out);
}

}  // extern "C"

namespace {
oj_status build_batch(oj_ctx* ctx, int32_t count, const int32_t* n, const int64_t* offset, const double* J_aug,
                      oj_batch** out, bool checked) {
  if (!ctx || !out || count < 0 || (count > 0 && (!n || !offset || !J_aug)))
    return arg_fail(ctx, "null argument or negative size");
  *out = nullptr;
  const int nmax = batch_max_sites();
  std::vector<int64_t> joff(count), hoff(count), j64off(count);
  int64_t tot32 = 0, toth = 0, tot64 = 0;
  int max_n = 0;
  for (int32_t k = 0; k < count; ++k) {
    if (n[k] < 0 || n[k] > nmax) return arg_fail(ctx, "batched instances need 0 <= n <= 4096");
    if (offset[k] < 0) return arg_fail(ctx, "negative instance offset");
    const int64_t npad = ((int64_t)n[k] + 127) / 128 * 128;
    joff[k] = tot32;
    hoff[k] = toth;
    j64off[k] = tot64;
    tot32 += (int64_t)n[k] * npad;
    toth += npad;
    tot64 += ((int64_t)n[k] + 1) * ((int64_t)n[k] + 1);
    max_n = std::max(max_n, (int)n[k]);
  }
  std::vector<float> J32, h32;
  std::vector<double> J64;
  try {
    J32.assign((size_t)std::max<int64_t>(tot32, 4), 0.0f);
    h32.assign((size_t)std::max<int64_t>(toth, 4), 0.0f);
    J64.assign((size_t)std::max<int64_t>(tot64, 1), 0.0);
  } catch (...) {
    return OJ_ERR_OOM;
  }
  for (int32_t k = 0; k < count; ++k) {
    const int64_t nk = n[k], n1 = nk + 1, npad = (nk + 127) / 128 * 128;
    const double* A = J_aug + offset[k];
    // graph::Dense::set_interaction_matrix checks (dense.hpp:117-140)
    if (A[nk * n1 + nk] != 1.0) return arg_fail(ctx, "the corner of an augmented matrix must be 1");
    for (int64_t q = 0; q < n1 * n1; ++q)
      if (!std::isfinite(A[q])) return arg_fail(ctx, "couplings and fields must be finite");
    for (int64_t i = 0; i < n1 && !checked; ++i) {
      if (i < nk && A[i * n1 + i] != 0.0) return arg_fail(ctx, "the diagonal of J must be zero (h goes in column n)");
      for (int64_t j = i + 1; j < n1; ++j)
        if (A[i * n1 + j] != A[j * n1 + i]) return arg_fail(ctx, "an augmented matrix is not symmetric");
    }
    for (int64_t i = 0; i < nk; ++i) {
      for (int64_t j = 0; j < nk; ++j) J32[(size_t)(joff[k] + i * npad + j)] = (float)A[i * n1 + j];
      h32[(size_t)(hoff[k] + i)] = (float)A[i * n1 + nk];
    }
    std::memcpy(J64.data() + j64off[k], A, (size_t)(n1 * n1) * sizeof(double));
  }
  // The FP32 fields are exact when every coupling and field is a multiple of
  // 2^-p and no field can reach 2^(24-p): then the sweep kernel's fields give
  // the FP64 energies exactly, E = 1/2 sum_i s_i (f_i + h_i).
  bool exact = true;
  int pmax = 0;
  double maxrow = 0.0, maxj = 0.0;  // largest row sum of |values| (h included), largest |J|
  auto grid_p = [](double v) {  // smallest p >= 0 with v 2^p an integer (v != 0), from its bits
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    const int ex = (int)((bits >> 52) & 0x7FF);
    if (ex == 0 || ex == 0x7FF) return 1000;  // subnormal, inf, nan
    const uint64_t mant = (bits & ((1ull << 52) - 1)) | (1ull << 52);
    const int low = ex - 1075 + __builtin_ctzll(mant);  // v = odd * 2^low
    return low >= 0 ? 0 : -low;
  };
  for (int32_t k = 0; k < count && exact; ++k) {
    const int64_t nk = n[k], n1 = nk + 1;
    const double* A = J_aug + offset[k];
    for (int64_t i = 0; i < nk && exact; ++i) {
      double row = 0.0;
      for (int64_t j = 0; j < n1; ++j) {
        const double v = A[i * n1 + j];
        if (v == 0.0) continue;
        const int p = grid_p(v);
        if (p > 24) {
          exact = false;
          break;
        }
        pmax = std::max(pmax, p);
        row += std::fabs(v);
        if (j < nk) maxj = std::max(maxj, std::fabs(v));
      }
      maxrow = std::max(maxrow, row);
    }
  }
  exact = exact && std::ldexp(maxrow, pmax) < 16777216.0;
  std::unique_ptr<oj_batch> b(new oj_batch());
  b->exact_fields = exact;
  b->device = ctx->device;
  b->count = count;
  b->max_n = max_n;
  b->n.assign(n, n + count);
  DeviceGuard dg(ctx->device);
  auto up = [&](DevBuf& d, const void* src, size_t bytes) -> cudaError_t {
    cudaError_t e = d.ensure(std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) return e;
    return bytes ? cudaMemcpy(d.ptr, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  OJ_CK(up(b->d_J, J32.data(), J32.size() * 4), "upload J");
  // flip rows in half the bytes when FP16 holds every FP32 coupling exactly
  // (integer and quarter-integer couplings of moderate size): the kernel
  // widens them back to the same FP32 values
  {
    // an FP32 value is an FP16 normal (or zero) when its exponent is within
    // [-14, 15] and its low 13 mantissa bits are zero; the FP16 bits are then
    // the sign, the rebiased exponent and the top 10 mantissa bits
    std::vector<uint16_t> J16(J32.size());
    bool exact16 = true;
    for (size_t q = 0; q < J32.size() && exact16; ++q) {
      uint32_t u;
      std::memcpy(&u, &J32[q], 4);
      if ((u & 0x7FFFFFFFu) == 0) {
        J16[q] = (uint16_t)(u >> 16);
        continue;
      }
      const int ex = (int)((u >> 23) & 0xFF) - 127;
      if (ex < -14 || ex > 15 || (u & 0x1FFFu) != 0) {
        exact16 = false;
        break;
      }
      J16[q] = (uint16_t)(((u >> 16) & 0x8000u) | ((uint32_t)(ex + 15) << 10) | ((u >> 13) & 0x3FFu));
    }
    if (exact16) {
      OJ_CK(up(b->d_J16, J16.data(), J16.size() * 2), "upload J16");
      b->j16 = true;
    }
  }
  // exact fields with every J 2^p an integer of at most 127: J 2^p as int8,
  // one digit of the tensor-core field kernel; other couplings get four digits
  std::vector<int8_t> J8;
  if (exact && std::ldexp(maxj, pmax) <= 127.0) {
    J8.resize(J32.size());
    for (size_t q = 0; q < J32.size(); ++q) J8[q] = (int8_t)std::ldexp((double)J32[q], pmax);
    b->j8 = true;
    b->j8_scale = (float)std::ldexp(1.0, -pmax);
  }
  OJ_CK(field_tc_prepare(b.get(), J32, joff, b->j8 ? &J8 : nullptr, pmax), "field digits");
  OJ_CK(up(b->d_h, h32.data(), h32.size() * 4), "upload h");
  OJ_CK(up(b->d_J64, J64.data(), J64.size() * 8), "upload J64");
  OJ_CK(up(b->d_joff, joff.data(), joff.size() * 8), "upload offsets");
  OJ_CK(up(b->d_hoff, hoff.data(), hoff.size() * 8), "upload offsets");
  OJ_CK(up(b->d_j64off, j64off.data(), j64off.size() * 8), "upload offsets");
  OJ_CK(up(b->d_n, n, (size_t)count * 4), "upload sizes");
  *out = b.release();
  return OJ_OK;
}
}  // namespace

extern "C" {

oj_status oj_batch_destroy(oj_batch* b) {
  delete b;
  return OJ_OK;
}

oj_status oj_sa_run_batched(oj_ctx* ctx, const oj_batch* b, const int32_t* reads, int8_t* spins,
                            const double* betas, const int32_t* mcs, int32_t num_sched, uint64_t seed,
                            int64_t first_sweep, int64_t instance_offset, uint32_t flags, double* energies,
                            oj_run_stats* stats) {
  if (!ctx || !b || num_sched < 0 || (b->count > 0 && !reads)) return arg_fail(ctx, "null argument or negative size");
  if (num_sched > 0 && (!betas || !mcs)) return arg_fail(ctx, "null schedule");
  if (b->device != ctx->device) return arg_fail(ctx, "batch belongs to another device");
  if (instance_offset < 0 || instance_offset + b->count > (1 << 24))
    return arg_fail(ctx, "instance_offset + count must be below 2^24");
  if ((flags & OJ_KERNEL_MASK) != OJ_KERNEL_AUTO) {
    ctx->last_error = "batched SA has a single kernel; pass OJ_KERNEL_AUTO";
    return OJ_ERR_UNSUPPORTED;
  }
  for (int32_t k = 0; k < num_sched; ++k)
    if (!(betas[k] >= 0.0) || std::isinf(betas[k])) return arg_fail(ctx, "beta must be finite and >= 0");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  const int count = b->count;
  std::vector<int64_t> soff(count), eoff(count), foff(count);
  int64_t sbytes = 0, nrep = 0, nfield = 0;
  int max_reads = 0;
  double attempts_per_sweep = 0.0;
  for (int k = 0; k < count; ++k) {
    if (reads[k] < 0) return arg_fail(ctx, "negative read count");
    soff[k] = sbytes;
    eoff[k] = nrep;
    foff[k] = nfield;
    sbytes += (int64_t)reads[k] * b->n[k];
    nfield += (int64_t)reads[k] * (((int64_t)b->n[k] + 127) / 128 * 128);
    nrep += reads[k];
    max_reads = std::max(max_reads, (int)reads[k]);
    attempts_per_sweep += (double)reads[k] * b->n[k];
  }
  if (nrep == 0) return OJ_OK;
  if (!spins && sbytes > 0) return arg_fail(ctx, "null spins");
  // work items (instance, group of W replicas), longest instance first; W is
  // the warps per CTA of the launch variant
  std::vector<int> order(count);
  for (int k = 0; k < count; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->n[x] > b->n[y]; });
  auto make_items = [&](int W) {
    std::vector<int32_t> it;
    for (int k : order) {
      if (b->n[k] == 0) continue;
      for (int gq = 0; gq * W < reads[k]; ++gq) {
        it.push_back(k);
        it.push_back(gq);
      }
    }
    return it;
  };
  oj_batch* bm = const_cast<oj_batch*>(b);
  int variant0 = bm->tuned_variant ? bm->tuned_variant : batch_default_variant();
  if (b->max_n > batch_variant_max_n(variant0)) variant0 = 83;
  std::vector<int32_t> items = make_items(batch_variant_warps(variant0));
  const size_t items_cap = make_items(batch_min_warps()).size();  // the most items of any variant
  int nitems = (int)(items.size() / 2);
  RngBase rb;
  if (oj_status st_ = rng_base(ctx, seed, first_sweep, 0, &rb)) return st_;
  DeviceGuard dg(ctx->device);
  std::vector<double> bexp;
  if (oj_status st_ = expand(ctx, betas, mcs, num_sched, bexp)) return st_;
  const int64_t S = (int64_t)bexp.size();
  std::vector<float> bf(bexp.begin(), bexp.end());
  const bool devp = (flags & OJ_DEVICE_POINTERS) != 0;
  cudaStream_t st = ctx->stream;
  int8_t* d_spins = spins;
  if (!devp) {
    OJ_CK(ctx->spins.ensure(std::max<int64_t>(sbytes, 16)), "alloc spins");
    d_spins = ctx->spins.as<int8_t>();
  } else if (sbytes > 0 && !is_device_ptr(spins)) {
    return arg_fail(ctx, "OJ_DEVICE_POINTERS set but spins is not device memory");
  }
  // one staging buffer: reads | soff | eoff | items | counter | betas | order | foff
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t b_reads = al((size_t)count * 4), b_soff = al((size_t)count * 8), b_eoff = al((size_t)count * 8),
               b_items = al(items_cap * 4 + 4), b_cnt = al(4), b_beta = al(bf.size() * 4 + 4),
               b_order = al((size_t)count * 4), b_foff = al((size_t)count * 8);
  OJ_CK(ctx->batch.ensure(b_reads + b_soff + b_eoff + b_items + b_cnt + b_beta + b_order + b_foff),
        "alloc batch tables");
  // initial fields of every replica of every instance, [reads][n rounded up to 128] floats each
  OJ_CK(ctx->fields.ensure(std::max<size_t>((size_t)nfield * 4, 16)), "alloc fields");
  float* d_fields = ctx->fields.as<float>();
  char* base = ctx->batch.as<char>();
  int32_t* d_reads = reinterpret_cast<int32_t*>(base);
  int64_t* d_soff = reinterpret_cast<int64_t*>(base + b_reads);
  int64_t* d_eoff = reinterpret_cast<int64_t*>(base + b_reads + b_soff);
  int32_t* d_items = reinterpret_cast<int32_t*>(base + b_reads + b_soff + b_eoff);
  int* d_counter = reinterpret_cast<int*>(base + b_reads + b_soff + b_eoff + b_items);
  float* d_beta = reinterpret_cast<float*>(base + b_reads + b_soff + b_eoff + b_items + b_cnt);
  int32_t* d_order = reinterpret_cast<int32_t*>(base + b_reads + b_soff + b_eoff + b_items + b_cnt + b_beta);
  int64_t* d_foff = reinterpret_cast<int64_t*>(base + b_reads + b_soff + b_eoff + b_items + b_cnt + b_beta + b_order);
  int launches = 0;
  RngBase rbm = rb;  // rb of the main annealing launch (counts accepted flips)
  if (oj_status cs = arm_counters(ctx, stats, &rbm)) return cs;
  FieldCall fc;
  if (oj_status fs = field_call(ctx, b, reads, order, max_reads, &fc)) return fs;
  OJ_CK(cudaEventRecord(ctx->ev[0], st), "event");
  if (!devp && sbytes > 0) OJ_CK(cudaMemcpyAsync(d_spins, spins, sbytes, cudaMemcpyHostToDevice, st), "H2D spins");
  OJ_CK(cudaMemcpyAsync(d_reads, reads, (size_t)count * 4, cudaMemcpyHostToDevice, st), "H2D reads");
  OJ_CK(cudaMemcpyAsync(d_soff, soff.data(), (size_t)count * 8, cudaMemcpyHostToDevice, st), "H2D offsets");
  OJ_CK(cudaMemcpyAsync(d_eoff, eoff.data(), (size_t)count * 8, cudaMemcpyHostToDevice, st), "H2D offsets");
  if (nitems) OJ_CK(cudaMemcpyAsync(d_items, items.data(), items.size() * 4, cudaMemcpyHostToDevice, st), "H2D items");
  if (S > 0) OJ_CK(cudaMemcpyAsync(d_beta, bf.data(), bf.size() * 4, cudaMemcpyHostToDevice, st), "H2D betas");
  if (count) OJ_CK(cudaMemcpyAsync(d_order, order.data(), (size_t)count * 4, cudaMemcpyHostToDevice, st), "H2D order");
  if (count) OJ_CK(cudaMemcpyAsync(d_foff, foff.data(), (size_t)count * 8, cudaMemcpyHostToDevice, st), "H2D offsets");
  bool tuned_now = false;
  if (bm->tuned_variant == 0 && autotune_requested(flags) && S > 0 && nitems > 0) {
    // the work per sweep follows the acceptance rate, so the candidates run 16
    // sweeps whose betas are spread over the whole schedule
    std::vector<int> cand;
    for (int v : {45, 82, 83, 84, 162, 321})
      if (b->max_n <= batch_variant_max_n(v)) cand.push_back(v);
    const int64_t Ssub = std::min<int64_t>(S, 32);
    std::vector<float> tb(Ssub);
    for (int64_t q = 0; q < Ssub; ++q) tb[q] = bf[(size_t)((q * S) / Ssub)];
    const size_t sb_al = ((size_t)std::max<int64_t>(sbytes, 16) + 255) & ~(size_t)255;
    OJ_CK(ctx->aux.ensure(sb_al + tb.size() * 4), "alloc tuning scratch");
    int8_t* scratch = ctx->aux.as<int8_t>();
    float* d_tb = reinterpret_cast<float*>(ctx->aux.as<char>() + sb_al);
    OJ_CK(cudaMemcpyAsync(d_tb, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice, st), "H2D tuning betas");
    cudaError_t terr = cudaSuccess;
    int loaded = -1;  // variant whose items are in d_items
    std::vector<int32_t> it;
    const int bi = time_candidates(
        st, (int)cand.size(), [&] { return cudaMemcpyAsync(scratch, d_spins, sbytes, cudaMemcpyDeviceToDevice, st); },
        [&](int i) {
          if (loaded != i) {
            it = make_items(batch_variant_warps(cand[i]));
            if (it.size() > items_cap) return cudaErrorInvalidValue;  // never past the table
            const cudaError_t e = cudaMemcpyAsync(d_items, it.data(), it.size() * 4, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return e;
            loaded = i;
          }
          return launch_sa_batch(b, d_reads, d_soff, d_items, (int)(it.size() / 2), d_counter, scratch, d_tb, Ssub,
                                 rb, (uint32_t)instance_offset, ctx->sm_count, st, nullptr, cand[i], d_fields, d_foff,
                                 fc);
        },
        &terr, (int)(std::find(cand.begin(), cand.end(), variant0) - cand.begin()));
    if (bi == -2) return cuda_fail(ctx, terr, "autotune");
    bm->tuned_variant = bi >= 0 ? cand[bi] : 83;
    tuned_now = true;
    items = make_items(batch_variant_warps(bm->tuned_variant));
    nitems = (int)(items.size() / 2);
    OJ_CK(cudaMemcpyAsync(d_items, items.data(), items.size() * 4, cudaMemcpyHostToDevice, st), "H2D items");
  }
  // exact FP32 fields: the sweep kernel writes the energies of the replicas it
  // anneals (every instance with n > 0 has items); instances with n = 0 have E = 0
  double* d_e = nullptr;
  if (energies) {
    d_e = devp ? energies : nullptr;
    if (!d_e) {
      OJ_CK(ctx->energies.ensure((size_t)nrep * 8), "alloc energies");
      d_e = ctx->energies.as<double>();
    }
  }
  const bool energies_in_kernel = energies && S > 0 && nitems > 0 && b->exact_fields;
  if (energies_in_kernel) OJ_CK(cudaMemsetAsync(d_e, 0, (size_t)nrep * 8, st), "energies of empty instances");
  OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
  const bool field_run = S > 0 && nitems > 0;
  if (field_run) {
    const SweepPlan sp{b, d_reads, d_soff, d_items, nitems, d_counter, d_spins, d_beta, (uint32_t)instance_offset,
                       bm->tuned_variant ? bm->tuned_variant : variant0, d_fields, d_foff,
                       energies_in_kernel ? d_e : nullptr, d_eoff};
    OJ_CK(run_batch(ctx, sp, S, rbm, fc, stats != nullptr, &launches), "sa batched kernel");
  }
  OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
  if (energies_in_kernel) {
    if (!devp) OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)nrep * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
  } else if (energies) {
    const int ns = batch_energy_splits(b, max_reads, ctx->sm_count);
    if (ns > 1) OJ_CK(ctx->eparts.ensure((size_t)ns * nrep * 8), "alloc energy parts");
    OJ_CK(launch_batch_energy(b, d_reads, d_soff, d_eoff, d_order, max_reads, d_spins, d_e, st, ns,
                              ctx->eparts.as<double>(), nrep),
          "batch energy kernel");
    launches += ns > 1 ? 2 : 1;
    if (!devp) OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)nrep * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
  }
  if (!devp && sbytes > 0) OJ_CK(cudaMemcpyAsync(spins, d_spins, sbytes, cudaMemcpyDeviceToHost, st), "D2H spins");
  OJ_CK(cudaEventRecord(ctx->ev[3], st), "event");
  OJ_CK(cudaStreamSynchronize(st), "run");
  const RunCounters rc = read_counters(ctx);
  if (field_run && rc.status) {
    ctx->last_error = "tensor-core field kernel: a bounded device wait ran out";
    return OJ_ERR_TIMEOUT;
  }
  if (stats) {
    stats->kernel = 0;
    stats->launches = launches;
    const int v = bm->tuned_variant ? bm->tuned_variant : variant0;
    stats->threads = batch_variant_warps(v) * 32;
    stats->variant = v;
    stats->tuned = tuned_now ? 1 : 0;
    stats->sweeps = S;
    stats->attempts = attempts_per_sweep * (double)S;
    cudaEventElapsedTime(&stats->anneal_ms, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&stats->total_ms, ctx->ev[0], ctx->ev[3]);
    stats->accepted = rc.flips;
    stats->field_drift = !field_run ? -1.0 : (b->exact_fields ? 0.0 : (double)rc.drift);
  }
  return OJ_OK;
}

oj_status oj_sw_run(oj_ctx* ctx, const oj_graph* gc, int32_t R, int8_t* spins, const double* betas,
                    const int32_t* mcs, int32_t num_sched, uint64_t seed, int64_t first_sweep,
                    int64_t replica_offset, uint32_t flags, double* energies, oj_run_stats* stats) {
  if (!ctx || !gc || R < 0 || num_sched < 0) return arg_fail(ctx, "null argument or negative size");
  if (num_sched > 0 && (!betas || !mcs)) return arg_fail(ctx, "null schedule");
  oj_graph* g = const_cast<oj_graph*>(gc);
  if (g->device != ctx->device) return arg_fail(ctx, "graph belongs to another device");
  const int n = g->n;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (R == 0 || n == 0) return OJ_OK;
  if (!spins) return arg_fail(ctx, "null spins");
  if ((flags & OJ_KERNEL_MASK) != OJ_KERNEL_AUTO) {
    ctx->last_error = "Swendsen-Wang has a single kernel; pass OJ_KERNEL_AUTO";
    return OJ_ERR_UNSUPPORTED;
  }
  for (int32_t k = 0; k < num_sched; ++k)
    if (!(betas[k] >= 0.0) || std::isinf(betas[k])) return arg_fail(ctx, "beta must be finite and >= 0");
  RngBase rb;
  if (oj_status st_ = rng_base(ctx, seed, first_sweep, replica_offset, &rb)) return st_;
  DeviceGuard dg(ctx->device);
  std::vector<double> bexp;
  if (oj_status st_ = expand(ctx, betas, mcs, num_sched, bexp)) return st_;
  const int64_t S = (int64_t)bexp.size();
  std::vector<float> bf(bexp.begin(), bexp.end());
  const bool devp = (flags & OJ_DEVICE_POINTERS) != 0;
  cudaStream_t st = ctx->stream;
  const size_t spin_bytes = (size_t)R * n;
  int8_t* d_spins = spins;
  if (!devp) {
    OJ_CK(ctx->spins.ensure(spin_bytes), "alloc spins");
    d_spins = ctx->spins.as<int8_t>();
  } else if (!is_device_ptr(spins)) {
    return arg_fail(ctx, "OJ_DEVICE_POINTERS set but spins is not device memory");
  }
  OJ_CK(sw_prepare(g), "bond list");
  int launches = 0;
  OJ_CK(cudaEventRecord(ctx->ev[0], st), "event");
  if (!devp) OJ_CK(cudaMemcpyAsync(d_spins, spins, spin_bytes, cudaMemcpyHostToDevice, st), "H2D spins");
  OJ_CK(ctx->params.ensure(std::max<size_t>(bf.size() * 4, 16)), "alloc params");
  float* d_beta = ctx->params.as<float>();
  if (S > 0) OJ_CK(cudaMemcpyAsync(d_beta, bf.data(), bf.size() * 4, cudaMemcpyHostToDevice, st), "H2D betas");
  OJ_CK(cudaEventRecord(ctx->ev[1], st), "event");
  // graphs above the shared-memory size keep the parent links of a chunk of
  // replicas in global scratch (at most 1 GiB)
  uint32_t* scratch = nullptr;
  int chunk = 0;
  if (n > sw_max_sites()) {
    const size_t per = ((size_t)n + 1) * 4;
    chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)R, ((size_t)1 << 30) / per));
    OJ_CK(ctx->aux.ensure(per * (size_t)chunk), "alloc union-find scratch");
    scratch = ctx->aux.as<uint32_t>();
  }
  if (S > 0) OJ_CK(launch_sw(g, R, d_spins, d_beta, S, rb, scratch, chunk, st, &launches), "swendsen-wang kernel");
  OJ_CK(cudaEventRecord(ctx->ev[2], st), "event");
  if (energies) {
    double* d_e = energies;
    if (!devp) {
      OJ_CK(ctx->energies.ensure((size_t)R * 8), "alloc energies");
      d_e = ctx->energies.as<double>();
    }
    OJ_CK(graph_energy(ctx, g, R, d_spins, d_e, st, &launches), "energy kernel");
    if (!devp) OJ_CK(cudaMemcpyAsync(energies, d_e, (size_t)R * 8, cudaMemcpyDeviceToHost, st), "D2H energies");
  }
  if (!devp) OJ_CK(cudaMemcpyAsync(spins, d_spins, spin_bytes, cudaMemcpyDeviceToHost, st), "D2H spins");
  OJ_CK(cudaEventRecord(ctx->ev[3], st), "event");
  if (!devp || stats) OJ_CK(cudaStreamSynchronize(st), "run");
  if (stats) {
    stats->kernel = (int32_t)(OJ_KERNEL_SWENDSEN_WANG >> OJ_KERNEL_SHIFT);
    stats->launches = launches;
    stats->sweeps = S;
    stats->attempts = (double)R * n * (double)S;
    stats->threads = 512;
    stats->accepted = -1.0;
    stats->field_drift = -1.0;
    cudaEventElapsedTime(&stats->anneal_ms, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&stats->total_ms, ctx->ev[0], ctx->ev[3]);
  }
  return OJ_OK;
}

}  // extern "C"
