// Allocation-free entry point of the bit-packed SA kernel.
//
// Some callers cannot call cudaMalloc while they run: an application whose
// device memory is already reserved by another framework's allocator (a
// caching allocator that owns the free memory), or latency-sensitive code
// that cannot accept cudaMalloc's implicit device synchronisation.  For them
// oj_sa_run_bitpacked_noalloc runs the same kernel as oj_sa_run's bit-packed
// path, but keeps every piece of per-call scratch (the 32-replica words and
// the per-sweep acceptance thresholds) in one fixed, file-scope device array
// instead of context workspace allocated on demand.
//
// The array is kNoAllocScratchBytes (16 MiB).  CUDA loads a library's device
// code and its __device__ arrays lazily, so oj_ctx_create does the set-up with
// the context's device current: it looks up the array's device address (which
// places the array on the device) and loads the kernels this entry point
// launches.  From then on the device holds the array until the process exits,
// and a call allocates nothing.  All calls share the array, and each call
// overwrites what it uses (the words are rebuilt from the caller's spins, the
// thresholds rewritten for the call's schedule), so nothing has to start at
// zero; two calls that overlap on the GPU (different streams or contexts on
// one device) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "oj_internal.h"

namespace oj {
namespace {

constexpr size_t kNoAllocScratchBytes = 16u << 20;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kMscMaxDegreeForNoAlloc = 8;  // the bit-packed kernel's degree limit

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array, looked up once per device with that
// device current (in host code the array's name is only a host-side handle).
std::mutex g_scratch_mu;
void* g_scratch_ptr[kNoAllocMaxDevices] = {};

// The device address recorded by noalloc_prepare, or null.
void* scratch_address(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  return g_scratch_ptr[device];
}

// thr = floor(exp(-beta*2c*m) * 2^32), m = 1..D; always bit m when the
// probability is 1 — the same host arithmetic as oj_sa_run's bit-packed path.
void threshold_row(float beta, double c, int D, uint32_t* thr, uint32_t* always) {
  *always = 0u;
  thr[0] = 0u;
  for (int m = 1; m <= D; ++m) {
    const double p = std::exp(-(double)beta * 2.0 * c * (double)m);
    const double t = std::floor(std::ldexp(p, 32));
    uint32_t v;
    if (p >= 1.0) {
      *always |= 1u << m;
      v = 0xFFFFFFFFu;
    } else {
      v = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
    }
    thr[m] = v;
  }
}

}  // namespace

// Once per device, with `device` current (oj_ctx_create).
cudaError_t noalloc_prepare(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return e;
      g_scratch_ptr[device] = p;
    }
  }
  const cudaError_t e = pack_preload();
  return e != cudaSuccess ? e : msc_preload();
}

}  // namespace oj

using namespace oj;

extern "C" oj_status oj_sa_run_bitpacked_noalloc(oj_ctx* ctx, const oj_graph* g, int32_t R, int8_t* spins,
                                                 const double* betas, const int32_t* mcs, int32_t num_sched,
                                                 uint64_t seed, int64_t first_sweep, int64_t replica_offset) {
  if (!ctx || !g || R < 0 || num_sched < 0 || (num_sched > 0 && (!betas || !mcs))) {
    if (ctx) ctx->last_error = "null argument or negative size";
    return OJ_ERR_ARG;
  }
  if (g->device != ctx->device) {
    ctx->last_error = "graph belongs to another device";
    return OJ_ERR_ARG;
  }
  const int n = g->n;
  if (R == 0 || n == 0) return OJ_OK;
  if (!spins) {
    ctx->last_error = "null spins";
    return OJ_ERR_ARG;
  }
  const oj_graph_info& inf = g->info;
  if (!(inf.bimodal && g->regular && inf.max_degree >= 1 && inf.max_degree <= msc_max_degree() &&
        inf.max_degree <= kMscMaxDegreeForNoAlloc)) {
    ctx->last_error = "bit-packed kernel needs a regular graph with couplings +-c (degree <= 8) and h = 0";
    return OJ_ERR_UNSUPPORTED;
  }
  if (!g->msc) {
    ctx->last_error = "the graph has no bit-packed site partition yet: run oj_sa_run once on it";
    return OJ_ERR_UNSUPPORTED;
  }
  if (first_sweep < 0 || first_sweep > 0xFFFFFFFFll || replica_offset < 0 || replica_offset > 0xFFFFFFFFll ||
      (replica_offset & 31) != 0) {
    ctx->last_error = "first_sweep / replica_offset out of range (replica_offset: a multiple of 32)";
    return OJ_ERR_ARG;
  }
  int64_t S = 0;
  for (int32_t k = 0; k < num_sched; ++k) {
    if (mcs[k] < 0 || !(betas[k] >= 0.0) || std::isinf(betas[k])) {
      ctx->last_error = "one_mc_step must be >= 0 and beta finite and >= 0";
      return OJ_ERR_ARG;
    }
    S += mcs[k];
  }
  const int D = inf.max_degree;
  const int G = (R + 31) / 32;
  const size_t words_bytes = (size_t)G * n * 4;
  const size_t thr_bytes = (size_t)S * (D + 1) * 4;
  const size_t alw_bytes = (size_t)S * 4;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t need = al(words_bytes) + al(thr_bytes) + al(alw_bytes);
  if (need > kNoAllocScratchBytes) {
    ctx->last_error = "replicas x spins x sweeps exceed the 16 MiB fixed scratch of the allocation-free entry point";
    return OJ_ERR_ARG;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != ctx->device) cudaSetDevice(ctx->device);
  auto fail = [&](cudaError_t e, const char* where) {
    ctx->last_error = std::string(where) + ": " + cudaGetErrorString(e);
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    return OJ_ERR_CUDA;
  };
  // the thresholds are uploaded from a stack buffer, which a captured copy
  // would read again at every replay, after this call has returned
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    ctx->last_error = "the context's stream is being captured; the allocation-free entry point cannot be captured";
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    return OJ_ERR_UNSUPPORTED;
  }
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, spins) != cudaSuccess ||
      !(pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged)) {
    cudaGetLastError();
    ctx->last_error = "spins must be device memory";
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    return OJ_ERR_ARG;
  }
  if (pa.device != ctx->device) {
    ctx->last_error = "spins are on another device than the context's";
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    return OJ_ERR_ARG;
  }
  void* base = scratch_address(ctx->device);
  if (!base) {
    ctx->last_error = ctx->noalloc_error.empty() ? "the allocation-free entry point was not set up on this device"
                                                 : ctx->noalloc_error;
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    return OJ_ERR_CUDA;
  }
  cudaError_t e = cudaSuccess;
  uint32_t* d_words = static_cast<uint32_t*>(base);
  uint32_t* d_thr = reinterpret_cast<uint32_t*>(static_cast<char*>(base) + al(words_bytes));
  uint32_t* d_alw = reinterpret_cast<uint32_t*>(static_cast<char*>(base) + al(words_bytes) + al(thr_bytes));
  cudaStream_t st = ctx->stream;
  // thresholds, a chunk of sweeps at a time through a stack buffer (a copy
  // from pageable memory is staged before cudaMemcpyAsync returns)
  constexpr int kChunk = 256;
  uint32_t thr_buf[kChunk * (kMscMaxDegreeForNoAlloc + 1)];
  uint32_t alw_buf[kChunk];
  int64_t k = 0, filled = 0;
  for (int32_t e_idx = 0; e_idx < num_sched; ++e_idx) {
    const float bf = (float)betas[e_idx];
    for (int32_t m = 0; m < mcs[e_idx]; ++m) {
      threshold_row(bf, inf.coupling_abs, D, thr_buf + filled * (D + 1), alw_buf + filled);
      ++filled;
      if (filled == kChunk) {
        if ((e = cudaMemcpyAsync(d_thr + k * (D + 1), thr_buf, (size_t)filled * (D + 1) * 4, cudaMemcpyHostToDevice, st)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(d_alw + k, alw_buf, (size_t)filled * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess)
          return fail(e, "threshold upload");
        k += filled;
        filled = 0;
      }
    }
  }
  if (filled > 0) {
    if ((e = cudaMemcpyAsync(d_thr + k * (D + 1), thr_buf, (size_t)filled * (D + 1) * 4, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(d_alw + k, alw_buf, (size_t)filled * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return fail(e, "threshold upload");
  }
  RngBase rb;
  rb.k0 = (uint32_t)seed;
  rb.k1 = (uint32_t)(seed >> 32);
  rb.sweep0 = (uint32_t)first_sweep;
  rb.rep0 = (uint32_t)replica_offset;
  if ((e = launch_pack(spins, R, n, d_words, st)) != cudaSuccess) return fail(e, "pack");
  if (S > 0 && (e = launch_sa_msc(g, G, d_words, d_thr, d_alw, S, rb, st, nullptr)) != cudaSuccess)
    return fail(e, "sa bit-packed kernel");
  if ((e = launch_unpack(d_words, R, n, spins, st)) != cudaSuccess) return fail(e, "unpack");
  if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  return OJ_OK;
}
