// Single-flip energy changes of a few spin configurations and the smallest
// coupling magnitude: the statistics from which SASampler picks its beta range
// when beta_min / beta_max are not given (openjij/sampler/sa_sampler.py:876-965).
// The reference forms them with a dense (n+1)x(n+1) matrix product and a pass of
// np.abs over the whole augmented matrix; here one warp per site reads the
// graph's FP64 neighbour lists once (CSR on the device).
#include <cuda_runtime.h>

#include <cstdint>

#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kStatsThreads = 256;
constexpr int kStatsMaxK = 8;

__device__ __forceinline__ void min_bits(unsigned long long* out, double v) {
  // non-negative doubles order like their bit patterns
  atomicMin(out, (unsigned long long)__double_as_longlong(v));
}

// quad[i][c] = -2 s_i^c * sum_j J_ij s_j^c   (couplings only, j < n)
// lin[i][c]  = h_i s_i^c
// amin       = min over |J_ij|, |h_i| above thr
__global__ void __launch_bounds__(kStatsThreads) flip_stats_kernel(const int32_t* rp, const int32_t* ci,
                                                                   const double* val, const double* h, int n, int K,
                                                                   const int8_t* s, double thr, double* quad,
                                                                   double* lin, unsigned long long* amin) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (kStatsThreads / 32) + (threadIdx.x >> 5);
  if (i >= n) return;
  double acc[kStatsMaxK];
#pragma unroll
  for (int c = 0; c < kStatsMaxK; ++c) acc[c] = 0.0;
  double mn = __longlong_as_double(0x7FF0000000000000LL);
  for (int p = rp[i] + lane; p < rp[i + 1]; p += 32) {
    const double v = val[p];
    const int j = ci[p];
#pragma unroll
    for (int c = 0; c < kStatsMaxK; ++c)
      if (c < K) acc[c] = __fma_rn(v, (double)s[(size_t)j * K + c], acc[c]);
    const double a = fabs(v);
    if (a > thr && a < mn) mn = a;
  }
#pragma unroll
  for (int c = 0; c < kStatsMaxK; ++c)
    for (int o = 16; o > 0; o >>= 1) acc[c] = __dadd_rn(acc[c], __shfl_xor_sync(0xffffffffu, acc[c], o));
  for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  if (lane == 0) {
    const double hi = h[i];
    for (int c = 0; c < K; ++c) {
      const double si = (double)s[(size_t)i * K + c];
      quad[(size_t)i * K + c] = __dmul_rn(acc[c], -2.0 * si);
      lin[(size_t)i * K + c] = __dmul_rn(hi, si);
    }
    if (fabs(hi) > thr && fabs(hi) < mn) mn = fabs(hi);
    if (mn < __longlong_as_double(0x7FF0000000000000LL)) min_bits(amin, mn);
  }
}

// The same statistics for every instance of a batch, from its FP64 augmented
// matrices (row-major (n+1)^2 at j64off[k]); warp per (instance, row), rows
// 0..n so that the minimum sees the field row and the corner too.
__global__ void __launch_bounds__(kStatsThreads) batch_flip_stats_kernel(const double* J64, const int64_t* j64off,
                                                                         const int32_t* nn, const int64_t* soff,
                                                                         int K, const int8_t* s, double thr,
                                                                         double* quad, double* lin,
                                                                         unsigned long long* amin) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x;
  const int nk = nn[k];
  const int i = blockIdx.y * (kStatsThreads / 32) + (threadIdx.x >> 5);
  if (i > nk) return;
  const int64_t n1 = (int64_t)nk + 1;
  const double* row = J64 + j64off[k] + (int64_t)i * n1;
  const int8_t* sk = s + soff[k] * K;
  double acc[kStatsMaxK];
#pragma unroll
  for (int c = 0; c < kStatsMaxK; ++c) acc[c] = 0.0;
  double mn = __longlong_as_double(0x7FF0000000000000LL);
  for (int j = lane; j <= nk; j += 32) {
    const double v = row[j];
    if (i < nk && j < nk) {
#pragma unroll
      for (int c = 0; c < kStatsMaxK; ++c)
        if (c < K) acc[c] = __fma_rn(v, (double)sk[(size_t)j * K + c], acc[c]);
    }
    const double a = fabs(v);
    if (a > thr && a < mn) mn = a;
  }
#pragma unroll
  for (int c = 0; c < kStatsMaxK; ++c)
    for (int o = 16; o > 0; o >>= 1) acc[c] = __dadd_rn(acc[c], __shfl_xor_sync(0xffffffffu, acc[c], o));
  for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  if (lane == 0) {
    if (i < nk) {
      const double hi = row[nk];
      double* q = quad + (soff[k] + i) * K;
      double* l = lin + (soff[k] + i) * K;
      for (int c = 0; c < K; ++c) {
        const double si = (double)sk[(size_t)i * K + c];
        q[c] = __dmul_rn(acc[c], -2.0 * si);
        l[c] = __dmul_rn(hi, si);
      }
    }
    if (mn < __longlong_as_double(0x7FF0000000000000LL)) min_bits(amin + k, mn);
  }
}

}  // namespace

int flip_stats_max_k() { return kStatsMaxK; }

cudaError_t launch_batch_flip_stats(const oj_batch* b, int K, const int8_t* s, const int64_t* soff, double thr,
                                    double* quad, double* lin, unsigned long long* amin, cudaStream_t st) {
  if (K < 1 || K > kStatsMaxK) return cudaErrorInvalidValue;
  if (b->count == 0) return cudaSuccess;
  const int wpb = kStatsThreads / 32;
  const dim3 grid((unsigned)b->count, (unsigned)((b->max_n + 1 + wpb - 1) / wpb));
  batch_flip_stats_kernel<<<grid, kStatsThreads, 0, st>>>(b->d_J64.as<double>(), b->d_j64off.as<int64_t>(),
                                                          b->d_n.as<int32_t>(), soff, K, s, thr, quad, lin, amin);
  return cudaGetLastError();
}

cudaError_t launch_flip_stats(const oj_graph* g, int K, const int8_t* s, double thr, double* quad, double* lin,
                              unsigned long long* amin, cudaStream_t st) {
  if (K < 1 || K > kStatsMaxK) return cudaErrorInvalidValue;
  const int wpb = kStatsThreads / 32;
  flip_stats_kernel<<<(g->n + wpb - 1) / wpb, kStatsThreads, 0, st>>>(
      g->d_rp.as<int32_t>(), g->d_ci.as<int32_t>(), g->d_val64.as<double>(), g->d_h64.as<double>(), g->n, K, s, thr,
      quad, lin, amin);
  return cudaGetLastError();
}

}  // namespace oj
