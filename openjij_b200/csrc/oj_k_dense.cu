// Plain sequential dense SA: one warp per replica, FP32 local fields in shared
// memory, J rows (FP32, row-major, symmetric) read from L2 on every accepted
// flip.  Update order and acceptance are the reference's
// (include/openjij/updater/single_spin_flip.hpp:66-95): sites 0..n-1 in order,
// accept when dE <= 0 or beta*dE < -ln(u); on a flip every field moves by
// -2 s_i J_ij (the reference's dE += 4 s_i J_ij s_j, classical_ising.hpp:87-90).
#include <cuda_runtime.h>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

__global__ void __launch_bounds__(128)
    sa_dense_plain_kernel(const float* __restrict__ J, const float* __restrict__ h, int n, int R,
                          int8_t* __restrict__ spins, const float* __restrict__ betas,
                          int64_t nsweeps, RngBase rb, int warps_per_cta) {
  extern __shared__ float shf[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * warps_per_cta + warp;
  if (r >= R) return;  // no block-wide barriers below
  float* f = shf + (size_t)warp * n;
  int8_t* s = reinterpret_cast<int8_t*>(shf + (size_t)warps_per_cta * n) + (size_t)warp * n;
  int8_t* gs = spins + (size_t)r * n;
  for (int j = lane; j < n; j += 32) s[j] = gs[j];
  __syncwarp();
  // f_j = h_j + sum_k J_jk s_k, k ascending (J symmetric: column j of row k)
  for (int j = lane; j < n; j += 32) {
    float acc = h[j];
    for (int k = 0; k < n; ++k) {
      const float v = J[(size_t)k * n + j];
      acc = __fadd_rn(acc, s[k] > 0 ? v : -v);
    }
    f[j] = acc;
  }
  __syncwarp();
  const uint32_t rg = rb.rep0 + (uint32_t)r;  // global replica index
  unsigned long long nflip = 0;  // lane 0 counts the warp's flips
  const uint32_t c2 = rg >> 2;
  const int lane_r = (int)(rg & 3u);
  for (int64_t k = 0; k < nsweeps; ++k) {
    const float beta = betas[k];
    for (int i0 = 0; i0 < n; i0 += 32) {
      float L = 0.0f;
      if (i0 + lane < n)
        L = ojd::neglog(ojd::pick(
            ojd::philox((uint32_t)(i0 + lane), rb.sweep0 + (uint32_t)k, c2, ojd::TAG_SA, rb.k0, rb.k1), lane_r));
      const int cnt = min(32, n - i0);
      for (int ii = 0; ii < cnt; ++ii) {
        const int i = i0 + ii;
        const int8_t si = s[i];
        const float fi = f[i];
        const float dE = si > 0 ? -2.0f * fi : 2.0f * fi;
        const float Li = __shfl_sync(0xffffffffu, L, ii);
        if (dE <= 0.0f || __fmul_rn(beta, dE) < Li) {
          const float c = si > 0 ? -2.0f : 2.0f;
          const float* Ji = J + (size_t)i * n;
          for (int j = lane; j < n; j += 32) f[j] = __fadd_rn(f[j], __fmul_rn(c, Ji[j]));
          __syncwarp();
          if (lane == 0) {
            s[i] = (int8_t)(-si);
            ++nflip;
          }
          __syncwarp();
        }
      }
    }
  }
  __syncwarp();
  for (int j = lane; j < n; j += 32) gs[j] = s[j];
  ojd::add_flips(rb.flips, nflip);
}

}  // namespace

cudaError_t launch_sa_dense_plain(const oj_graph* g, int R, int8_t* spins, const float* betas,
                                  int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches) {
  const int n = g->n;
  const size_t per_warp = (size_t)n * 5;
  int wpc = 4;
  while (wpc > 1 && per_warp * wpc > 200 * 1024) wpc >>= 1;
  const size_t smem = per_warp * wpc + 16;
  if (smem > 220 * 1024) return cudaErrorInvalidValue;
  auto kern = sa_dense_plain_kernel;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int blocks = (R + wpc - 1) / wpc;
  kern<<<blocks, 32 * wpc, smem, st>>>(g->d_dense.as<float>(), g->d_h.as<float>(), n, R, spins, betas,
                                       nsweeps, rb, wpc);
  if (launches) ++*launches;
  return cudaGetLastError();
}

}  // namespace oj
