// Colour-class Metropolis kernels for arbitrary coupling graphs (FP32 fields
// gathered from the neighbour list), the FP64 energy kernel and the
// int8 <-> bit-packed conversion kernels.
//
// SA (reference: include/openjij/updater/single_spin_flip.hpp:66-95).  The
// reference visits sites 0..n-1 in order.  Here the sites are split into the
// classes of a greedy colouring of the coupling graph; sites of one class have
// no coupling between them, so a whole class is updated at once and classes
// are visited in order.  On a 2-colourable lattice this is the checkerboard
// sweep; on a complete graph every class is a single site and the order is the
// reference's.  Acceptance: dE <= 0, or beta*dE < -ln(u) (equivalent to
// exp(-beta*dE) > u, single_spin_flip.hpp:80-82).
//
// SQA (single_spin_flip.hpp:127-258): slice groups {even t < T - T%2}, {odd t},
// {T-1 if T odd} in that order as the reference's OpenMP loops, and inside a
// group the colour classes of the spatial graph.  dE = a*dE_sp + B*dE_trot with
// a = s*beta/T and B = 0.5*log(tanh(beta*Gamma*(1-s)/T)) precomputed per sweep;
// accept when dE < -ln(u) (single_spin_flip.hpp:240: dE < 0 || exp(-dE) > u).
#include <cuda_runtime.h>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kColourThreads = 256;
constexpr int kSmemBudget = 200 * 1024;

// One CTA per replica quad q (replicas 4q..4q+3); one thread per (site, quad):
// the four replicas share the neighbour loads and one Philox call.
template <bool SMEM>
__global__ void __launch_bounds__(kColourThreads)
    sa_colour_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                     const float* __restrict__ val, const float* __restrict__ h,
                     const int32_t* __restrict__ order, const int32_t* __restrict__ coff, int ncol,
                     int n, int R, int8_t* __restrict__ spins, const float* __restrict__ betas,
                     int64_t nsweeps, RngBase rb) {
  extern __shared__ int8_t sh[];
  const int q = blockIdx.x;
  const int r0 = 4 * q;
  const int nr = min(4, R - r0);
  int8_t* S = SMEM ? sh : spins + (size_t)r0 * n;
  unsigned long long nflip = 0;
  if (SMEM) {
    for (int idx = threadIdx.x; idx < 4 * n; idx += blockDim.x) {
      const int rl = idx / n;
      S[idx] = rl < nr ? spins[(size_t)r0 * n + idx] : (int8_t)1;
    }
    __syncthreads();
  }
  for (int64_t k = 0; k < nsweeps; ++k) {
    const float beta2 = 2.0f * betas[k];
    for (int c = 0; c < ncol; ++c) {
      const int lo = coff[c], hi = coff[c + 1];
      for (int idx = lo + threadIdx.x; idx < hi; idx += blockDim.x) {
        const int i = order[idx];
        const float hi_f = h[i];
        float f0 = hi_f, f1 = hi_f, f2 = hi_f, f3 = hi_f;
        const int p1 = rp[i + 1];
        for (int p = rp[i]; p < p1; ++p) {
          const int j = ci[p];
          const float v = val[p];
          f0 = __fadd_rn(f0, S[j] > 0 ? v : -v);
          if (nr > 1) f1 = __fadd_rn(f1, S[n + j] > 0 ? v : -v);
          if (nr > 2) f2 = __fadd_rn(f2, S[2 * n + j] > 0 ? v : -v);
          if (nr > 3) f3 = __fadd_rn(f3, S[3 * n + j] > 0 ? v : -v);
        }
        const ojd::u4 rnd = ojd::philox((uint32_t)i, rb.sweep0 + (uint32_t)k, (rb.rep0 >> 2) + (uint32_t)q,
                                        ojd::TAG_SA, rb.k0, rb.k1);
        const float fs[4] = {f0, f1, f2, f3};
#pragma unroll
        for (int rl = 0; rl < 4; ++rl) {
          if (rl < nr) {
            const int8_t si = S[rl * n + i];
            // beta*dE, dE = -+2 f, is (2 beta) f with the sign of -s_i (scaling
            // by 2 is exact); dE <= 0 accepts without a draw, and so does the
            // comparison, since -ln u > 0 and beta is finite and >= 0
            const float bf = __fmul_rn(beta2, fs[rl]);
            if ((si > 0 ? -bf : bf) < ojd::neglog(ojd::pick(rnd, rl))) {
              S[rl * n + i] = (int8_t)(-si);
              ++nflip;
            }
          }
        }
      }
      __syncthreads();
    }
  }
  if (SMEM) {
    for (int idx = threadIdx.x; idx < nr * n; idx += blockDim.x) spins[(size_t)r0 * n + idx] = S[idx];
  }
  ojd::add_flips(rb.flips, nflip);
}

constexpr int kSqaThreads = 512;

// One CTA per replica; one thread per (site, slice quad) of the active group.
template <bool SMEM>
__global__ void __launch_bounds__(kSqaThreads)
    sqa_colour_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                      const float* __restrict__ val, const float* __restrict__ h,
                      const int32_t* __restrict__ order, const int32_t* __restrict__ coff, int ncol,
                      int n, int T, int8_t* __restrict__ spins, const float2* __restrict__ coef,
                      int64_t nsweeps, RngBase rb) {
  extern __shared__ int8_t sh[];
  const int r = blockIdx.x;
  const size_t tn = (size_t)T * n;
  int8_t* S = SMEM ? sh : spins + (size_t)r * tn;
  unsigned long long nflip = 0;
  if (SMEM) {
    for (size_t idx = threadIdx.x; idx < tn; idx += blockDim.x) S[idx] = spins[(size_t)r * tn + idx];
    __syncthreads();
  }
  const int upper = (T & 1) ? T - 1 : T;
  const int nquad = (T + 7) >> 3;
  for (int64_t k = 0; k < nsweeps; ++k) {
    const float2 ab = coef[k];
    for (int grp = 0; grp < 3; ++grp) {
      if (grp == 2 && !(T & 1)) break;
      const int par = grp == 1 ? 1 : 0;
      const int tmin = grp == 2 ? T - 1 : 0;
      const int tmax = grp == 0 ? upper : T;  // exclusive
      for (int c = 0; c < ncol; ++c) {
        const int lo = coff[c], cnt = coff[c + 1] - lo;
        const int items = cnt * nquad;
        for (int it = threadIdx.x; it < items; it += blockDim.x) {
          const int a = it / cnt;
          const int i = order[lo + (it - a * cnt)];
          const int tq = 8 * a + par;
          if (tq + 6 < tmin || tq >= tmax) continue;
          const ojd::u4 rnd = ojd::philox((uint32_t)i, rb.sweep0 + (uint32_t)k, rb.rep0 + (uint32_t)r,
                                          ((uint32_t)a << 9) | ((uint32_t)par << 8) | ojd::TAG_SQA,
                                          rb.k0, rb.k1);
          const float hi_f = h[i];
          const int p0 = rp[i], p1 = rp[i + 1];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int t = tq + 2 * j;
            if (t < tmin || t >= tmax) continue;
            int8_t* St = S + (size_t)t * n;
            float f = hi_f;
            for (int p = p0; p < p1; ++p) {
              const float v = val[p];
              f = __fadd_rn(f, St[ci[p]] > 0 ? v : -v);
            }
            const int8_t si = St[i];
            const float dEsp = si > 0 ? -2.0f * f : 2.0f * f;
            const int tp = t + 1 == T ? 0 : t + 1;
            const int tm = t == 0 ? T - 1 : t - 1;
            const int ssum = (int)S[(size_t)tp * n + i] + (int)S[(size_t)tm * n + i];
            const float dEtrot = (float)(-2 * (int)si * ssum);
            const float dE = __fadd_rn(__fmul_rn(ab.x, dEsp), __fmul_rn(ab.y, dEtrot));
            const float L = ojd::neglog(ojd::pick(rnd, j));
            if (dE < L) {
              St[i] = (int8_t)(-si);
              ++nflip;
            }
          }
        }
        __syncthreads();
      }
    }
  }
  if (SMEM) {
    for (size_t idx = threadIdx.x; idx < tn; idx += blockDim.x) spins[(size_t)r * tn + idx] = S[idx];
  }
  ojd::add_flips(rb.flips, nflip);
}

// FP64 energies of 32 spin vectors per CTA:
// E = sum_{i<j} J_ij s_i s_j + sum_i h_i s_i  (= dense.hpp:176-192).
// The 32 vectors' spins at a site are packed into one word (bit r set iff
// s = -1), so every coupling is read once for 32 vectors and s_i s_j is the
// xor of two words.  Partial sums are combined in a fixed order, so the result
// does not depend on timing.
constexpr int kEnergyThreads = 256;
__global__ void __launch_bounds__(kEnergyThreads)
    energy_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                  const double* __restrict__ val, const double* __restrict__ h, int n, int count,
                  const int8_t* __restrict__ spins, double* __restrict__ out) {
  // CTA (x, y): replicas 32x .. 32x + 31, sites [y n / Y, (y + 1) n / Y); with
  // Y > 1 the sums go to out[y * count + replica], summed in order of y by
  // energy_sum_kernel (no dependence on timing)
  extern __shared__ uint32_t wsh[];  // [n] words, then [8][32] partial sums
  const int v0 = blockIdx.x * 32;
  const int ilo = (int)(((int64_t)blockIdx.y * n) / gridDim.y);
  const int ihi = (int)(((int64_t)(blockIdx.y + 1) * n) / gridDim.y);
  const int nv = min(32, count - v0);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    uint32_t w = 0;
    for (int r = 0; r < nv; ++r)
      if (spins[(size_t)(v0 + r) * n + i] < 0) w |= 1u << r;
    wsh[i] = w;
  }
  __syncthreads();
  double acc[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) acc[r] = 0.0;
  for (int i = ilo + threadIdx.x; i < ihi; i += blockDim.x) {
    const uint32_t wi = wsh[i];
    const double hi = h[i];
#pragma unroll
    for (int r = 0; r < 32; ++r) acc[r] += ((wi >> r) & 1u) ? -hi : hi;
    const int p1 = rp[i + 1];
    for (int p = rp[i]; p < p1; ++p) {
      const int j = ci[p];
      if (j <= i) continue;
      const uint32_t x = wi ^ wsh[j];
      const double v = val[p];
#pragma unroll
      for (int r = 0; r < 32; ++r) acc[r] += ((x >> r) & 1u) ? -v : v;
    }
  }
  // warp reduction, then warps in order
  double* part = reinterpret_cast<double*>(wsh + ((n + 1) & ~1));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    double x = acc[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) part[warp * 32 + r] = x;
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double t = 0.0;
    for (int w = 0; w < kEnergyThreads / 32; ++w) t += part[w * 32 + threadIdx.x];
    out[(size_t)blockIdx.y * count + v0 + threadIdx.x] = t;
  }
}

// First slice of minimum energy per replica (get_solution.hpp:69-76, strict <).
__global__ void best_slice_kernel(const double* __restrict__ e, int R, int T, int32_t* __restrict__ best) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  int b = 0;
  double m = e[(size_t)r * T];
  for (int t = 1; t < T; ++t) {
    const double v = e[(size_t)r * T + t];
    if (v < m) {
      m = v;
      b = t;
    }
  }
  best[r] = b;
}

// int8 [R][n] -> words [ceil(R/32)][n]; bit j of word (g, i) set iff replica
// 32g+j has s_i = -1.  Replicas past R read as +1.
__global__ void pack_kernel(const int8_t* __restrict__ spins, int R, int n, uint32_t* __restrict__ words) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (i >= n) return;
  uint32_t w = 0;
  for (int j = 0; j < 32; ++j) {
    const int r = 32 * g + j;
    if (r < R && spins[(size_t)r * n + i] < 0) w |= 1u << j;
  }
  words[(size_t)g * n + i] = w;
}

__global__ void unpack_kernel(const uint32_t* __restrict__ words, int R, int n, int8_t* __restrict__ spins) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (i >= n) return;
  const uint32_t w = words[(size_t)g * n + i];
  for (int j = 0; j < 32; ++j) {
    const int r = 32 * g + j;
    if (r < R) spins[(size_t)r * n + i] = ((w >> j) & 1u) ? (int8_t)-1 : (int8_t)1;
  }
}

}  // namespace

int sa_colour_max_smem_sites() { return kSmemBudget / 4; }

cudaError_t launch_sa_colour(const oj_graph* g, int R, int8_t* spins, const float* betas,
                             int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches) {
  const int quads = (R + 3) / 4;
  const size_t smem = (size_t)4 * g->n;
  const bool use_smem = smem <= (size_t)kSmemBudget;
  if (use_smem) {
    auto kern = sa_colour_kernel<true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<quads, kColourThreads, smem, st>>>(g->d_rp.as<int32_t>(), g->d_ci.as<int32_t>(),
                                             g->d_val.as<float>(), g->d_h.as<float>(),
                                             g->d_order.as<int32_t>(), g->d_coff.as<int32_t>(),
                                             g->info.num_colours, g->n, R, spins, betas, nsweeps, rb);
  } else {
    sa_colour_kernel<false><<<quads, kColourThreads, 0, st>>>(
        g->d_rp.as<int32_t>(), g->d_ci.as<int32_t>(), g->d_val.as<float>(), g->d_h.as<float>(),
        g->d_order.as<int32_t>(), g->d_coff.as<int32_t>(), g->info.num_colours, g->n, R, spins,
        betas, nsweeps, rb);
  }
  if (launches) ++*launches;
  return cudaGetLastError();
}

cudaError_t launch_sqa_colour(const oj_graph* g, int R, int T, int8_t* spins, const float2* coef,
                              int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches) {
  const size_t smem = (size_t)T * g->n;
  const bool use_smem = smem <= (size_t)kSmemBudget;
  if (use_smem) {
    auto kern = sqa_colour_kernel<true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<R, kSqaThreads, smem, st>>>(g->d_rp.as<int32_t>(), g->d_ci.as<int32_t>(),
                                        g->d_val.as<float>(), g->d_h.as<float>(),
                                        g->d_order.as<int32_t>(), g->d_coff.as<int32_t>(),
                                        g->info.num_colours, g->n, T, spins, coef, nsweeps, rb);
  } else {
    sqa_colour_kernel<false><<<R, kSqaThreads, 0, st>>>(
        g->d_rp.as<int32_t>(), g->d_ci.as<int32_t>(), g->d_val.as<float>(), g->d_h.as<float>(),
        g->d_order.as<int32_t>(), g->d_coff.as<int32_t>(), g->info.num_colours, g->n, T, spins,
        coef, nsweeps, rb);
  }
  if (launches) ++*launches;
  return cudaGetLastError();
}

// out[v] = sum over y of parts[y * count + v], y in order.
__global__ void energy_sum_kernel(const double* __restrict__ parts, int nsplit, int count, double* __restrict__ out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= count) return;
  double t = 0.0;
  for (int y = 0; y < nsplit; ++y) t += parts[(size_t)y * count + v];
  out[v] = t;
}

int energy_splits(const oj_graph* g, int count, int sm_count) {
  // sites split over CTAs until the grid covers the SMs twice (at least 256
  // sites a CTA)
  const int groups = (count + 31) / 32;
  int k = 1;
  while (k < 16 && groups * k < 2 * sm_count && g->n / (2 * k) >= 256) k *= 2;
  return k;
}

cudaError_t launch_energy(const oj_graph* g, int count, const int8_t* spins, double* out, cudaStream_t st,
                          int nsplit, double* parts) {
  if (count <= 0) return cudaSuccess;
  if (nsplit < 1 || (nsplit > 1 && !parts)) return cudaErrorInvalidValue;
  const size_t smem = (size_t)((g->n + 1) & ~1) * 4 + (kEnergyThreads / 32) * 32 * 8;
  auto kern = energy_kernel;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<dim3((count + 31) / 32, nsplit), kEnergyThreads, smem, st>>>(
      g->d_rp.as<int32_t>(), g->d_ci.as<int32_t>(), g->d_val64.as<double>(), g->d_h64.as<double>(), g->n, count,
      spins, nsplit > 1 ? parts : out);
  if (nsplit > 1) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    energy_sum_kernel<<<(count + 255) / 256, 256, 0, st>>>(parts, nsplit, count, out);
  }
  return cudaGetLastError();
}

cudaError_t launch_best_slice(const double* energies, int R, int T, int32_t* best, cudaStream_t st) {
  best_slice_kernel<<<(R + 127) / 128, 128, 0, st>>>(energies, R, T, best);
  return cudaGetLastError();
}

cudaError_t launch_pack(const int8_t* spins, int R, int n, uint32_t* words, cudaStream_t st) {
  dim3 grid((n + 255) / 256, (R + 31) / 32);
  pack_kernel<<<grid, 256, 0, st>>>(spins, R, n, words);
  return cudaGetLastError();
}

cudaError_t launch_unpack(const uint32_t* words, int R, int n, int8_t* spins, cudaStream_t st) {
  dim3 grid((n + 255) / 256, (R + 31) / 32);
  unpack_kernel<<<grid, 256, 0, st>>>(words, R, n, spins);
  return cudaGetLastError();
}

cudaError_t pack_preload() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, pack_kernel);
  return e != cudaSuccess ? e : cudaFuncGetAttributes(&fa, unpack_kernel);
}

}  // namespace oj
