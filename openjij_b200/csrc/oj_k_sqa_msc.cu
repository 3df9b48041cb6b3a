// Bit-packed SQA sweep for regular graphs with couplings +-c and h = 0: one
// 32-bit word holds the T <= 32 Trotter slices of one site of one replica
// (bit t set iff s_{i,t} = -1).
//
// The update order is the colour-class SQA order (oj_k_colour.cu, after the
// reference's single_spin_flip.hpp:163-192): slice groups {even t < T - T%2},
// {odd t}, {T-1 if T odd}, and inside a group the colour classes of the
// spatial graph.  A group is a bit mask, so one word operation decides every
// slice of the group at once; the Trotter neighbours t+-1 are the word
// rotated by one bit inside T bits.  For each slice bit:
//   u  = unsatisfied spatial bonds (bit-sliced count over the d neighbours),
//        dE_sp = 2c(d - 2u);
//   k  = Trotter neighbours aligned with it, dE_trot = 4 - 4k;
//   dE = a*dE_sp + B*dE_trot  (FP32 on the host, a = s*beta/T,
//        B = 0.5*log(tanh(beta*Gamma*(1-s)/T)), single_spin_flip.hpp:147-148,216-217).
// The (u, k) class of a bit selects its acceptance: always when dE <= 0, never
// when dE is NaN or +inf, else when the 32-bit uniform U < floor(exp(-dE)*2^32),
// compared one bit level at a time with the Philox words
//   W_l(r, k, i, group) = Philox(i, k, r, (l>>2)<<16 | group<<8 | 0xC3)[l&3].
// One CTA per replica keeps its n words and the neighbour tables in shared
// memory for the whole schedule.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kSqaMscThreads = 512;

struct SqaMscArgs {
  const int32_t* order;   // sites sorted by colour
  const int32_t* coff;    // [ncol+1]
  const uint16_t* nbr;    // [n][D] neighbour sites
  const uint16_t* jm;     // [n] bit l: J(i, nbr l) > 0
  int n, ncol, T;
  uint32_t* words;        // [R][n]
  const uint32_t* thr;    // [nsweeps][(D+1)*3] threshold of class u*3+k
  const uint32_t* mode;   // [nsweeps][2]: always-mask, live-mask over classes
  int64_t nsweeps;
  ojd::Keys keys;
  uint32_t sweep0, rep0;
  unsigned long long* flips;  // accepted-flip counter, or null
};

template <int D>
__device__ __forceinline__ uint32_t sqa_site(uint32_t w, const uint32_t* __restrict__ Wsh,
                                             const uint16_t* __restrict__ nb, uint32_t jmk, uint32_t gmask,
                                             uint32_t tmask, int T, const uint32_t (&th)[(D + 1) * 3],
                                             uint32_t always, uint32_t live, uint32_t site, uint32_t sweep,
                                             uint32_t rep, uint32_t grp, const ojd::Keys& K) {
  constexpr int NB = D <= 1 ? 1 : (D <= 3 ? 2 : (D <= 7 ? 3 : 4));
  constexpr int NC = (D + 1) * 3;
  uint32_t cnt[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) cnt[b] = 0u;
#pragma unroll
  for (int l = 0; l < D; ++l) {
    uint32_t x = w ^ Wsh[nb[l]] ^ (0u - ((jmk >> l) & 1u));
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const uint32_t t = cnt[b] & x;
      cnt[b] ^= x;
      x = t;
    }
  }
  // Trotter neighbours: bit t of `up` is slice t+1, of `dn` slice t-1 (periodic in T)
  const uint32_t up = ((w >> 1) | (w << (T - 1))) & tmask;
  const uint32_t dn = ((w << 1) | (w >> (T - 1))) & tmask;
  const uint32_t al_up = ~(w ^ up), al_dn = ~(w ^ dn);
  const uint32_t k1 = al_up & al_dn;          // both aligned (k = 2)
  const uint32_t k0 = al_up ^ al_dn;          // exactly one (k = 1)
  const uint32_t kz = ~(al_up | al_dn);       // none (k = 0)
  uint32_t cls[NC];
  uint32_t flip = 0u, pending = 0u;
#pragma unroll
  for (int u = 0; u <= D; ++u) {
    uint32_t mu = 0xFFFFFFFFu;
#pragma unroll
    for (int b = 0; b < NB; ++b) mu &= ((u >> b) & 1) ? cnt[b] : ~cnt[b];
    mu &= gmask;
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
      const int c = u * 3 + kk;
      const uint32_t m = mu & (kk == 0 ? kz : (kk == 1 ? k0 : k1));
      if ((always >> c) & 1u) flip |= m;
      cls[c] = ((live >> c) & 1u) ? m : 0u;
      pending |= cls[c];
    }
  }
  uint32_t lt = 0u;
#pragma unroll 1
  for (int q = 0; q < 8 && pending; ++q) {
    const ojd::u4 r = ojd::philox(site, sweep, rep, ((uint32_t)q << 16) | (grp << 8) | ojd::TAG_SQA_MSC, K);
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int bitpos = 31 - (4 * q + l);
      const uint32_t wl = ojd::pick(r, l);
      uint32_t pm = 0u;
#pragma unroll
      for (int c = 0; c < NC; ++c) pm |= cls[c] & (0u - ((th[c] >> bitpos) & 1u));
      lt |= pending & pm & ~wl;
      pending &= ~(pm ^ wl);
    }
  }
  return w ^ ((flip | lt) & gmask);
}

template <int D>
__global__ void __launch_bounds__(kSqaMscThreads) sqa_msc_kernel(SqaMscArgs a) {
  extern __shared__ __align__(16) uint32_t sh[];
  constexpr int NC = (D + 1) * 3;
  const int r = blockIdx.x;
  const int n = a.n;
  uint32_t* W = sh;                                                  // [n]
  uint16_t* nbr = reinterpret_cast<uint16_t*>(W + n);               // [n][D]
  uint16_t* jm = nbr + (size_t)n * D;                                // [n]
  uint32_t* gw = a.words + (size_t)r * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    W[i] = gw[i];
    jm[i] = a.jm[i];
  }
  for (int e = threadIdx.x; e < n * D; e += blockDim.x) nbr[e] = a.nbr[e];
  const int T = a.T;
  const uint32_t tmask = T >= 32 ? 0xFFFFFFFFu : ((1u << T) - 1u);
  const int upper = (T & 1) ? T - 1 : T;
  uint32_t gm0 = 0u, gm1 = 0u;
  for (int t = 0; t < upper; t += 2) gm0 |= 1u << t;
  for (int t = 1; t < T; t += 2) gm1 |= 1u << t;
  const uint32_t gm2 = (T & 1) ? (1u << (T - 1)) : 0u;
  const uint32_t rep = a.rep0 + (uint32_t)r;
  unsigned long long nflip = 0;
  __syncthreads();
  for (int64_t k = 0; k < a.nsweeps; ++k) {
    uint32_t th[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) th[c] = __ldg(a.thr + (size_t)k * NC + c);
    const uint32_t always = __ldg(a.mode + 2 * k), live = __ldg(a.mode + 2 * k + 1);
    const uint32_t kk = a.sweep0 + (uint32_t)k;
    for (int grp = 0; grp < 3; ++grp) {
      const uint32_t gmask = grp == 0 ? gm0 : (grp == 1 ? gm1 : gm2);
      if (gmask == 0u) continue;
      for (int c = 0; c < a.ncol; ++c) {
        const int lo = a.coff[c], hi = a.coff[c + 1];
        for (int idx = lo + threadIdx.x; idx < hi; idx += blockDim.x) {
          const int i = a.order[idx];
          const uint32_t w0 = W[i];
          const uint32_t w1 = sqa_site<D>(w0, W, nbr + (size_t)i * D, jm[i], gmask, tmask, T, th, always, live,
                                          (uint32_t)i, kk, rep, (uint32_t)grp, a.keys);
          W[i] = w1;
          nflip += __popc(w1 ^ w0);
        }
        __syncthreads();
      }
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) gw[i] = W[i];
  ojd::add_flips(a.flips, nflip);
}

// [R][T][n] int8 <-> [R][n] words (bit t = slice t, set iff s = -1)
__global__ void sqa_pack_kernel(const int8_t* __restrict__ spins, int R, int T, int n, uint32_t* __restrict__ words) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (i >= n) return;
  uint32_t w = 0;
  for (int t = 0; t < T; ++t)
    if (spins[((size_t)r * T + t) * n + i] < 0) w |= 1u << t;
  words[(size_t)r * n + i] = w;
}

__global__ void sqa_unpack_kernel(const uint32_t* __restrict__ words, int R, int T, int n, int8_t* __restrict__ spins) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (i >= n) return;
  const uint32_t w = words[(size_t)r * n + i];
  for (int t = 0; t < T; ++t) spins[((size_t)r * T + t) * n + i] = ((w >> t) & 1u) ? (int8_t)-1 : (int8_t)1;
}

size_t sqa_msc_smem(int n, int D) { return (size_t)n * 4 + (size_t)n * D * 2 + (size_t)n * 2 + 16; }

template <int D>
cudaError_t launch_d(const SqaMscArgs& a, int R, cudaStream_t st) {
  const size_t smem = sqa_msc_smem(a.n, D);
  if (smem > 220 * 1024) return cudaErrorInvalidValue;
  auto kern = sqa_msc_kernel<D>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<R, kSqaMscThreads, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

bool sqa_msc_fits(const oj_graph* g) {
  return g->n <= 65535 && g->info.max_degree >= 1 && g->info.max_degree <= 8 &&
         sqa_msc_smem(g->n, g->info.max_degree) <= 220 * 1024;
}

cudaError_t sqa_msc_prepare(oj_graph* g) {
  if (g->sqa_nbr.ptr) return cudaSuccess;
  const int n = g->n, D = g->info.max_degree;
  std::vector<uint16_t> nbr((size_t)n * D), jm(n, 0);
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int q = g->rp[i]; q < g->rp[i + 1]; ++q, ++l) {
      nbr[(size_t)i * D + l] = (uint16_t)g->ci[q];
      if (g->val64[q] > 0) jm[i] |= (uint16_t)(1u << l);
    }
  }
  cudaError_t e = g->sqa_nbr.ensure(std::max<size_t>(nbr.size() * 2, 16));
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpy(g->sqa_nbr.ptr, nbr.data(), nbr.size() * 2, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  if ((e = g->sqa_jm.ensure(std::max<size_t>(jm.size() * 2, 16))) != cudaSuccess) return e;
  return cudaMemcpy(g->sqa_jm.ptr, jm.data(), jm.size() * 2, cudaMemcpyHostToDevice);
}

cudaError_t launch_sqa_msc(const oj_graph* g, int R, int T, uint32_t* words, const uint32_t* thr,
                           const uint32_t* mode, int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches) {
  SqaMscArgs a;
  a.order = g->d_order.as<int32_t>();
  a.coff = g->d_coff.as<int32_t>();
  a.nbr = g->sqa_nbr.as<uint16_t>();
  a.jm = g->sqa_jm.as<uint16_t>();
  a.n = g->n;
  a.ncol = g->info.num_colours;
  a.T = T;
  a.words = words;
  a.thr = thr;
  a.mode = mode;
  a.nsweeps = nsweeps;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.rep0 = rb.rep0;
  a.flips = rb.flips;
  if (launches) ++*launches;
  switch (g->info.max_degree) {
    case 1: return launch_d<1>(a, R, st);
    case 2: return launch_d<2>(a, R, st);
    case 3: return launch_d<3>(a, R, st);
    case 4: return launch_d<4>(a, R, st);
    case 5: return launch_d<5>(a, R, st);
    case 6: return launch_d<6>(a, R, st);
    case 7: return launch_d<7>(a, R, st);
    case 8: return launch_d<8>(a, R, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_sqa_pack(const int8_t* spins, int R, int T, int n, uint32_t* words, cudaStream_t st) {
  dim3 grid((n + 255) / 256, R);
  sqa_pack_kernel<<<grid, 256, 0, st>>>(spins, R, T, n, words);
  return cudaGetLastError();
}

cudaError_t launch_sqa_unpack(const uint32_t* words, int R, int T, int n, int8_t* spins, cudaStream_t st) {
  dim3 grid((n + 255) / 256, R);
  sqa_unpack_kernel<<<grid, 256, 0, st>>>(words, R, T, n, spins);
  return cudaGetLastError();
}

}  // namespace oj
