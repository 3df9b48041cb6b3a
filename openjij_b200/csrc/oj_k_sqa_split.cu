// Slice-split bit-packed SQA sweep for regular graphs with couplings +-c,
// h = 0 and an even number of Trotter slices T <= 64.
//
// Layout.  With H = T/2 and P the largest power of two with P*H <= 32, replica
// group g holds replicas P*g .. P*g+P-1.  Each site has two words: E (even
// slices) and O (odd slices); bit p*H + m of E is slice 2m of replica P*g + p,
// the same bit of O is slice 2m+1.  For even T the reference's update order
// (slice groups {even t}, {odd t}, each over the colour classes; the colour
// kernel restates single_spin_flip.hpp:163-192) becomes: an even phase updates
// E reading the Trotter neighbours 2m+1 and 2m-1 from O (O itself, and O
// rotated left by one bit inside every H-bit segment); an odd phase updates O
// from E (E, and E rotated right by one inside every segment).  Every bit of
// the updated word is an attempt.
//
// Acceptance per bit: u unsatisfied spatial bonds (dE_sp = 2c(d - 2u)), k
// aligned Trotter neighbours (dE_trot = 4 - 4k), class 3u + k; always when the
// class's FP32 dE <= 0, else U < floor(exp(-dE)*2^32) with U's bit (31 - l)
// taken from W_l = Philox(i, k, g, (l>>2)<<16 | q<<8 | TAG_SQA_SPLIT)[l & 3],
// compared one bit level at a time for all bits of the word.
//
// Parallel structure as the bit-packed SA kernel (oj_k_msc.cu): one thread
// block cluster per replica group, its CTAs splitting the sites into
// contiguous ranges with a halo of remote neighbours in shared memory (both
// halves), interior sites first, split cluster barrier, halo refresh of the
// previous phase's class out of the owners' shared memory.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <string>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace cg = cooperative_groups;

namespace oj {
namespace {

constexpr int kSplitMaxThreads = 512;
constexpr int kSplitDefaultThreads = 512;
constexpr int kSplitMaxCluster = 16;
constexpr size_t kSplitSmemBytes = 200 * 1024;

struct SplitArgs {
  const int32_t* gidx;
  const int32_t* coff;
  const int32_t* cb;
  const int32_t* hoff;
  const uint32_t* hsrc;
  const uint16_t* hdst;
  const uint16_t* nbr;
  const uint16_t* jm;
  int slots, nlocmax, hmax, ncol;
  int n;
  int H;                       // slices per half (T/2)
  uint32_t low, high, valid;   // first / last bit of every segment, used bits
  uint32_t* words;             // [G][2][n]: E then O
  const uint32_t* thr;         // [nsweeps][(D+1)*3]
  const uint32_t* mode;        // [nsweeps][2]: always, live
  int64_t nsweeps;
  ojd::Keys keys;
  uint32_t sweep0, group0;
  unsigned long long* flips;   // accepted-flip counter (every used bit of the words), or null
};

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Acceptance tables of one sweep, in shared memory.  For row l < 32 (bit
// 31 - l of the thresholds), Trotter alignment k (0..2 aligned neighbours) and
// unsatisfied-bond count u, word [l][k][u] is all ones when class c = 3u + k
// is live (compared against U) and bit 31 - l of its threshold is set; row 32
// marks the always-accepting classes, row 33 the live ones.  A word's class
// bits are then sets of its bits: with the count u held as NB bit planes, the
// table word of every bit is picked by a multiplexer tree over the planes (one
// three-input logic operation per node) instead of a pass over every class.
template <int D>
struct SplitTab {
  static constexpr int NB = D <= 1 ? 1 : (D <= 3 ? 2 : (D <= 7 ? 3 : 4));  // bit planes of u
  static constexpr int E = 1 << NB;                                        // words per (row, k)
  static constexpr int ROWS = 34;
  static constexpr int WORDS = ROWS * 3 * E;
};

// Per bit, the table word of its count u: a multiplexer tree over the planes.
template <int NB>
__device__ __forceinline__ uint32_t tab_pick(const uint32_t* __restrict__ t, const uint32_t (&cnt)[NB]) {
  constexpr int E = 1 << NB;
  uint32_t v[E];
  if constexpr (E >= 4) {
#pragma unroll
    for (int e = 0; e < E; e += 4) {
      const uint4 q4 = *reinterpret_cast<const uint4*>(t + e);
      v[e] = q4.x;
      v[e + 1] = q4.y;
      v[e + 2] = q4.z;
      v[e + 3] = q4.w;
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = t[e];
  }
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int e = 0; e < (E >> (b + 1)); ++e) v[e] = (cnt[b] & v[2 * e + 1]) | (~cnt[b] & v[2 * e]);
  return v[0];
}

// The bits of a word whose class has its table word set in `row` ([3][E]).
template <int D>
__device__ __forceinline__ uint32_t tab_eval(const uint32_t* __restrict__ row, uint32_t kk0, uint32_t kk1,
                                             uint32_t kk2, const uint32_t (&cnt)[SplitTab<D>::NB]) {
  constexpr int NB = SplitTab<D>::NB, E = SplitTab<D>::E;
  return (kk0 & tab_pick<NB>(row, cnt)) | (kk1 & tab_pick<NB>(row + E, cnt)) |
         (kk2 & tab_pick<NB>(row + 2 * E, cnt));
}

// Count planes that tell apart u = 0 .. ceil(D/2) - 1 (the uphill counts of a
// class with one aligned Trotter neighbour).
template <int D>
struct SplitLow {
  static constexpr int U = (D + 1) / 2;
  static constexpr int NB = U <= 2 ? 1 : (U <= 4 ? 2 : 3);
};

// Classes whose being live rules out the Trotter-dominated evaluation: every
// class with no aligned Trotter neighbour (k = 0) and the classes with one
// aligned neighbour and u >= ceil(D/2) (dE_sp <= 0 there).
template <int D>
__host__ __device__ constexpr uint32_t split_not_dominated_mask() {
  uint32_t m = 0u;
  for (int u = 0; u <= D; ++u) {
    m |= 1u << (3 * u);
    if (u >= SplitLow<D>::U) m |= 1u << (3 * u + 1);
  }
  return m;
}

// The row's bits for a sweep whose live classes all lie in
// {(u, 1) : u < ceil(D/2)} and {(u, 2)}: the value only matters on live bits
// (every other bit is neither pending nor compared), so the k = 0 group is
// dropped, a k = 1 bit takes its table word from the low count planes alone
// (u < ceil(D/2) on a live bit) and k = 2 from all of them.  Equal to tab_eval
// on every live bit.
template <int D>
__device__ __forceinline__ uint32_t tab_eval_dominated(const uint32_t* __restrict__ row, uint32_t kk1,
                                                       const uint32_t (&cnt)[SplitTab<D>::NB]) {
  constexpr int NB = SplitTab<D>::NB, E = SplitTab<D>::E, NBL = SplitLow<D>::NB;
  uint32_t low[NBL];
#pragma unroll
  for (int b = 0; b < NBL; ++b) low[b] = cnt[b];
  const uint32_t p1 = tab_pick<NBL>(row + E, low);
  const uint32_t p2 = tab_pick<NB>(row + 2 * E, cnt);
  return (kk1 & p1) | (~kk1 & p2);
}

// New value of word x (half q) of one site: nb are the neighbour slots in X
// (the array being updated), y the site's other half, tab the sweep's tables.
template <int D, bool DOM>
__device__ __forceinline__ uint32_t split_site(uint32_t x, const uint32_t* __restrict__ X,
                                               const uint16_t* __restrict__ nb, uint32_t jmk, uint32_t y,
                                               int q, const SplitArgs& a, const uint32_t* __restrict__ tab,
                                               uint32_t site, uint32_t sweep, uint32_t grp) {
  constexpr int NB = SplitTab<D>::NB, E = SplitTab<D>::E;
  uint32_t cnt[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) cnt[b] = 0u;
#pragma unroll
  for (int l = 0; l < D; ++l) {
    uint32_t v = x ^ X[nb[l]] ^ (0u - ((jmk >> l) & 1u));
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const uint32_t t = cnt[b] & v;
      cnt[b] ^= v;
      v = t;
    }
  }
  // even half: neighbours 2m+1 (y bit m) and 2m-1 (y bit m-1, cyclic in the segment)
  // odd half:  neighbours 2m   (y bit m) and 2m+2 (y bit m+1, cyclic in the segment)
  const uint32_t z = q == 0 ? (((y << 1) & ~a.low) | ((y >> (a.H - 1)) & a.low))
                            : (((y >> 1) & ~a.high) | ((y << (a.H - 1)) & a.high));
  const uint32_t al_y = ~(x ^ y), al_z = ~(x ^ z);
  const uint32_t kk2 = al_y & al_z, kk1 = al_y ^ al_z, kk0 = ~(al_y | al_z);
  const uint32_t flip = tab_eval<D>(tab + 32 * 3 * E, kk0, kk1, kk2, cnt) & a.valid;
  uint32_t pending = tab_eval<D>(tab + 33 * 3 * E, kk0, kk1, kk2, cnt) & a.valid;
  uint32_t lt = 0u;
#pragma unroll 1
  for (int qq = 0; qq < 8; ++qq) {
    if (!pending) break;
    const ojd::u4 r =
        ojd::philox(site, sweep, grp, ((uint32_t)qq << 16) | ((uint32_t)q << 8) | ojd::TAG_SQA_SPLIT, a.keys);
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const uint32_t wl = ojd::pick(r, l);
      const uint32_t* row = tab + (4 * qq + l) * 3 * E;
      uint32_t pm;
      if constexpr (DOM)
        pm = tab_eval_dominated<D>(row, kk1, cnt);
      else
        pm = tab_eval<D>(row, kk0, kk1, kk2, cnt);
      lt |= pending & pm & ~wl;
      pending &= ~(pm ^ wl);
    }
  }
  return x ^ flip ^ lt;
}

// Updates slots [lo, hi) of half X; returns the spins this thread flipped.
// DOM: the sweep's live classes allow tab_eval_dominated.
template <int D, bool DOM>
__device__ __forceinline__ uint32_t split_range(int lo, int hi, uint32_t* __restrict__ X,
                                                const uint32_t* __restrict__ Y, const int32_t* __restrict__ gid,
                                                const uint16_t* __restrict__ jm, const uint16_t* __restrict__ nbr,
                                                int q, const SplitArgs& a, const uint32_t* __restrict__ tab,
                                                uint32_t k, uint32_t g) {
  const int T = blockDim.x;
  uint32_t nf = 0u;
  if constexpr (D <= 4) {  // two independent sites per iteration
    for (int s = lo + threadIdx.x; s < hi; s += 2 * T) {
      const int s2 = s + T;
      const uint32_t x0 = X[s];
      const uint32_t v = split_site<D, DOM>(x0, X, nbr + (size_t)s * D, jm[s], Y[s], q, a, tab, (uint32_t)gid[s], k, g);
      if (s2 < hi) {
        const uint32_t x2 = X[s2];
        const uint32_t w2 =
            split_site<D, DOM>(x2, X, nbr + (size_t)s2 * D, jm[s2], Y[s2], q, a, tab, (uint32_t)gid[s2], k, g);
        X[s2] = w2;
        nf += __popc(w2 ^ x2);
      }
      X[s] = v;
      nf += __popc(v ^ x0);
    }
  } else {
    for (int s = lo + threadIdx.x; s < hi; s += T) {
      const uint32_t x0 = X[s];
      const uint32_t v = split_site<D, DOM>(x0, X, nbr + (size_t)s * D, jm[s], Y[s], q, a, tab, (uint32_t)gid[s], k, g);
      X[s] = v;
      nf += __popc(v ^ x0);
    }
  }
  return nf;
}

// Shared memory: E[slots] | O[slots] | gid[nlocmax] | jm[nlocmax] | nbr[nlocmax][D]
// CL: the group's sites are split over a cluster of CTAs (halo exchange);
// without it one CTA owns all sites and a phase ends with one block barrier.
template <int D, bool CL>
__global__ void __launch_bounds__(kSplitMaxThreads) sqa_split_kernel(SplitArgs a) {
  extern __shared__ __align__(16) uint32_t sh[];
  constexpr int NC = (D + 1) * 3;
  constexpr int E = SplitTab<D>::E;
  __shared__ __align__(16) uint32_t tab[SplitTab<D>::WORDS];
  const int p = CL ? (int)cg::this_cluster().block_rank() : 0;
  const int g = blockIdx.y;
  const int32_t* gid_g = a.gidx + (size_t)p * a.slots;
  const int32_t* co = a.coff + (size_t)p * (a.ncol + 1);
  const int32_t* cb = a.cb + (size_t)p * a.ncol;
  const int32_t* ho = a.hoff + (size_t)p * (a.ncol + 1);
  const uint32_t* hs = a.hsrc + (size_t)p * a.hmax;
  const uint16_t* hd = a.hdst + (size_t)p * a.hmax;
  const uint16_t* nbr_g = a.nbr + (size_t)p * a.nlocmax * D;
  const uint16_t* jm_g = a.jm + (size_t)p * a.nlocmax;
  uint32_t* WE = sh;
  uint32_t* WO = sh + a.slots;
  int32_t* gid = reinterpret_cast<int32_t*>(WO + a.slots);
  uint16_t* jm = reinterpret_cast<uint16_t*>(gid + a.nlocmax);
  uint16_t* nbr = jm + a.nlocmax;
  const int nloc = co[a.ncol];
  const int nhalo = ho[a.ncol];
  uint32_t* gE = a.words + (size_t)g * 2 * a.n;
  uint32_t* gO = gE + a.n;
  for (int s = threadIdx.x; s < nloc + nhalo; s += blockDim.x) {
    const int i = gid_g[s];
    WE[s] = gE[i];
    WO[s] = gO[i];
  }
  for (int s = threadIdx.x; s < nloc; s += blockDim.x) {
    gid[s] = gid_g[s];
    jm[s] = jm_g[s];
  }
  for (int s = threadIdx.x; s < nloc * D; s += blockDim.x) nbr[s] = nbr_g[s];
  __syncthreads();
  if constexpr (CL) cluster_arrive();
  unsigned long long nflip = 0;
  int prev_c = -1, prev_q = 0;  // colour class and half updated by the previous phase
  const uint32_t gg = a.group0 + (uint32_t)g;
  for (int64_t k = 0; k < a.nsweeps; ++k) {
    {
      // the sweep's tables (every thread finished the previous sweep's last
      // phase at its closing barrier)
      const uint32_t alw = __ldg(a.mode + 2 * k), live = __ldg(a.mode + 2 * k + 1);
      for (int idx = threadIdx.x; idx < SplitTab<D>::WORDS; idx += blockDim.x) {
        const int row = idx / (3 * E), kq = (idx / E) % 3, u = idx % E;
        uint32_t w = 0u;
        if (u <= D) {
          const int c = 3 * u + kq;
          bool on;
          if (row < 32)
            on = ((live >> c) & 1u) && ((__ldg(a.thr + (size_t)k * NC + c) >> (31 - row)) & 1u);
          else
            on = row == 32 ? ((alw >> c) & 1u) : ((live >> c) & 1u);
          w = on ? 0xFFFFFFFFu : 0u;
        }
        tab[idx] = w;
      }
      __syncthreads();
    }
    const uint32_t kk = a.sweep0 + (uint32_t)k;
    // the sweep's live classes allow the Trotter-dominated table evaluation
    const bool dom = (__ldg(a.mode + 2 * k + 1) & split_not_dominated_mask<D>()) == 0u;
    auto range = [&](int lo, int hi, uint32_t* X, const uint32_t* Y, int q) {
      return dom ? split_range<D, true>(lo, hi, X, Y, gid, jm, nbr, q, a, tab, kk, gg)
                 : split_range<D, false>(lo, hi, X, Y, gid, jm, nbr, q, a, tab, kk, gg);
    };
    for (int q = 0; q < 2; ++q) {
      uint32_t* X = q ? WO : WE;
      const uint32_t* Y = q ? WE : WO;
      for (int c = 0; c < a.ncol; ++c) {
        if constexpr (CL) {
          cg::cluster_group cl = cg::this_cluster();
          nflip += range(co[c], cb[c], X, Y, q);
          cluster_wait();
          if (prev_c >= 0) {
            uint32_t* P = prev_q ? WO : WE;
            const int hlo = ho[prev_c], hhi = ho[prev_c + 1];
            for (int e = hlo + threadIdx.x; e < hhi; e += blockDim.x) {
              const uint32_t src = hs[e];
              const uint32_t* remote = cl.map_shared_rank(P, (int)(src >> 16));
              P[hd[e]] = remote[src & 0xFFFFu];
            }
          }
          __syncthreads();
          nflip += range(cb[c], co[c + 1], X, Y, q);
          cluster_arrive();
          __syncthreads();
          prev_c = c;
          prev_q = q;
        } else {
          nflip += range(co[c], co[c + 1], X, Y, q);
          __syncthreads();
        }
      }
    }
  }
  if constexpr (CL) cluster_wait();
  for (int s = threadIdx.x; s < nloc; s += blockDim.x) {
    const int i = gid[s];
    gE[i] = WE[s];
    gO[i] = WO[s];
  }
  ojd::add_flips(a.flips, nflip);
}

// [R][T][n] int8 <-> [G][2][n] words
__global__ void split_pack_kernel(const int8_t* __restrict__ spins, int R, int T, int n, int P,
                                  uint32_t* __restrict__ words) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (i >= n) return;
  const int H = T / 2;
  uint32_t e = 0u, o = 0u;
  for (int p = 0; p < P; ++p) {
    const int r = g * P + p;
    if (r >= R) break;
    const int8_t* s = spins + (size_t)r * T * n + i;
    for (int m = 0; m < H; ++m) {
      if (s[(size_t)(2 * m) * n] < 0) e |= 1u << (p * H + m);
      if (s[(size_t)(2 * m + 1) * n] < 0) o |= 1u << (p * H + m);
    }
  }
  words[(size_t)g * 2 * n + i] = e;
  words[(size_t)g * 2 * n + n + i] = o;
}

__global__ void split_unpack_kernel(const uint32_t* __restrict__ words, int R, int T, int n, int P,
                                    int8_t* __restrict__ spins) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  if (i >= n) return;
  const int H = T / 2;
  const uint32_t e = words[(size_t)g * 2 * n + i], o = words[(size_t)g * 2 * n + n + i];
  for (int p = 0; p < P; ++p) {
    const int r = g * P + p;
    if (r >= R) break;
    int8_t* s = spins + (size_t)r * T * n + i;
    for (int m = 0; m < H; ++m) {
      s[(size_t)(2 * m) * n] = ((e >> (p * H + m)) & 1u) ? (int8_t)-1 : (int8_t)1;
      s[(size_t)(2 * m + 1) * n] = ((o >> (p * H + m)) & 1u) ? (int8_t)-1 : (int8_t)1;
    }
  }
}

size_t split_smem_bytes(const MscPlan& pl) {
  return (size_t)pl.slots * 8 + (size_t)pl.nlocmax * (4 + 2 + 2 * pl.D) + 16;
}

int split_threads() {
  int threads = kSplitDefaultThreads;
  if (const char* env = std::getenv("OJ_SQA_THREADS")) {
    const int v = std::atoi(env);
    if (v >= 32 && v <= kSplitMaxThreads && v % 32 == 0) threads = v;
  }
  return threads;
}

template <int D>
cudaError_t launch_d(const MscPlan& pl, const SplitArgs& a, int G, cudaStream_t st, int threads) {
  const size_t smem = split_smem_bytes(pl);
  if (smem > kSplitSmemBytes) return cudaErrorInvalidValue;
  if (pl.P == 1) {
    auto k1 = sqa_split_kernel<D, false>;
    cudaError_t e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k1<<<dim3(1, G, 1), threads, smem, st>>>(a);
    return cudaGetLastError();
  }
  auto kern = sqa_split_kernel<D, true>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (pl.P > 8) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(pl.P, G, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = pl.P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

}  // namespace

int split_default_threads() { return split_threads(); }

int sqa_split_replicas_per_group(int T) {
  const int H = T / 2;
  int P = 1;
  while (2 * P * H <= 32) P *= 2;
  return P;
}

bool sqa_split_applies(const oj_graph* g, int T) {
  return g->info.bimodal && g->regular && g->info.max_degree >= 1 && g->info.max_degree <= 8 && T >= 2 &&
         T <= 64 && T % 2 == 0;
}

// Cluster size for G replica groups: as many CTAs per group as the SMs allow
// (one CTA per SM), at least 256 sites per CTA, and a partition whose two
// halves, halo and tables fit the shared-memory budget.
cudaError_t sqa_split_prepare(oj_graph* g, int G, int sm_count, std::string* why, int cluster) {
  int P = std::max(1, std::min(kSplitMaxCluster, sm_count / std::max(G, 1)));
  while (P > 1 && g->n / P < 256) --P;
  if (const char* env = std::getenv("OJ_SQA_CLUSTER")) {
    const int v = std::atoi(env);
    if (v >= 1 && v <= kSplitMaxCluster && v <= g->n) P = v;
  }
  if (cluster >= 1 && cluster <= kSplitMaxCluster && cluster <= g->n) P = cluster;
  for (; P <= kSplitMaxCluster; ++P) {
    std::string w;
    const cudaError_t e = msc_prepare(g, P, &w);
    if (e == cudaSuccess && split_smem_bytes(*g->msc) <= kSplitSmemBytes) return cudaSuccess;
    if (e != cudaSuccess && e != cudaErrorInvalidValue) return e;
  }
  if (why) *why = "slice-split SQA kernel: no cluster partition fits shared memory";
  return cudaErrorInvalidValue;
}

cudaError_t launch_sqa_split(const oj_graph* g, int G, int T, uint32_t* words, const uint32_t* thr,
                             const uint32_t* mode, int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches,
                             int threads) {
  if (threads == 0) threads = split_threads();
  if (threads < 32 || threads > kSplitMaxThreads || threads % 32) return cudaErrorInvalidValue;
  const MscPlan& pl = *g->msc;
  SplitArgs a;
  a.gidx = pl.gidx;
  a.coff = pl.coff;
  a.cb = pl.cb;
  a.hoff = pl.hoff;
  a.hsrc = pl.hsrc;
  a.hdst = pl.hdst;
  a.nbr = pl.nbr;
  a.jm = pl.jm;
  a.slots = pl.slots;
  a.nlocmax = pl.nlocmax;
  a.hmax = pl.hmax;
  a.ncol = pl.ncol;
  a.n = g->n;
  const int H = T / 2, P = sqa_split_replicas_per_group(T);
  a.H = H;
  a.low = 0u;
  a.high = 0u;
  for (int p = 0; p < P; ++p) {
    a.low |= 1u << (p * H);
    a.high |= 1u << (p * H + H - 1);
  }
  a.valid = P * H >= 32 ? 0xFFFFFFFFu : ((1u << (P * H)) - 1u);
  a.words = words;
  a.thr = thr;
  a.mode = mode;
  a.nsweeps = nsweeps;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.group0 = rb.rep0 / (uint32_t)P;
  a.flips = rb.flips;
  if (launches) ++*launches;
  switch (pl.D) {
    case 1: return launch_d<1>(pl, a, G, st, threads);
    case 2: return launch_d<2>(pl, a, G, st, threads);
    case 3: return launch_d<3>(pl, a, G, st, threads);
    case 4: return launch_d<4>(pl, a, G, st, threads);
    case 5: return launch_d<5>(pl, a, G, st, threads);
    case 6: return launch_d<6>(pl, a, G, st, threads);
    case 7: return launch_d<7>(pl, a, G, st, threads);
    case 8: return launch_d<8>(pl, a, G, st, threads);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_sqa_split_pack(const int8_t* spins, int R, int T, int n, int G, uint32_t* words,
                                  cudaStream_t st) {
  dim3 grid((n + 255) / 256, G);
  split_pack_kernel<<<grid, 256, 0, st>>>(spins, R, T, n, sqa_split_replicas_per_group(T), words);
  return cudaGetLastError();
}

cudaError_t launch_sqa_split_unpack(const uint32_t* words, int R, int T, int n, int G, int8_t* spins,
                                    cudaStream_t st) {
  dim3 grid((n + 255) / 256, G);
  split_unpack_kernel<<<grid, 256, 0, st>>>(words, R, T, n, sqa_split_replicas_per_group(T), spins);
  return cudaGetLastError();
}

}  // namespace oj
