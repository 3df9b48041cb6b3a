// Bit-packed ("multi-spin coded") SA sweep for regular graphs with couplings
// +-c and no fields — the 2D +-J lattice and random regular +-J graphs.
//
// Word (g, i) holds site i of replicas 32g..32g+31, bit j set iff that
// replica's spin is -1.  For bond (i, j) the bit word
//     unsat = b_i ^ b_j ^ (J_ij > 0 ? ~0 : 0)
// marks the replicas where the bond is unsatisfied (J s_i s_j > 0); with u the
// per-replica count of unsatisfied bonds, flipping s_i changes the energy by
// dE = 2c(d - 2u) (the reference's dE_i = -2 s_i sum_j J_ij s_j,
// include/openjij/system/classical_ising.hpp:87-90).  Replicas with dE <= 0
// flip (single_spin_flip.hpp:80); the others flip when the 32-bit uniform U
// is below thr[k][d-2u] = floor(exp(-beta_k*dE)*2^32).  U is compared one
// bit level at a time for all 32 replicas at once, most significant level
// first, drawing a fresh Philox word per level; the loop stops as soon as
// every replica is decided.
//
// Sites follow the classes of a greedy colouring (checkerboard on a bipartite
// lattice).  One thread block cluster owns one replica group: its P CTAs split
// the sites into contiguous ranges and keep, in shared memory, their own words,
// a halo copy of the remote neighbours and the neighbour tables.  Per colour
// class a CTA first updates its interior sites (no remote neighbour), then
// waits on the cluster barrier (split arrive / wait, so the barrier latency
// hides behind the interior work), updates its boundary sites, and the thread
// that updated a boundary site stores the new word straight into the halo
// slots of the CTAs that read it (DSMEM stores, made visible to them by the
// release of its next arrive), so no copy sits between a wait and the work
// after it.  A halo slot of class c is written only in class c's phase, after
// the writer's wait of that phase, when every reader has left the phase before
// it, and it is read only in other classes' phases, after the reader's wait.
// Nothing touches global memory between the initial load and the final store.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace cg = cooperative_groups;

namespace oj {
namespace {

constexpr int kMscMaxThreads = 1024;
constexpr int kMscDefaultThreads = 512;
constexpr int kMscMaxDegree = 8;
constexpr int kMscMaxCluster = 16;
constexpr size_t kMscSmemBytes = 200 * 1024;

struct MscArgs {
  const int32_t* gidx;
  const int32_t* coff;
  const int32_t* cb;
  const int32_t* hoff;
  const uint32_t* hsrc;
  const uint16_t* hdst;
  const uint16_t* nbr;
  const uint16_t* jm;
  const int32_t* poff;
  const uint32_t* pent;
  int slots, nlocmax, hmax, ncol, pmax;
  int n;
  uint32_t* words;
  const uint32_t* thr;     // [nsweeps][D+1]
  const uint32_t* always;  // [nsweeps]
  int64_t nsweeps;
  ojd::Keys keys;
  uint32_t sweep0;  // global index of the first sweep
  uint32_t group0;  // global index of the first replica group
  unsigned long long* flips;  // accepted-flip counter (every bit of the group's words), or null
};

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Per-sweep acceptance data of the uphill classes u = 0..UMAX-1 (dE = 2c(D-2u)).
template <int D>
struct MscSweep {
  static constexpr int UMAX = (D + 1) / 2;
  uint32_t tv[UMAX];  // thresholds
  uint32_t alw;       // bit u: class u always accepts
  uint32_t live;      // bit u: class u has a non-zero threshold and is not always-accept
};

template <int D>
__device__ __forceinline__ MscSweep<D> msc_sweep(const uint32_t* __restrict__ thr_k, uint32_t always_k) {
  MscSweep<D> sw;
  sw.alw = 0u;
  sw.live = 0u;
#pragma unroll
  for (int u = 0; u < MscSweep<D>::UMAX; ++u) {
    const int dm = D - 2 * u;
    sw.tv[u] = thr_k[dm];
    if ((always_k >> dm) & 1u)
      sw.alw |= 1u << u;
    else if (sw.tv[u] != 0u)
      sw.live |= 1u << u;
  }
  return sw;
}

// One bit level of the comparison U < thr for all 32 replicas.
template <int D>
__device__ __forceinline__ void msc_level(const MscSweep<D>& sw, const uint32_t (&cls)[MscSweep<D>::UMAX],
                                          int bitpos, uint32_t wl, uint32_t& pending, uint32_t& lt) {
  uint32_t pm = 0u;
#pragma unroll
  for (int u = 0; u < MscSweep<D>::UMAX; ++u) pm |= cls[u] & (0u - ((sw.tv[u] >> bitpos) & 1u));
  lt |= pending & pm & ~wl;
  pending &= ~(pm ^ wl);
}

template <int D>
__device__ __forceinline__ uint32_t msc_site(uint32_t w, const uint32_t* __restrict__ Wsh,
                                             const uint16_t* __restrict__ nb, uint32_t jmk,
                                             const MscSweep<D>& sw, uint32_t site, uint32_t sweep,
                                             uint32_t grp, const ojd::Keys& K) {
  constexpr int NB = D <= 1 ? 1 : (D <= 3 ? 2 : (D <= 7 ? 3 : 4));
  constexpr int UMAX = MscSweep<D>::UMAX;
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
  uint32_t cls[UMAX];
  uint32_t uphill = 0u, pending = 0u, flip = 0u;
#pragma unroll
  for (int u = 0; u < UMAX; ++u) {
    uint32_t m = 0xFFFFFFFFu;
#pragma unroll
    for (int b = 0; b < NB; ++b) m &= ((u >> b) & 1) ? cnt[b] : ~cnt[b];
    uphill |= m;
    if ((sw.alw >> u) & 1u) flip |= m;
    m = ((sw.live >> u) & 1u) ? m : 0u;
    cls[u] = m;
    pending |= m;
  }
  flip |= ~uphill;
  uint32_t lt = 0u;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    if (!pending) break;
    const ojd::u4 r = ojd::philox(site, sweep, grp, ((uint32_t)q << 8) | ojd::TAG_SA_MSC, K);
    msc_level<D>(sw, cls, 31 - 4 * q, r.x, pending, lt);
    msc_level<D>(sw, cls, 30 - 4 * q, r.y, pending, lt);
    msc_level<D>(sw, cls, 29 - 4 * q, r.z, pending, lt);
    msc_level<D>(sw, cls, 28 - 4 * q, r.w, pending, lt);
  }
  return w ^ (flip | lt);
}

// Stores word w of own slot s into the readers' halo slots (boundary slots).
__device__ __forceinline__ void msc_push(const cg::cluster_group& cl, uint32_t* Wsh, int e0, int e1,
                                         const uint32_t* __restrict__ pent, uint32_t w) {
  for (int e = e0; e < e1; ++e) {
    const uint32_t d = __ldg(pent + e);
    uint32_t* remote = cl.map_shared_rank(Wsh, (int)(d >> 16));
    remote[d & 0xFFFFu] = w;
  }
}

// Updates own slots [lo, hi), two independent sites per thread and iteration,
// and pushes the new words of slots >= bnd (the boundary sites) to their
// readers; returns the number of spins this thread flipped.
template <int D>
__device__ __forceinline__ uint32_t msc_range(int lo, int hi, int bnd, uint32_t* __restrict__ Wsh,
                                              const int32_t* __restrict__ gid, const uint16_t* __restrict__ jm,
                                              const uint16_t* __restrict__ nbr, const int32_t* __restrict__ poff,
                                              const uint32_t* __restrict__ pent, const cg::cluster_group& cl,
                                              const MscSweep<D>& sw, uint32_t k, uint32_t g, const ojd::Keys& K) {
  const int T = blockDim.x;
  uint32_t nf = 0u;
  for (int s = lo + threadIdx.x; s < hi; s += 2 * T) {
    const int s2 = s + T;
    // the later slot first: boundary slots close a class's range, so its
    // halo stores are in flight while the other site is updated
    if (s2 < hi) {
      const uint32_t w2 = Wsh[s2];
      const uint32_t b = msc_site<D>(w2, Wsh, nbr + (size_t)s2 * D, jm[s2], sw, (uint32_t)gid[s2], k, g, K);
      Wsh[s2] = b;
      nf += __popc(b ^ w2);
      if (s2 >= bnd) msc_push(cl, Wsh, __ldg(poff + s2), __ldg(poff + s2 + 1), pent, b);
    }
    const uint32_t w0 = Wsh[s];
    const uint32_t a = msc_site<D>(w0, Wsh, nbr + (size_t)s * D, jm[s], sw, (uint32_t)gid[s], k, g, K);
    Wsh[s] = a;
    nf += __popc(a ^ w0);
    if (s >= bnd) msc_push(cl, Wsh, __ldg(poff + s), __ldg(poff + s + 1), pent, a);
  }
  return nf;
}

// Shared memory: words[slots] | gid[nlocmax] | jm[nlocmax] | nbr[nlocmax][D]
// MAXT: the launch bound (512: up to 128 registers a thread; 1024: 64).
template <int D, int MAXT>
__global__ void __launch_bounds__(MAXT) sa_msc_kernel(MscArgs a) {
  extern __shared__ __align__(16) uint32_t Wsh[];
  cg::cluster_group cl = cg::this_cluster();
  const int p = (int)cl.block_rank();
  const int g = blockIdx.y;
  const int32_t* gid_g = a.gidx + (size_t)p * a.slots;
  const int32_t* co = a.coff + (size_t)p * (a.ncol + 1);
  const int32_t* cb = a.cb + (size_t)p * a.ncol;
  const int32_t* ho = a.hoff + (size_t)p * (a.ncol + 1);
  const uint16_t* nbr_g = a.nbr + (size_t)p * a.nlocmax * D;
  const uint16_t* jm_g = a.jm + (size_t)p * a.nlocmax;
  const int32_t* poff = a.poff + (size_t)p * (a.nlocmax + 1);
  const uint32_t* pent = a.pent + (size_t)p * a.pmax;
  int32_t* gid = reinterpret_cast<int32_t*>(Wsh + a.slots);
  uint16_t* jm = reinterpret_cast<uint16_t*>(gid + a.nlocmax);
  uint16_t* nbr = jm + a.nlocmax;
  const int nloc = co[a.ncol];
  const int nhalo = ho[a.ncol];
  uint32_t* gw = a.words + (size_t)g * a.n;
  for (int s = threadIdx.x; s < nloc + nhalo; s += blockDim.x) Wsh[s] = gw[gid_g[s]];
  for (int s = threadIdx.x; s < nloc; s += blockDim.x) {
    gid[s] = gid_g[s];
    jm[s] = jm_g[s];
  }
  for (int s = threadIdx.x; s < nloc * D; s += blockDim.x) nbr[s] = nbr_g[s];
  __syncthreads();
  cluster_arrive();
  unsigned long long nflip = 0;
  for (int64_t k = 0; k < a.nsweeps; ++k) {
    const MscSweep<D> sw = msc_sweep<D>(a.thr + (size_t)k * (D + 1), a.always[k]);
    const uint32_t kk = a.sweep0 + (uint32_t)k, gg = a.group0 + (uint32_t)g;
    for (int c = 0; c < a.ncol; ++c) {
      // the class's sites go in rounds of 2 x blockDim.x (two per thread):
      // the interior sites of all rounds but the last run before the cluster
      // wait, the rest of the interior with the boundary sites after the halo
      // refresh, so that no round is left to the few boundary sites alone
      // (sites of one class do not read each other: any order gives the same
      // words)
      const int step = 2 * (int)blockDim.x, nc = co[c + 1] - co[c];
      const int split = co[c] + min(cb[c] - co[c], max(0, (nc + step - 1) / step * step - step));
      nflip += msc_range<D>(co[c], split, cb[c], Wsh, gid, jm, nbr, poff, pent, cl, sw, kk, gg, a.keys);
      // after the wait every halo word this class reads has been pushed (the
      // same-class sites of this round do not read each other)
      cluster_wait();
      nflip += msc_range<D>(split, co[c + 1], cb[c], Wsh, gid, jm, nbr, poff, pent, cl, sw, kk, gg, a.keys);
      // arrive first (its release covers this thread's halo stores), then the
      // CTA barrier (the next phase reads this phase's words of other
      // threads); the other order measured slower
      cluster_arrive();
      __syncthreads();
    }
  }
  cluster_wait();
  for (int s = threadIdx.x; s < nloc; s += blockDim.x) gw[gid[s]] = Wsh[s];
  ojd::add_flips(a.flips, nflip);
}

size_t msc_smem_bytes(const MscPlan& pl) {
  return (size_t)pl.slots * 4 + (size_t)pl.nlocmax * (4 + 2 + 2 * pl.D) + 16;
}

int msc_threads() {
  int threads = kMscDefaultThreads;
  if (const char* env = std::getenv("OJ_MSC_THREADS")) {
    const int v = std::atoi(env);
    if (v >= 32 && v <= kMscMaxThreads && v % 32 == 0) threads = v;
  }
  return threads;
}

template <int D>
cudaError_t launch_d(const MscPlan& pl, const MscArgs& a, int G, cudaStream_t st, int threads) {
  auto kern = threads <= 512 ? sa_msc_kernel<D, 512> : sa_msc_kernel<D, kMscMaxThreads>;
  const size_t smem = msc_smem_bytes(pl);
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

int msc_max_degree() { return kMscMaxDegree; }

cudaError_t msc_preload() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaSuccess;
  auto load = [&](auto k512, auto k1024) {
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k512);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k1024);
  };
  load(sa_msc_kernel<1, 512>, sa_msc_kernel<1, kMscMaxThreads>);
  load(sa_msc_kernel<2, 512>, sa_msc_kernel<2, kMscMaxThreads>);
  load(sa_msc_kernel<3, 512>, sa_msc_kernel<3, kMscMaxThreads>);
  load(sa_msc_kernel<4, 512>, sa_msc_kernel<4, kMscMaxThreads>);
  load(sa_msc_kernel<5, 512>, sa_msc_kernel<5, kMscMaxThreads>);
  load(sa_msc_kernel<6, 512>, sa_msc_kernel<6, kMscMaxThreads>);
  load(sa_msc_kernel<7, 512>, sa_msc_kernel<7, kMscMaxThreads>);
  load(sa_msc_kernel<8, 512>, sa_msc_kernel<8, kMscMaxThreads>);
  return e;
}
int msc_default_threads() { return msc_threads(); }

// Cluster size: the number of CTAs per replica group.  One CTA per SM, as
// many CTAs as fit on the SMs (measured on the L=128 lattice: one 512-thread
// CTA per SM beats two smaller ones and uneven multi-CTA packings), within the
// shared-memory budget and the 16-CTA non-portable cluster limit.
int msc_choose_cluster(const oj_graph* g, int G, int sm_count) {
  if (const char* env = std::getenv("OJ_MSC_CLUSTER")) {
    const int v = std::atoi(env);
    if (v >= 1 && v <= kMscMaxCluster) return v;
  }
  const int D = g->info.max_degree;
  auto fits = [&](int P) {
    const size_t per = (size_t)((g->n + P - 1) / P);
    return per * (4 + 6 + 2 * (size_t)D) + per / 2 * 4 <= kMscSmemBytes;
  };
  int P = std::max(1, std::min(kMscMaxCluster, sm_count / std::max(G, 1)));
  while (P > 1 && g->n / P < 256) --P;
  while (P < kMscMaxCluster && !fits(P)) ++P;
  return P;
}

// Host-side partition of the sites over the P CTAs of a cluster.
cudaError_t msc_prepare(oj_graph* g, int P, std::string* why) {
  if (g->msc && g->msc->P == P) return cudaSuccess;
  const int n = g->n;
  const int D = g->info.max_degree;
  const int ncol = g->info.num_colours;
  std::vector<int> bound(P + 1);
  for (int p = 0; p <= P; ++p) bound[p] = (int)(((int64_t)p * n) / P);
  std::vector<int> part_of(n), slot_of(n);
  std::vector<char> is_bnd(n, 0);
  for (int p = 0; p < P; ++p)
    for (int i = bound[p]; i < bound[p + 1]; ++i) part_of[i] = p;
  for (int i = 0; i < n; ++i)
    for (int q = g->rp[i]; q < g->rp[i + 1]; ++q)
      if (part_of[g->ci[q]] != part_of[i]) is_bnd[i] = 1;
  struct Part {
    std::vector<int> own, halo;  // global site ids in slot order
    std::vector<int> coff, cb, hoff;
  };
  std::vector<Part> parts(P);
  for (int p = 0; p < P; ++p) {
    Part& pt = parts[p];
    for (int i = bound[p]; i < bound[p + 1]; ++i) pt.own.push_back(i);
    std::sort(pt.own.begin(), pt.own.end(), [&](int a, int b) {
      if (g->colour[a] != g->colour[b]) return g->colour[a] < g->colour[b];
      if (is_bnd[a] != is_bnd[b]) return is_bnd[a] < is_bnd[b];
      return a < b;
    });
    for (size_t s = 0; s < pt.own.size(); ++s) slot_of[pt.own[s]] = (int)s;
  }
  int slots = 0, nlocmax = 0, hmax = 0;
  for (int p = 0; p < P; ++p) {
    Part& pt = parts[p];
    std::vector<char> mark(n, 0);
    for (int i : pt.own)
      for (int q = g->rp[i]; q < g->rp[i + 1]; ++q) {
        const int j = g->ci[q];
        if (part_of[j] != p && !mark[j]) {
          mark[j] = 1;
          pt.halo.push_back(j);
        }
      }
    std::sort(pt.halo.begin(), pt.halo.end(), [&](int a, int b) {
      return g->colour[a] != g->colour[b] ? g->colour[a] < g->colour[b] : a < b;
    });
    pt.coff.assign(ncol + 1, 0);
    pt.cb.assign(ncol, 0);
    pt.hoff.assign(ncol + 1, 0);
    for (int i : pt.own) pt.coff[g->colour[i] + 1]++;
    for (int j : pt.halo) pt.hoff[g->colour[j] + 1]++;
    for (int c = 0; c < ncol; ++c) {
      pt.coff[c + 1] += pt.coff[c];
      pt.hoff[c + 1] += pt.hoff[c];
    }
    for (int c = 0; c < ncol; ++c) {
      int s = pt.coff[c];
      while (s < pt.coff[c + 1] && !is_bnd[pt.own[s]]) ++s;
      pt.cb[c] = s;
    }
    slots = std::max(slots, (int)(pt.own.size() + pt.halo.size()));
    nlocmax = std::max(nlocmax, (int)pt.own.size());
    hmax = std::max(hmax, (int)pt.halo.size());
  }
  // push lists: every halo slot of every part, filed under the slot of the
  // part that owns the site
  std::vector<std::vector<std::pair<int, uint32_t>>> push(P);  // (own slot, reader part << 16 | reader slot)
  for (int q = 0; q < P; ++q) {
    const int nloc_q = (int)parts[q].own.size();
    for (size_t h = 0; h < parts[q].halo.size(); ++h) {
      const int j = parts[q].halo[h];
      push[part_of[j]].emplace_back(slot_of[j], ((uint32_t)q << 16) | (uint32_t)(nloc_q + h));
    }
  }
  int pmax = 1;
  for (int p = 0; p < P; ++p) {
    std::sort(push[p].begin(), push[p].end());
    pmax = std::max(pmax, (int)push[p].size());
  }
  if (slots > 65535 || (size_t)slots * 4 + (size_t)nlocmax * (6 + 2 * D) + 16 > kMscSmemBytes) {
    if (why) *why = "bit-packed kernel: partition does not fit shared memory; use a larger cluster";
    return cudaErrorInvalidValue;
  }
  hmax = std::max(hmax, 1);
  std::vector<int32_t> gidx((size_t)P * slots, 0), coff((size_t)P * (ncol + 1)), cbv((size_t)P * ncol),
      hoff((size_t)P * (ncol + 1));
  std::vector<uint32_t> hsrc((size_t)P * hmax, 0);
  std::vector<uint16_t> hdst((size_t)P * hmax, 0), nbr((size_t)P * nlocmax * D, 0), jm((size_t)P * nlocmax, 0);
  std::vector<int32_t> poff((size_t)P * (nlocmax + 1), 0);
  std::vector<uint32_t> pent((size_t)P * pmax, 0);
  for (int p = 0; p < P; ++p) {
    int32_t* po = poff.data() + (size_t)p * (nlocmax + 1);
    for (const auto& e : push[p]) ++po[e.first + 1];
    for (int s = 0; s < nlocmax; ++s) po[s + 1] += po[s];
    for (size_t e = 0; e < push[p].size(); ++e) pent[(size_t)p * pmax + e] = push[p][e].second;
  }
  for (int p = 0; p < P; ++p) {
    Part& pt = parts[p];
    const int nloc = (int)pt.own.size();
    std::vector<int> local_slot_of_halo(n, -1);
    for (size_t h = 0; h < pt.halo.size(); ++h) local_slot_of_halo[pt.halo[h]] = nloc + (int)h;
    for (int s = 0; s < nloc; ++s) gidx[(size_t)p * slots + s] = pt.own[s];
    for (size_t h = 0; h < pt.halo.size(); ++h) {
      const int j = pt.halo[h];
      gidx[(size_t)p * slots + nloc + h] = j;
      hsrc[(size_t)p * hmax + h] = ((uint32_t)part_of[j] << 16) | (uint32_t)slot_of[j];
      hdst[(size_t)p * hmax + h] = (uint16_t)(nloc + h);
    }
    for (int c = 0; c <= ncol; ++c) {
      coff[(size_t)p * (ncol + 1) + c] = pt.coff[c];
      hoff[(size_t)p * (ncol + 1) + c] = pt.hoff[c];
    }
    for (int c = 0; c < ncol; ++c) cbv[(size_t)p * ncol + c] = pt.cb[c];
    for (int s = 0; s < nloc; ++s) {
      const int i = pt.own[s];
      uint16_t bits = 0;
      int l = 0;
      for (int q = g->rp[i]; q < g->rp[i + 1]; ++q, ++l) {
        const int j = g->ci[q];
        const int ls = part_of[j] == p ? slot_of[j] : local_slot_of_halo[j];
        nbr[((size_t)p * nlocmax + s) * D + l] = (uint16_t)ls;
        if (g->val64[q] > 0) bits |= (uint16_t)(1u << l);
      }
      jm[(size_t)p * nlocmax + s] = bits;
    }
  }
  auto plan = std::make_unique<MscPlan>();
  plan->P = P;
  plan->D = D;
  plan->ncol = ncol;
  plan->slots = slots;
  plan->nlocmax = nlocmax;
  plan->hmax = hmax;
  plan->pmax = pmax;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_gidx = al(gidx.size() * 4), b_coff = al(coff.size() * 4), b_cb = al(cbv.size() * 4),
               b_hoff = al(hoff.size() * 4), b_hsrc = al(hsrc.size() * 4), b_hdst = al(hdst.size() * 2),
               b_nbr = al(nbr.size() * 2), b_jm = al(jm.size() * 2), b_poff = al(poff.size() * 4),
               b_pent = al(pent.size() * 4);
  cudaError_t e = plan->tables.ensure(b_gidx + b_coff + b_cb + b_hoff + b_hsrc + b_hdst + b_nbr + b_jm + b_poff +
                                      b_pent);
  if (e != cudaSuccess) return e;
  char* base = plan->tables.as<char>();
  size_t off = 0;
  auto put = [&](auto*& dst, const auto& vec, size_t bytes) -> cudaError_t {
    dst = reinterpret_cast<std::remove_reference_t<decltype(dst)>>(base + off);
    off += bytes;
    return cudaMemcpy(dst, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice);
  };
  if ((e = put(plan->gidx, gidx, b_gidx)) != cudaSuccess) return e;
  if ((e = put(plan->coff, coff, b_coff)) != cudaSuccess) return e;
  if ((e = put(plan->cb, cbv, b_cb)) != cudaSuccess) return e;
  if ((e = put(plan->hoff, hoff, b_hoff)) != cudaSuccess) return e;
  if ((e = put(plan->hsrc, hsrc, b_hsrc)) != cudaSuccess) return e;
  if ((e = put(plan->hdst, hdst, b_hdst)) != cudaSuccess) return e;
  if ((e = put(plan->nbr, nbr, b_nbr)) != cudaSuccess) return e;
  if ((e = put(plan->jm, jm, b_jm)) != cudaSuccess) return e;
  if ((e = put(plan->poff, poff, b_poff)) != cudaSuccess) return e;
  if ((e = put(plan->pent, pent, b_pent)) != cudaSuccess) return e;
  g->msc = std::move(plan);
  return cudaSuccess;
}

cudaError_t launch_sa_msc(const oj_graph* g, int G, uint32_t* words, const uint32_t* thr,
                          const uint32_t* always, int64_t nsweeps, RngBase rb, cudaStream_t st,
                          int* launches, int threads) {
  if (threads == 0) threads = msc_threads();
  if (threads < 32 || threads > kMscMaxThreads || threads % 32) return cudaErrorInvalidValue;
  const MscPlan& pl = *g->msc;
  MscArgs a;
  a.gidx = pl.gidx;
  a.coff = pl.coff;
  a.cb = pl.cb;
  a.hoff = pl.hoff;
  a.hsrc = pl.hsrc;
  a.hdst = pl.hdst;
  a.nbr = pl.nbr;
  a.jm = pl.jm;
  a.poff = pl.poff;
  a.pent = pl.pent;
  a.pmax = pl.pmax;
  a.slots = pl.slots;
  a.nlocmax = pl.nlocmax;
  a.hmax = pl.hmax;
  a.ncol = pl.ncol;
  a.n = g->n;
  a.words = words;
  a.thr = thr;
  a.always = always;
  a.nsweeps = nsweeps;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.group0 = rb.rep0 >> 5;
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

}  // namespace oj
