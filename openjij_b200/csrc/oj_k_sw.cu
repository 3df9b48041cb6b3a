// Swendsen-Wang cluster updates for sparse Ising graphs, one CTA per replica
// (state in shared memory up to sw_max_sites() spins, in global memory above).
//
// The reference's SwendsenWang updater (include/openjij/updater/swendsen_wang.hpp:43-182)
// works on the n spins plus the dummy spin n that carries the fields (bond
// (i, n) with coupling h_i).  One update:
//   1. every bond (i, j), i < j, that is satisfied (J s_i s_j < 0) is kept
//      with probability 1 - exp(-2 beta |J|);
//   2. the kept bonds define clusters (union-find);
//   3. every cluster flips with probability 1/2.
// Here, per replica and sweep, in shared memory:
//   1. bond e is kept when -ln(u_e) < 2 beta |J| (FP32; the same event as
//      u'_e < 1 - exp(-2 beta |J|) with u' = 1 - u), u_e from
//      Philox((e >> 2, k, r, TAG_SW_BOND))[e & 3];
//   2. union-find with lock-free hooking of the larger root under the smaller
//      one, so every cluster's root is its smallest site, whatever the order
//      in which the threads hook;
//   3. the cluster of the dummy spin stays, every other cluster flips when bit 0
//      of Philox((root >> 2, k, r, TAG_SW_FLIP))[root & 3] is set.  Holding
//      the dummy fixed leaves the distribution of the physical spins s_i s_n
//      unchanged (get_solution, include/openjij/result/get_solution.hpp:39-49,
//      reads s_i s_n): flipping the dummy's cluster with probability 1/2 is
//      the same as flipping every other cluster once more with probability 1/2.
// The partition into clusters does not depend on thread timing, so the result
// is a pure function of seed, sweep, replica and state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kSwThreads = 512;

struct SwArgs {
  const int32_t* ei;   // [ne] bond endpoints, ei < ej (ej == n: the dummy spin)
  const int32_t* ej;
  const float* w;      // [ne] |J| of the bond (FP32)
  const uint8_t* pos;  // [ne] 1 when J > 0
  int ne, n;
  int8_t* spins;       // [R][n]
  const float* betas;  // [nsweeps]
  int64_t nsweeps;
  ojd::Keys keys;
  uint32_t sweep0, rep0;
};

// Parent links live in shared memory (SMEM) or, for graphs too large for it,
// in a global scratch array; there they are read past L1 (__ldcg), which does
// not see the L2 atomics of the other threads.
template <bool SMEM>
__device__ __forceinline__ uint32_t ld_parent(const uint32_t* p) {
  if constexpr (SMEM) {
    return *p;
  } else {
    return __ldcg(p);
  }
}

template <bool SMEM>
__device__ __forceinline__ uint32_t find_root(uint32_t* parent, uint32_t x) {
  uint32_t p = ld_parent<SMEM>(parent + x);
  while (p != x) {
    const uint32_t gp = ld_parent<SMEM>(parent + p);
    if (gp != p) parent[x] = gp;  // path halving (only ever points a node at an ancestor)
    x = p;
    p = gp;
  }
  return x;
}

template <bool SMEM>
__device__ __forceinline__ void unite(uint32_t* parent, uint32_t a, uint32_t b) {
  for (int guard = 0; guard < (1 << 20); ++guard) {
    a = find_root<SMEM>(parent, a);
    b = find_root<SMEM>(parent, b);
    if (a == b) return;
    if (a < b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    // hook the larger root under the smaller; retry if a moved meanwhile
    if (atomicCAS(&parent[a], a, b) == a) return;
  }
}

// SMEM: shared memory holds parent[n + 1] (u32) | spins[n] (int8).  Otherwise
// parent is replica r's slice of gparent ([gridDim.x][n + 1]) and the spins
// are updated in place in global memory.
template <bool SMEM>
__global__ void __launch_bounds__(kSwThreads) sw_kernel(SwArgs a, uint32_t* gparent) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int n = a.n;
  const int r = blockIdx.x;
  int8_t* gs = a.spins + (size_t)r * n;
  uint32_t* parent = SMEM ? smem : gparent + (size_t)r * (n + 1);
  int8_t* s = SMEM ? reinterpret_cast<int8_t*>(smem + n + 1) : gs;
  if (SMEM)
    for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = gs[i];
  const uint32_t rg = a.rep0 + (uint32_t)r;
  for (int64_t k = 0; k < a.nsweeps; ++k) {
    const float beta2 = __fmul_rn(2.0f, __ldg(a.betas + k));
    const uint32_t kk = a.sweep0 + (uint32_t)k;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) parent[i] = (uint32_t)i;
    __syncthreads();
    // 1. bonds, four per thread and Philox call
    for (int e0 = 4 * threadIdx.x; e0 < a.ne; e0 += 4 * blockDim.x) {
      const ojd::u4 x = ojd::philox((uint32_t)(e0 >> 2), kk, rg, ojd::TAG_SW_BOND, a.keys);
      const uint32_t xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = e0 + q;
        if (e >= a.ne) break;
        const int i = a.ei[e], j = a.ej[e];
        const int si = s[i], sj = j < n ? s[j] : 1;
        const bool satisfied = (si * sj > 0) != (a.pos[e] != 0);  // J s_i s_j < 0
        if (satisfied && ojd::neglog(xs[q]) < __fmul_rn(beta2, a.w[e])) unite<SMEM>(parent, (uint32_t)i, (uint32_t)j);
      }
    }
    __syncthreads();
    // 2./3. roots and flips; the dummy spin's cluster stays
    const uint32_t rn = find_root<SMEM>(parent, (uint32_t)n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t root = find_root<SMEM>(parent, (uint32_t)i);
      if (root == rn) continue;
      const ojd::u4 c = ojd::philox(root >> 2, kk, rg, ojd::TAG_SW_FLIP, a.keys);
      if (ojd::pick(c, (int)(root & 3u)) & 1u) s[i] = (int8_t)-s[i];
    }
    __syncthreads();
  }
  if (SMEM)
    for (int i = threadIdx.x; i < n; i += blockDim.x) gs[i] = s[i];
}

}  // namespace

size_t sw_smem_bytes(int n) { return (size_t)(n + 1) * 4 + (size_t)n + 16; }

// Bond list of the graph: (i, j) with i < j from the neighbour lists, then
// (i, n) for every non-zero h_i; built once per graph.
cudaError_t sw_prepare(oj_graph* g) {
  if (g->sw_ne >= 0) return cudaSuccess;
  std::vector<int32_t> ei, ej;
  std::vector<float> w;
  std::vector<uint8_t> pos;
  for (int i = 0; i < g->n; ++i)
    for (int q = g->rp[i]; q < g->rp[i + 1]; ++q) {
      const int j = g->ci[q];
      if (j <= i) continue;
      ei.push_back(i);
      ej.push_back(j);
      w.push_back((float)std::fabs(g->val64[q]));
      pos.push_back(g->val64[q] > 0 ? 1 : 0);
    }
  for (int i = 0; i < g->n; ++i)
    if (g->h64[i] != 0.0) {
      ei.push_back(i);
      ej.push_back(g->n);
      w.push_back((float)std::fabs(g->h64[i]));
      pos.push_back(g->h64[i] > 0 ? 1 : 0);
    }
  const size_t ne = ei.size();
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_i = al(ne * 4 + 4), b_w = al(ne * 4 + 4), b_p = al(ne + 1);
  cudaError_t e = g->sw_tables.ensure(2 * b_i + b_w + b_p);
  if (e != cudaSuccess) return e;
  char* base = g->sw_tables.as<char>();
  if (ne) {
    if ((e = cudaMemcpy(base, ei.data(), ne * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(base + b_i, ej.data(), ne * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(base + 2 * b_i, w.data(), ne * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(base + 2 * b_i + b_w, pos.data(), ne, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
  }
  g->sw_ne = (int64_t)ne;
  return cudaSuccess;
}

cudaError_t launch_sw(const oj_graph* g, int R, int8_t* spins, const float* betas, int64_t nsweeps, RngBase rb,
                      uint32_t* scratch, int chunk, cudaStream_t st, int* launches) {
  const int n = g->n;
  const bool in_smem = n <= sw_max_sites();
  const size_t smem = in_smem ? sw_smem_bytes(n) : 0;
  if (g->sw_ne > (int64_t)0x7FFFFFFF || (!in_smem && (!scratch || chunk < 1))) return cudaErrorInvalidValue;
  const int64_t ne = g->sw_ne;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t b_i = al((size_t)ne * 4 + 4), b_w = al((size_t)ne * 4 + 4);
  const char* base = g->sw_tables.as<char>();
  SwArgs a;
  a.ei = reinterpret_cast<const int32_t*>(base);
  a.ej = reinterpret_cast<const int32_t*>(base + b_i);
  a.w = reinterpret_cast<const float*>(base + 2 * b_i);
  a.pos = reinterpret_cast<const uint8_t*>(base + 2 * b_i + b_w);
  a.ne = (int)ne;
  a.n = n;
  a.spins = spins;
  a.betas = betas;
  a.nsweeps = nsweeps;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.rep0 = rb.rep0;
  if (in_smem) {
    cudaError_t e = cudaFuncSetAttribute(sw_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    sw_kernel<true><<<R, kSwThreads, smem, st>>>(a, nullptr);
    if (launches) ++*launches;
    return cudaGetLastError();
  }
  // replicas in chunks whose parent arrays fit the scratch ([chunk][n + 1])
  for (int r0 = 0; r0 < R; r0 += chunk) {
    SwArgs c = a;
    c.spins = spins + (size_t)r0 * n;
    c.rep0 = rb.rep0 + (uint32_t)r0;
    sw_kernel<false><<<std::min(chunk, R - r0), kSwThreads, 0, st>>>(c, scratch);
    if (launches) ++*launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int sw_max_sites() { return (220 * 1024 - 20) / 5; }

}  // namespace oj
