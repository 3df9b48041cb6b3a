// Local fields of a batch of dense instances on the tensor cores (tcgen05.mma
// kind::i8, accumulators in tensor memory):
//
//     F[m][r][j] = fp32( fp64(h_j) + u_m * sum_i q_ij s_ri ),   q_ij = J_ij / u_m
//
// The classical system's dE = -2 s (J s) of the reference
// (include/openjij/system/classical_ising.hpp:87-90, reset_dE), computed for
// every replica of every instance at once.  J enters as integers on a per-
// instance grid u_m = 2^e_m: couplings that are int8 multiples of 2^-p (the
// exact-field integer QUBOs) use q = J 2^p directly, one int8 "digit"; any
// other FP32 couplings are rounded (half to even) to the grid
// u_m = 2^(E - 26), E the binary exponent of max |J| (2^(E-1) <= max|J| < 2^E),
// and q is split into four balanced base-128 digits d_t in [-64, 63],
// q = sum_t d_t 128^t.  Each digit is one int8 x int8 -> int32 MMA pass with
// the +-1 spins; the passes are combined exactly in int64, converted exactly to
// FP64, scaled by u_m, added to h_j in FP64 and rounded once to FP32.  The
// result is a deterministic function of (J, h, s) that the CPU replay
// reproduces exactly, and it is within n u_m / 2 of the exact field (for the
// exact-field batches it is the exact field).
//
// Tiles: a CTA computes 128 sites (TMEM lanes) x NT replicas (TMEM columns per
// digit).  The digits are stored tiled in global memory in the canonical
// K-major layout of the MMA operand (8 x 16-byte core matrices, no swizzle), so
// one 16 KB tile (128 sites x 128 sites) is one bulk copy; the spins of the
// NT replicas are copied into shared memory by the threads in the same layout
// (16-byte cp.async pieces).  A ring of stages: the copies of the next K
// chunks overlap the MMAs of the current one.  Epilogue: tcgen05.ld of the accumulators, the exact
// combination above, coalesced FP32 stores of F (replica-major, sites
// contiguous), and in compare mode max |F_new - F_old| before the store (the
// drift of the sweep kernel's incremental fields).  Every wait is bounded:
// a wait that runs out sets *status and the kernel finishes without hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kTileSites = 128;                    // GEMM M: sites per tile (TMEM lanes)
constexpr int kChunk = 128;                        // GEMM K per stage: sites (bytes)
constexpr uint32_t kTileBytes = kTileSites * kChunk;  // one int8 digit tile
constexpr int kFieldThreads = 128;
constexpr long long kDrainLimit = 1ll << 26;  // iterations of a drain wait (the default wait limit too)

struct FieldArgs {
  const int8_t* digits;    // tiled digits, instance m at dtoff[m]: [D][mt][kt] tiles
  const int64_t* dtoff;    // [count] byte offsets
  const int32_t* uexp;     // [count] grid exponent e_m
  const float* h;          // padded fields
  const int64_t* hoff;
  const int32_t* n;
  const int32_t* reads;
  const int64_t* soff;     // spins of instance m: [reads][n] int8
  const int8_t* spins;
  float* F;                // [reads][npad] per instance
  const int64_t* foff;
  const int32_t* items;    // [nitems][3]: instance, site tile, replica tile
  int nitems;
  int compare;             // measure max |F_new - F_old| into *drift
  unsigned int* drift;     // float bits (non-negative values order as integers)
  int* status;
  long long wait_limit;    // iterations of a pipeline wait (0: give up at once)
};

using ojd::bulk_copy;
using ojd::mbar_init;
using ojd::mbar_wait;
using ojd::smem_u32;

// Matrix descriptor, K-major, no swizzle: LBO = distance of K-adjacent core
// matrices, SBO = distance of adjacent 8-row groups.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor: s8 x s8 -> s32, K-major A and B, M = 128, N = nn.
__device__ __forceinline__ uint32_t idesc_i8(int nn) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nn >> 3) << 17) | ((uint32_t)(kTileSites >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          dtmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = (int32_t)r[j];
}

// Ampere-style asynchronous copies into shared memory (the source aligned to
// the copy size); each thread waits for its own groups.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// byte offset of (row, k) in a canonical K-major tile of 128-byte rows
__host__ __device__ __forceinline__ uint32_t canon(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15));
}

template <int D, int NT>
struct FieldShape {
  // digits per stage: four-digit tiles with at most 256 accumulator columns go
  // two digits a stage, so that two CTAs share an SM (one's prologue and
  // epilogue overlap the other's copies); a K chunk is then two stages
  static constexpr int DS = (D > 1 && D * NT <= 256) ? 2 : D;
  static constexpr int H = D / DS;                       // stages per K chunk
  static constexpr uint32_t kA = DS * kTileBytes;        // digit tiles of one stage
  static constexpr uint32_t kB = NT * kChunk;            // spin tile of the stage's K chunk
  static constexpr uint32_t kStage = (kA + kB + 1023) / 1024 * 1024;
  // stages in the ring: two-digit stages as many as fit 110 KB (two CTAs an
  // SM), other four-digit tiles three when 220 KB hold them; one-digit tiles
  // keep two, so that two CTAs share an SM
  static constexpr int kStages = DS < D ? (3u * kStage <= 110u * 1024u ? 3 : 2)
                                        : ((D > 1 && 3u * kStage <= 220u * 1024u) ? 3 : 2);
  static constexpr uint32_t kCols = D * NT <= 32 ? 32 : (D * NT <= 64 ? 64 : (D * NT <= 128 ? 128 : (D * NT <= 256 ? 256 : 512)));
  static constexpr size_t kSmem = kStages * (size_t)kStage + 16 * kStages + 16;  // mbarriers, TMEM slot, abort flag
};

template <int D, int NT>
__global__ void __launch_bounds__(kFieldThreads, 1) field_tc_kernel(FieldArgs a) {
  using S = FieldShape<D, NT>;
  static_assert(D * NT <= 512, "accumulators exceed tensor memory");
  static_assert(NT % 16 == 0 && NT >= 16 && NT <= 256, "MMA N with M = 128");
  extern __shared__ __align__(1024) unsigned char sm[];
  const int item = blockIdx.x;
  if (item >= a.nitems) return;  // the whole CTA
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = a.items[3 * item], mt = a.items[3 * item + 1], nt = a.items[3 * item + 2];
  const int n = a.n[m], R = a.reads[m];
  const int nch = (n + kChunk - 1) / kChunk;
  const int npad = nch * kChunk;
  constexpr int ST = S::kStages;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + ST * S::kStage);  // full[ST], done[ST]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2 * ST);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(S::kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < 2 * ST; ++q) mbar_init(bar + q, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  // Ring of ST stages: the digit tiles of unit u + ST - 1 are copied while
  // unit u's spins are written and its MMAs run.  Pipeline waits use
  // a.wait_limit; one that runs out aborts the loop: no new copies or MMAs are
  // issued, the ones in flight are waited for with the default limit
  // (kDrainLimit), tensor memory is freed and F is left as it was.
  // thread 0's bookkeeping, bit s for stage s: phase parities of the full and
  // done barriers, and copies / MMA commits issued but not yet seen complete
  uint32_t ph_full = 0u, ph_done = 0u, pend_full = 0u, pend_done = 0u;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  if (tid == 0) *abort_flag = 0;
  const int8_t* dig = a.digits + a.dtoff[m];
  const int8_t* sp = a.spins + a.soff[m];
  const int r0 = nt * NT;
  // unit u = (K chunk u / H, digits (u % H) DS .. + DS - 1) is one stage
  constexpr int H = S::H, DS = S::DS;
  const int nu = nch * H;
  // digit tiles of unit u into stage u % ST (thread 0; the stage is free)
  auto issue_a = [&](int u) {
    const int s = u % ST, kc = u / H, t0 = (u % H) * DS;
    unsigned char* As = sm + s * S::kStage;
    ojd::mbar_expect_tx(bar + s, S::kA);
#pragma unroll
    for (int tt = 0; tt < DS; ++tt)
      bulk_copy(As + tt * kTileBytes, dig + ((size_t)((t0 + tt) * nch + mt) * nch + kc) * kTileBytes, kTileBytes,
                bar + s);
    pend_full |= 1u << s;
  };
  // spins of replicas r0..r0+NT-1 at sites 128 kc .. +127 into stage kc % ST
  // (every thread; the stage is free), 16 bytes a piece: asynchronous copies
  // where the piece is 16- or 4-byte aligned, else byte loads; zero past the
  // instance's reads and sites.  One commit group per call.
  auto issue_b = [&](int u) {
    const int kc = u / H;
    unsigned char* Bs = sm + (u % ST) * S::kStage + S::kA;
    for (int idx = tid; idx < NT * 8; idx += kFieldThreads) {
      const int rr = idx >> 3, pc = idx & 7;
      const int r = r0 + rr, k = kc * kChunk + 16 * pc;
      unsigned char* dst = Bs + canon(rr, 16 * pc);
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (r < R && k < n) {
        const int8_t* p = sp + (size_t)r * n + k;
        const int valid = min(16, n - k);
        const uintptr_t al = reinterpret_cast<uintptr_t>(p);
        if (valid == 16 && (al & 15u) == 0u) {
          cp_async16(dst, p);
          continue;
        }
        if (valid == 16 && (al & 3u) == 0u) {
#pragma unroll
          for (int q = 0; q < 4; ++q) cp_async4(dst + 4 * q, p + 4 * q);
          continue;
        }
        unsigned long long lo = 0ull, hi = 0ull;
        for (int e = 0; e < valid; ++e) {
          const unsigned long long bv = (unsigned long long)(uint8_t)p[e];
          if (e < 8) lo |= bv << (8 * e);
          else hi |= bv << (8 * (e - 8));
        }
        v = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
      }
      *reinterpret_cast<uint4*>(dst) = v;
    }
    cp_async_commit();
  };
  if (tid == 0)
    for (int u = 0; u < ST - 1 && u < nu; ++u) issue_a(u);
  for (int u = 0; u < ST - 1; ++u) {
    if (u < nu) issue_b(u);
    else cp_async_commit();  // an empty group keeps the count per chunk
  }
  for (int u = 0; u < nu; ++u) {
    const int s = u % ST, kc = u / H, t0 = (u % H) * DS;
    unsigned char* As = sm + s * S::kStage;
    unsigned char* Bs = As + S::kA;
    if (tid == 0 && u + ST - 1 < nu) {
      // the stage of unit u + ST - 1 last held unit u - 1: its MMAs first
      const int sn = (u + ST - 1) % ST;
      if ((pend_done >> sn) & 1u) {
        if (mbar_wait(bar + ST + sn, (ph_done >> sn) & 1u, a.wait_limit)) {
          ph_done ^= 1u << sn;
          pend_done &= ~(1u << sn);
        } else {
          *abort_flag = 1;
        }
      }
      if (!*abort_flag) issue_a(u + ST - 1);
    }
    __syncthreads();  // the stage of unit u + ST - 1 is free (unit u - 1's MMAs were seen complete)
    if (*abort_flag) break;
    if (u + ST - 1 < nu) issue_b(u + ST - 1);
    else cp_async_commit();
    cp_async_wait<ST - 1>();  // this thread's copies of unit u's spins have landed
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      if (mbar_wait(bar + s, (ph_full >> s) & 1u, a.wait_limit)) {
        ph_full ^= 1u << s;
        pend_full &= ~(1u << s);
        tc_fence_after();
        const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll
        for (int tt = 0; tt < DS; ++tt)
#pragma unroll
          for (int kk = 0; kk < kChunk / 32; ++kk)
            mma_i8(tbase + (uint32_t)((t0 + tt) * NT), desc_kmajor(a0 + tt * kTileBytes + kk * 256, 128, 1024),
                   desc_kmajor(b0 + kk * 256, 128, 1024), idesc_i8(NT), (kc | kk) ? 1u : 0u);
        mma_commit(bar + ST + s);
        pend_done |= 1u << s;
      } else {
        *abort_flag = 1;
      }
    }
  }
  // drain: every copy and MMA this CTA issued has completed before it goes on
  asm volatile("cp.async.wait_all;" ::: "memory");
  bool ok = true;
  if (tid == 0) {
    for (int q = 0; q < ST; ++q) {
      if ((pend_full >> q) & 1u) ok &= mbar_wait(bar + q, (ph_full >> q) & 1u, kDrainLimit);
      if ((pend_done >> q) & 1u) ok &= mbar_wait(bar + ST + q, (ph_done >> q) & 1u, kDrainLimit);
    }
    if (*abort_flag || !ok) atomicExch(a.status, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (*abort_flag) {
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(S::kCols));
    return;
  }
  // ---- epilogue: warp w reads TMEM lanes 32w..32w+31 = sites of the tile
  const int site = mt * kTileSites + 32 * warp + lane;
  const float hf = a.h[a.hoff[m] + site];  // zero past n (padding)
  const double hv = (double)hf;
  // 2^e: multiplying by it is exact (the products stay normal)
  const double scale = ldexp(1.0, a.uexp[m]);
  const float scale_f = (float)scale;
  float* Fm = a.F + a.foff[m] + site;
  float dmax = 0.0f;
  for (int j0 = 0; j0 < NT; j0 += 16) {
    if (r0 + j0 >= R) break;  // warp-uniform
    long long tot[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) tot[j] = 0;
#pragma unroll
    for (int t = 0; t < D; ++t) {
      int32_t acc[16];
      tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(t * NT + j0), acc);
#pragma unroll
      for (int j = 0; j < 16; ++j) tot[j] += (long long)acc[j] * (1ll << (7 * t));
    }
    // compare mode: the sweep kernel's fields of the 16 replicas, all loaded
    // before any store (no load waits behind the previous replica's store)
    float old[16];
    if (a.compare && site < n) {
#pragma unroll
      for (int j = 0; j < 16; ++j) old[j] = r0 + j0 + j < R ? Fm[(size_t)(r0 + j0 + j) * npad] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int r = r0 + j0 + j;
      if (r >= R) break;
      // one int8 digit: the exact-field integer batches, where h + 2^e acc is
      // an FP32 value and the FP32 operations are exact (the same value)
      const float f = D == 1 ? __fadd_rn(hf, __fmul_rn(__ll2float_rn(tot[j]), scale_f))
                             : __double2float_rn(__dadd_rn(hv, __dmul_rn(__ll2double_rn(tot[j]), scale)));
      float* dst = Fm + (size_t)r * npad;
      if (a.compare && site < n) dmax = fmaxf(dmax, fabsf(f - old[j]));
      *dst = f;
    }
  }
  if (a.compare) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if (lane == 0 && dmax > 0.0f) atomicMax(a.drift, __float_as_uint(dmax));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(S::kCols));
}

template <int D, int NT>
cudaError_t launch_field_dn(const FieldArgs& a, cudaStream_t st) {
  using S = FieldShape<D, NT>;
  auto kern = field_tc_kernel<D, NT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem);
  if (e != cudaSuccess) return e;
  // every CTA resident on an SM must find its tensor-memory columns
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFieldThreads, S::kSmem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1 || (size_t)per_sm * S::kCols > 512) return cudaErrorInvalidConfiguration;
  kern<<<a.nitems, kFieldThreads, S::kSmem, st>>>(a);
  return cudaGetLastError();
}

template <int D>
cudaError_t launch_field_d(const FieldArgs& a, int NT, cudaStream_t st) {
  switch (NT) {
    case 16: return launch_field_dn<D, 16>(a, st);
    case 32: return launch_field_dn<D, 32>(a, st);
    case 64: return launch_field_dn<D, 64>(a, st);
    case 128: return launch_field_dn<D, 128>(a, st);
    default:
      if constexpr (D == 1) return launch_field_dn<1, 256>(a, st);
      return cudaErrorInvalidValue;
  }
}

}  // namespace

int field_tc_tile_replicas(const oj_batch* b, int max_reads) {
  const int cap = b->ndig == 1 ? 256 : 128;
  int nt = 16;
  while (nt < max_reads && nt < cap) nt *= 2;
  return nt;
}

void field_tc_items(const oj_batch* b, const int32_t* reads, const std::vector<int>& order, int NT,
                    std::vector<int32_t>& items) {
  items.clear();
  for (int m : order) {
    const int n = b->n[m];
    if (n == 0 || reads[m] == 0) continue;
    const int nch = (n + kChunk - 1) / kChunk;
    for (int mt = 0; mt < nch; ++mt)
      for (int nt = 0; nt * NT < reads[m]; ++nt) {
        items.push_back(m);
        items.push_back(mt);
        items.push_back(nt);
      }
  }
}

cudaError_t launch_field_tc(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff, const int8_t* spins,
                            float* F, const int64_t* d_foff, const int32_t* d_items, int nitems, int NT, bool compare,
                            unsigned int* d_drift, int* d_status, long long wait_limit, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  FieldArgs a;
  a.digits = b->d_dig.as<int8_t>();
  a.dtoff = b->d_dtoff.as<int64_t>();
  a.uexp = b->d_uexp.as<int32_t>();
  a.h = b->d_h.as<float>();
  a.hoff = b->d_hoff.as<int64_t>();
  a.n = b->d_n.as<int32_t>();
  a.reads = d_reads;
  a.soff = d_soff;
  a.spins = spins;
  a.F = F;
  a.foff = d_foff;
  a.items = d_items;
  a.nitems = nitems;
  a.compare = compare ? 1 : 0;
  a.drift = d_drift;
  a.status = d_status;
  a.wait_limit = wait_limit >= 0 ? wait_limit : kDrainLimit;
  return b->ndig == 1 ? launch_field_d<1>(a, NT, st) : launch_field_d<4>(a, NT, st);
}

// Host side: the grid of every instance and its digits, tiled.  Instance m's
// couplings J32 (n x npad, row-major, FP32, zero padding) become q_ij on the
// grid 2^uexp[m]; with j8 (int8 couplings J 2^p) one digit q = J8 and
// uexp = -p, otherwise four balanced base-128 digits on 2^(E - 26).
cudaError_t field_tc_prepare(oj_batch* b, const std::vector<float>& J32, const std::vector<int64_t>& joff,
                             const std::vector<int8_t>* J8, int pmax) {
  const int count = b->count;
  const int D = (J8 && b->j8) ? 1 : 4;
  std::vector<int64_t> dtoff(std::max(count, 1), 0);
  std::vector<int32_t> uexp(std::max(count, 1), 0);
  int64_t total = 0;
  for (int m = 0; m < count; ++m) {
    const int64_t nch = ((int64_t)b->n[m] + kChunk - 1) / kChunk;
    dtoff[m] = total;
    total += (int64_t)D * nch * nch * kTileBytes;
  }
  std::vector<int8_t> tiles((size_t)std::max<int64_t>(total, 16), 0);
  // one-chunk batches with four digits also keep q as int32 for the sweep
  // kernel's own recompute (sa_batch1_kernel)
  const bool q32 = D == 4 && b->max_n <= kChunk;
  std::vector<int32_t> Q(q32 ? std::max<size_t>(J32.size(), 4) : 0, 0);
  for (int m = 0; m < count; ++m) {
    const int n = b->n[m];
    if (n == 0) continue;
    const int nch = (n + kChunk - 1) / kChunk, npad = nch * kChunk;
    const float* Jm = J32.data() + joff[m];
    int e = 0;
    if (D == 1) {
      e = -pmax;
    } else {
      float amax = 0.0f;
      for (int64_t q = 0; q < (int64_t)n * npad; ++q) amax = std::max(amax, std::fabs(Jm[q]));
      int E = 0;
      if (amax > 0.0f) std::frexp((double)amax, &E);  // 2^(E-1) <= amax < 2^E
      e = amax > 0.0f ? E - 26 : 0;
    }
    uexp[m] = e;
    int8_t* base = tiles.data() + dtoff[m];
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int mt = j / kChunk, kt = i / kChunk;
        const uint32_t off = canon(j % kChunk, i % kChunk);
        if (D == 1) {
          base[((size_t)mt * nch + kt) * kTileBytes + off] = (*J8)[(size_t)(joff[m] + (int64_t)j * npad + i)];
          continue;
        }
        int64_t q = (int64_t)std::nearbyint(std::ldexp((double)Jm[(size_t)j * npad + i], -e));
        if (q32) Q[(size_t)joff[m] + (size_t)i * npad + j] = (int32_t)q;  // element [i][j] = q_ji
        for (int t = 0; t < 4; ++t) {
          const int64_t d = ((q + 64) & 127) - 64;
          q = (q - d) >> 7;
          base[((size_t)(t * nch + mt) * nch + kt) * kTileBytes + off] = (int8_t)d;
        }
      }
  }
  b->ndig = D;
  cudaError_t err;
  if (q32) {
    if ((err = b->d_q32.ensure(Q.size() * 4)) != cudaSuccess) return err;
    if ((err = cudaMemcpy(b->d_q32.ptr, Q.data(), Q.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return err;
  }
  if ((err = b->d_dig.ensure(tiles.size())) != cudaSuccess) return err;
  if ((err = cudaMemcpy(b->d_dig.ptr, tiles.data(), tiles.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return err;
  if ((err = b->d_dtoff.ensure(dtoff.size() * 8)) != cudaSuccess) return err;
  if ((err = cudaMemcpy(b->d_dtoff.ptr, dtoff.data(), dtoff.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess)
    return err;
  if ((err = b->d_uexp.ensure(uexp.size() * 4)) != cudaSuccess) return err;
  return cudaMemcpy(b->d_uexp.ptr, uexp.data(), uexp.size() * 4, cudaMemcpyHostToDevice);
}

}  // namespace oj
