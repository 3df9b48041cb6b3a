// Sequential dense SA with delayed tensor-core field updates (tcgen05 + TMEM).
//
// Same update order, random stream and acceptance rule as the plain dense
// kernel (the reference's single_spin_flip.hpp:66-95: sites 0..n-1 in order,
// accept when dE <= 0 or beta*dE < -ln u), but the O(n) field update of every
// accepted flip is deferred and batched into a tensor-core GEMM:
//
//  * A thread block cluster of P CTAs owns a tile of 128 replicas.  The local
//    fields F (128 replicas x n spins, FP32) live in tensor memory, split by
//    spin columns: CTA c holds columns [c*Ncta, (c+1)*Ncta), one TMEM lane per
//    replica.
//  * The sweep walks blocks of 32 spins.  The CTA owning a block reads its 32
//    field columns from TMEM (thread = replica), adds h, and makes the 32
//    decisions in order, updating the in-block fields exactly with an FP32
//    32x32 tile of J.  The block's flips dS (128 x 32, {-2, 0, +2}, exact in
//    BF16) go to every CTA of the cluster through distributed shared memory.
//  * Every CTA then issues  F[:, own cols] += dS (128x32) * J[block, own cols]
//    (32 x Ncta, BF16, fetched by bulk copy) with tcgen05.mma, FP32
//    accumulation in TMEM.  For half-integer |J| <= 256 every product and sum
//    is exact, so the fields — and the trajectories — equal the plain kernel's
//    bit for bit.  Real couplings use a hi/lo BF16 split of J (two MMAs) and a
//    full recompute F = S*J every `recompute` sweeps to cancel drift.
//  * Four more warps per CTA draw the block's -ln(u) values ahead of time.
//
// All waits are bounded: a wait that runs out sets *status and the kernel
// runs to its end without touching memory outside its buffers.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace cg = cooperative_groups;

namespace oj {
namespace {

constexpr int kBlk = 32;          // spins per block (GEMM K)
constexpr int kTile = 128;        // replicas per cluster (GEMM M, TMEM lanes)
constexpr int kThreads = 256;     // warps 0-3: sweep, warps 4-7: random numbers
constexpr int kMaxNcta = 512;     // TMEM columns per CTA
constexpr long long kWaitLimit = 1ll << 26;

struct TcArgs {
  int n, nblk, bpc, Ncta, P;
  const uint8_t* bt_hi;  // [nblk][P][Ncta*32] bf16, canonical K-major tiles
  const uint8_t* bt_lo;  // same, J - bf16(J); null for exact couplings
  const float* jblk;     // [nblk][32][32] FP32 in-block couplings
  const float* h;        // [nblk*32]
  int8_t* spins;         // [R][n]
  int R;
  const float* betas;    // [nsweeps]
  int64_t nsweeps;
  int recompute;         // recompute F every this many sweeps (0: only at start)
  ojd::Keys keys;
  uint32_t sweep0, rep0;
  int* status;
  unsigned long long* flips;  // accepted-flip counter, or null
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// tcgen05 shared-memory matrix descriptor, K-major, no swizzle (8x16B core matrices).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor: BF16 x BF16 -> FP32, K-major A and B, M = 128.
__device__ __forceinline__ uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

// byte offset of (row, k) in a K-major canonical tile with K = 32 (LBO 128 B, SBO 512 B)
__host__ __device__ __forceinline__ int canon_off(int row, int k) {
  return (row >> 3) * 512 + (row & 7) * 16 + (k >> 3) * 128 + (k & 7) * 2;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

// Bounded wait on phase parity `ph`; returns false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t ph) {
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(ph)
        : "memory");
    if (done) return true;
  }
  return false;
}

// global -> shared bulk copy completing `bytes` of transaction count on `bar`
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          dtmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// -ln(u) of replica r for the 32 sites of block kb in sweep k, written to
// L[j][t] (t = r - tile base).  One Philox call serves four replicas of a site
// (the stream u(r,k,i) = Philox(i, k, r>>2)[r&3]); a rotation inside each
// group of four lanes hands every lane its own four values per call.
__device__ __forceinline__ void produce_L(float* L, int t, uint32_t r, int kb, uint32_t k, const ojd::Keys& K,
                                          int q0, int q1, int qstep) {
  const int lane = threadIdx.x & 31, m = lane & 3, qb = lane & ~3;
#pragma unroll 1
  for (int q = q0; q < q1; q += qstep) {
    const uint32_t site = (uint32_t)(kb * kBlk + 4 * q + m);
    const ojd::u4 v = ojd::philox(site, k, r >> 2, ojd::TAG_SA, K);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int idx = (m - s) & 3;
      const uint32_t val = idx == 0 ? v.x : (idx == 1 ? v.y : (idx == 2 ? v.z : v.w));
      const int src = (m + s) & 3;
      const uint32_t got = __shfl_sync(0xffffffffu, val, qb + src);
      L[(4 * q + src) * kTile + t] = ojd::neglog(got);
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1) sa_dense_tc_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int cta = (int)cl.block_rank();
  const int tile = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int Ncta = a.Ncta, nblk = a.nblk, bpc = a.bpc;
  const bool has_lo = a.bt_lo != nullptr;
  const uint32_t btile = (uint32_t)Ncta * kBlk * 2;  // bytes of one B tile
  // ---- shared memory carve-up
  unsigned char* A = sm;                                     // 2 x 8 KB MMA A operand (dS / S tiles)
  unsigned char* Bh = A + 2 * 8192;                          // 2 x btile (hi)
  unsigned char* Bl = Bh + 2 * btile;                        // 2 x btile (lo), if any
  float* Jb = reinterpret_cast<float*>(Bl + (has_lo ? 2 * btile : 0));  // 2 x 32 x 32 FP32
  float* Lb = Jb + 2 * kBlk * kBlk;                          // 2 x 32 x 128 FP32
  float* Hb = Lb + 2 * kBlk * kTile;                         // 2 x 32 FP32
  uint32_t* bits = reinterpret_cast<uint32_t*>(Hb + 2 * kBlk);  // [nblk][128]
  uint64_t* bar = reinterpret_cast<uint64_t*>(bits + (size_t)nblk * kTile);  // mma, bfull[2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 4);
  uint64_t* bar_mma = bar;
  uint64_t* bar_full = bar + 1;  // [2]

  const uint32_t tmem_cols = Ncta <= 32 ? 32 : (Ncta <= 64 ? 64 : (Ncta <= 128 ? 128 : (Ncta <= 256 ? 256 : 512)));
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(bar_mma, 1);
    mbar_init(bar_full, 1);
    mbar_init(bar_full + 1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // ---- spins of the tile -> bit words (bit j of bits[kb][t] set iff s = -1)
  const int r_base = tile * kTile;
  for (int idx = tid; idx < nblk * kTile; idx += kThreads) {
    const int kb = idx / kTile, t = idx % kTile;
    const int r = r_base + t;
    uint32_t w = 0;
    if (r < a.R) {
      const int8_t* sp = a.spins + (size_t)r * a.n;
      for (int j = 0; j < kBlk; ++j) {
        const int i = kb * kBlk + j;
        if (i < a.n && sp[i] < 0) w |= 1u << j;
      }
    }
    bits[kb * kTile + t] = w;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  uint32_t ph_mma = 0, ph_full[2] = {0, 0};  // phase parities (meaningful in thread 0)
  bool ok = true;
  unsigned long long nflip = 0;

  // B tile of block kb (hi and lo) into buffer `buf` (thread 0 only)
  auto load_b = [&](int kb, int buf) {
    const size_t off = ((size_t)kb * a.P + cta) * btile;
    const uint32_t total = btile * (has_lo ? 2u : 1u);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar_full + buf)),
                 "r"(total) : "memory");
    bulk_copy(Bh + buf * btile, a.bt_hi + off, btile, bar_full + buf);
    if (has_lo) bulk_copy(Bl + buf * btile, a.bt_lo + off, btile, bar_full + buf);
  };
  auto wait_full = [&](int buf) {
    ok &= mbar_wait(bar_full + buf, ph_full[buf]);
    ph_full[buf] ^= 1u;
  };
  auto wait_mma = [&]() {
    ok &= mbar_wait(bar_mma, ph_mma);
    ph_mma ^= 1u;
  };
  // F[:, own cols] (+)= A(buf) * B(buf) for hi (and lo)
  auto issue_mma = [&](int abuf, int bbuf, uint32_t acc_first) {
    const uint32_t a0 = smem_u32(A + abuf * 8192);
    for (int pass = 0; pass < (has_lo ? 2 : 1); ++pass) {
      const uint32_t b0 = smem_u32((pass ? Bl : Bh) + bbuf * btile);
      for (int n0 = 0; n0 < Ncta; n0 += 256) {
        const int nn = min(256, Ncta - n0);
        for (int j = 0; j < 2; ++j) {
          const uint64_t da = desc_kmajor(a0 + j * 256, 128, 512);
          const uint64_t db = desc_kmajor(b0 + (n0 >> 3) * 512 + j * 256, 128, 512);
          mma_bf16(tbase + n0, da, db, idesc_bf16(nn), (pass | j) ? 1u : acc_first);
        }
      }
    }
    mma_commit(bar_mma);
  };
  // A tile row t = the tile's spins of block kb as BF16 +-1 (sweepers)
  auto write_s_tile = [&](int kb, int t) {
    const uint32_t w = bits[kb * kTile + t];
    unsigned char* row = A + (t >> 3) * 512 + (t & 7) * 16;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t pk[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k0 = 8 * q + 2 * e;
        const uint32_t lo = ((w >> k0) & 1u) ? 0xBF80u : 0x3F80u;  // -1 / +1 in BF16
        const uint32_t hi = ((w >> (k0 + 1)) & 1u) ? 0xBF80u : 0x3F80u;
        pk[e] = lo | (hi << 16);
      }
      *reinterpret_cast<uint4*>(row + q * 128) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  };
  // F = S * J over all blocks (every CTA, serially; buffers drained after)
  auto recompute = [&]() {
    for (int kb = 0; kb < nblk; ++kb) {
      if (tid == 0) load_b(kb, 0);
      if (tid < kTile) write_s_tile(kb, tid);
      proxy_fence();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (tid == 0) {
        wait_full(0);
        issue_mma(0, 0, kb > 0 ? 1u : 0u);
        wait_mma();
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
  };

  recompute();
  // Blocks are owned round-robin: block kb belongs to CTA kb % P.  The g-th
  // block owned by this CTA (counting across sweeps) is block (g % bpc)*P + cta
  // of sweep g / bpc; its -ln(u) values and in-block couplings are prepared by
  // the producer warps into slot g & 1 while other CTAs own the sweep.
  const int64_t own_total = a.nsweeps * bpc;
  // part `part` of `parts` of the inputs of owned block g, by all 256 threads:
  // thread = (replica tid % 128, half tid / 128); the block's 8 groups of four
  // sites are split over the parts and the two halves.
  auto produce = [&](int64_t g, int part, int parts) {
    const int okb = (int)(g % bpc) * a.P + cta;
    const uint32_t ok_sweep = a.sweep0 + (uint32_t)(g / bpc);
    const int slot = (int)(g & 1);
    if (part == 0) {
      float* Jd = Jb + slot * kBlk * kBlk;
      for (int e = tid; e < kBlk * kBlk; e += kThreads) Jd[e] = a.jblk[(size_t)okb * kBlk * kBlk + e];
      if (tid < kBlk) Hb[slot * kBlk + tid] = a.h[okb * kBlk + tid];
    }
    const int q0 = (8 * part) / parts, q1 = (8 * (part + 1)) / parts;
    const int t = tid & (kTile - 1), half = tid >> 7;
    produce_L(Lb + slot * kBlk * kTile, t, a.rep0 + r_base + t, okb, ok_sweep, a.keys, q0 + half, q1, 2);
  };
  int64_t own_count = 0;    // owned blocks swept so far
  int64_t produced = 0;     // owned blocks whose inputs are ready
  int part = 0;             // parts of the next owned block done
  const int parts = a.P > 1 ? a.P - 1 : 1;
  if (own_total > 0) produce(0, 0, 1);
  produced = 1;
  if (tid == 0) load_b(0, 0);
  __syncthreads();
  cluster_arrive();
  cluster_wait();

  int64_t gblk = 0;  // global block counter (buffer parity)
  for (int64_t k = 0; k < a.nsweeps; ++k) {
    const float beta = a.betas[k];
    if (a.recompute > 0 && k > 0 && (k % a.recompute) == 0) {
      // drain: the next-block load issued at the end of the last sweep
      if (tid == 0) wait_full((int)(gblk & 1));
      __syncthreads();
      recompute();
      if (tid == 0) load_b(0, (int)(gblk & 1));
      cluster_arrive();
      cluster_wait();
    }
    for (int kb = 0; kb < nblk; ++kb, ++gblk) {
      const int buf = (int)(gblk & 1);
      const int owner = kb % a.P;
      // prefetch the next block's B tile into the other buffer (free: its last
      // MMAs completed before the previous block's cluster barrier)
      if (tid == 0) {
        const int nkb = kb + 1 < nblk ? kb + 1 : 0;
        const bool more = kb + 1 < nblk || k + 1 < a.nsweeps;
        if (more) load_b(nkb, buf ^ 1);
      }
      if (owner == cta) {
        const int slot = (int)(own_count & 1);
        if (tid < kTile) {
          const float* Jd = Jb + slot * kBlk * kBlk;
          float f[32];
          tmem_ld32(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)((kb / a.P) * kBlk), f);
#pragma unroll
          for (int j = 0; j < 32; ++j) f[j] = __fadd_rn(f[j], Hb[slot * kBlk + j]);
          const uint32_t w = bits[kb * kTile + tid];
          uint32_t flips = 0;
          const float* L = Lb + slot * kBlk * kTile;
          // Four sub-blocks of 8 sites: inside a sub-block every decision
          // updates the fields still ahead in it at once (short dependent
          // chain); the sub-block's flips then reach the later fields as one
          // rank-8 update.  Every field accumulates c_j * J_jm in increasing
          // j, one rounding each (c_j * J_jm is exact), as in the sequential
          // kernel.
          float c[32], Lr[32];
          const int nvalid = a.n - kb * kBlk;  // sites of this block below n
#pragma unroll
          for (int j = 0; j < 32; ++j) Lr[j] = j < nvalid ? L[j * kTile + tid] : -1.0f;
#pragma unroll
          for (int sb = 0; sb < 4; ++sb) {
#pragma unroll
            for (int j = 8 * sb; j < 8 * sb + 8; ++j) {
              const bool neg = (w >> j) & 1u;
              const float s2 = neg ? 2.0f : -2.0f;  // -2 s: dE = -2 s f, and the flip's dS
              const float dE = s2 * f[j];
              // padded sites (L = -1) never flip
              const bool acc = Lr[j] >= 0.0f && (dE <= 0.0f || __fmul_rn(beta, dE) < Lr[j]);
              c[j] = acc ? s2 : 0.0f;
              flips |= acc ? (1u << j) : 0u;
#pragma unroll
              for (int m = j + 1; m < 8 * sb + 8; ++m) f[m] = __fmaf_rn(c[j], Jd[j * kBlk + m], f[m]);
            }
#pragma unroll
            for (int m = 8 * sb + 8; m < 32; ++m) {
#pragma unroll
              for (int j = 8 * sb; j < 8 * sb + 8; ++j) f[m] = __fmaf_rn(c[j], Jd[j * kBlk + m], f[m]);
            }
          }
          const uint32_t nw = w ^ flips;
          if (r_base + tid < a.R) nflip += __popc(flips);
          // dS row (BF16: +-2 where flipped = new s - old s) into every CTA's A buffer
          uint32_t pk[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int k0 = 2 * e;
            const uint32_t d0 = ((flips >> k0) & 1u) ? (((nw >> k0) & 1u) ? 0xC000u : 0x4000u) : 0u;
            const uint32_t d1 = ((flips >> (k0 + 1)) & 1u) ? (((nw >> (k0 + 1)) & 1u) ? 0xC000u : 0x4000u) : 0u;
            pk[e] = d0 | (d1 << 16);
          }
          const int roff = (tid >> 3) * 512 + (tid & 7) * 16;
          for (int p = 0; p < a.P; ++p) {
            unsigned char* Ab = cl.map_shared_rank(A, p) + buf * 8192 + roff;
#pragma unroll
            for (int q = 0; q < 4; ++q)
              *reinterpret_cast<uint4*>(Ab + q * 128) = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
            *cl.map_shared_rank(bits + kb * kTile + tid, p) = nw;
          }
          asm volatile("fence.proxy.async.shared::cluster;" ::: "memory");
        }
        ++own_count;
      } else if (produced <= own_count && produced < own_total) {
        produce(produced, part, parts);
        if (++part == parts) {
          part = 0;
          ++produced;
        }
      }
      if (a.P == 1 && produced <= own_count && produced < own_total) {
        // single-CTA cluster: no foreign blocks to hide behind
        __syncthreads();
        produce(produced, 0, 1);
        ++produced;
      }
      tc_fence_before();
      cluster_arrive();
      cluster_wait();
      tc_fence_after();
      if (tid == 0) {
        proxy_fence();
        wait_full(buf);
        issue_mma(buf, buf, 1u);
        wait_mma();
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
  }
  // ---- write back the spins of the owned blocks
  for (int idx = tid; idx < bpc * kTile; idx += kThreads) {
    const int kb = (idx / kTile) * a.P + cta, t = idx % kTile;
    const int r = r_base + t;
    if (kb >= nblk || r >= a.R) continue;
    const uint32_t w = bits[kb * kTile + t];
    int8_t* sp = a.spins + (size_t)r * a.n;
    for (int j = 0; j < kBlk; ++j) {
      const int i = kb * kBlk + j;
      if (i < a.n) sp[i] = ((w >> j) & 1u) ? (int8_t)-1 : (int8_t)1;
    }
  }
  if (!ok && tid == 0) atomicExch(a.status, 1);
  ojd::add_flips(a.flips, nflip);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(tmem_cols));
  cluster_arrive();
  cluster_wait();
}

}  // namespace

size_t dense_tc_smem(const TcPlan& pl) {
  const size_t btile = (size_t)pl.ncta * kBlk * 2;
  return 2 * 8192 + 2 * btile * (pl.exact ? 1 : 2) + 2 * kBlk * kBlk * 4 + 2 * kBlk * kTile * 4 + 2 * kBlk * 4 +
         (size_t)pl.nblk * kTile * 4 + 4 * 8 + 16;
}

// Host-side tiling of J for the tensor-core kernel.
cudaError_t dense_tc_prepare(oj_graph* g, std::string* why) {
  if (g->tc) return cudaSuccess;
  const int n = g->n;
  const bool exact = g->info.integer_exact != 0;
  // non-exact couplings carry a second (lo) B tile per buffer: narrower CTAs
  const int maxc = exact ? kMaxNcta : kMaxNcta / 2;
  int P = (n + maxc - 1) / maxc;
  if (P < 1) P = 1;
  const int ncta = ((n + P - 1) / P + kBlk - 1) / kBlk * kBlk;
  if (ncta > maxc || P > 8) {
    if (why) *why = exact ? "tensor-core dense kernel supports n <= 4096" : "tensor-core dense kernel supports n <= 2048 for non-integer couplings";
    return cudaErrorInvalidValue;
  }
  const int bpc = ncta / kBlk;
  const int nblk = P * bpc;
  const int npad = nblk * kBlk;
  // dense FP32 / FP64 J on the host
  std::vector<double> J((size_t)npad * npad, 0.0);
  for (int i = 0; i < n; ++i)
    for (int q = g->rp[i]; q < g->rp[i + 1]; ++q) J[(size_t)i * npad + g->ci[q]] = g->val64[q];
  const size_t tile_elems = (size_t)ncta * kBlk;
  std::vector<__nv_bfloat16> hi((size_t)nblk * P * tile_elems), lo(exact ? 0 : hi.size());
  for (int kb = 0; kb < nblk; ++kb)
    for (int c = 0; c < P; ++c) {
      const size_t base = ((size_t)kb * P + c) * tile_elems;
      for (int row = 0; row < ncta; ++row)
        for (int k = 0; k < kBlk; ++k) {
          const int i = kb * kBlk + k, j = ((row / kBlk) * P + c) * kBlk + row % kBlk;
          const float v = (float)J[(size_t)i * npad + j];
          const __nv_bfloat16 bh = __float2bfloat16_rn(v);
          const size_t e = base + canon_off(row, k) / 2;
          hi[e] = bh;
          if (!exact) lo[e] = __float2bfloat16_rn(v - __bfloat162float(bh));
        }
    }
  std::vector<float> jb((size_t)nblk * kBlk * kBlk, 0.0f), h(npad, 0.0f);
  for (int kb = 0; kb < nblk; ++kb)
    for (int a = 0; a < kBlk; ++a)
      for (int b = 0; b < kBlk; ++b)
        jb[((size_t)kb * kBlk + a) * kBlk + b] = (float)J[(size_t)(kb * kBlk + a) * npad + kb * kBlk + b];
  for (int i = 0; i < n; ++i) h[i] = g->h[i];
  {
    TcPlan probe;
    probe.P = P;
    probe.ncta = ncta;
    probe.nblk = nblk;
    probe.exact = exact;
    if (dense_tc_smem(probe) > 227 * 1024) {
      if (why) *why = "tensor-core dense kernel: tiles do not fit shared memory";
      return cudaErrorInvalidValue;
    }
  }
  auto plan = std::make_unique<TcPlan>();
  plan->P = P;
  plan->ncta = ncta;
  plan->bpc = bpc;
  plan->nblk = nblk;
  plan->exact = exact;
  cudaError_t e;
  auto up = [&](DevBuf& b, const void* src, size_t bytes) -> cudaError_t {
    cudaError_t r = b.ensure(std::max<size_t>(bytes, 16));
    if (r != cudaSuccess || bytes == 0) return r;
    return cudaMemcpy(b.ptr, src, bytes, cudaMemcpyHostToDevice);
  };
  if ((e = up(plan->bt_hi, hi.data(), hi.size() * 2)) != cudaSuccess) return e;
  if (!exact && (e = up(plan->bt_lo, lo.data(), lo.size() * 2)) != cudaSuccess) return e;
  if ((e = up(plan->jblk, jb.data(), jb.size() * 4)) != cudaSuccess) return e;
  if ((e = up(plan->h, h.data(), h.size() * 4)) != cudaSuccess) return e;
  if ((e = plan->status.ensure(16)) != cudaSuccess) return e;
  g->tc = std::move(plan);
  return cudaSuccess;
}

cudaError_t launch_sa_dense_tc(const oj_graph* g, int R, int8_t* spins, const float* betas, int64_t nsweeps,
                               RngBase rb, int recompute, cudaStream_t st, int* launches) {
  const TcPlan& pl = *g->tc;
  TcArgs a;
  a.n = g->n;
  a.nblk = pl.nblk;
  a.bpc = pl.bpc;
  a.Ncta = pl.ncta;
  a.P = pl.P;
  a.bt_hi = pl.bt_hi.as<uint8_t>();
  a.bt_lo = pl.exact ? nullptr : pl.bt_lo.as<uint8_t>();
  a.jblk = pl.jblk.as<float>();
  a.h = pl.h.as<float>();
  a.spins = spins;
  a.R = R;
  a.betas = betas;
  a.nsweeps = nsweeps;
  a.recompute = pl.exact ? 0 : recompute;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.rep0 = rb.rep0;
  a.status = pl.status.as<int>();
  a.flips = rb.flips;
  const size_t smem = dense_tc_smem(pl);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  auto kern = sa_dense_tc_kernel;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(pl.P, (R + kTile - 1) / kTile, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = pl.P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (launches) ++*launches;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

}  // namespace oj
