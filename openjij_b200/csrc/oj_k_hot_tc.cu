// Flip-heavy first sweeps of exact-field dense instances on the tensor cores.
//
// From a random state the first sweeps of an anneal flip a large share of the
// spins (on a dense n = 2048 integer QUBO about 900 per replica in the first
// sweep), and the dense-jump kernel pays one coupling-row read from L2 per flip
// and per replica.  This kernel runs those sweeps with the replicas of a tile
// in lock step, one 128-site chunk at a time:
//
//   * the int32 fields acc[j][r] (F = h + 2^e acc, exact for these batches) of
//     all n sites of RT = 16 replicas live in tensor memory, chunk c' at
//     columns 16 c' (lanes = the chunk's sites; two CTAs share an SM);
//   * a chunk is decided replica by replica exactly as the jump kernel decides
//     it (same uniforms, same acceptance test, same site order, the chunk's own
//     fields updated after every flip from the diagonal coupling tile in shared
//     memory), and each replica's spin changes ds in {0, +-2} form one row of
//     an int8 tile;
//   * the chunk's changes then reach every field of every replica as int8 MMAs
//     acc[c'] += J[c', c] ds (tcgen05.mma kind::i8, M = 128 sites, N = 16
//     replicas, K = 128), the coupling tiles streamed through a ring of shared-
//     memory stages by bulk copies (the field kernel's tiles, canonical K-major).
//
// For these batches every partial sum is exact, so the fields are the jump
// kernel's fields bit for bit and the spins are the sequential sweep's.  A tile
// of replicas leaves after the first sweep in which it flipped fewer than
// n/16 spins per replica (or after the last sweep): it stores its spins and
// FP32 fields and the sweep to continue from, and the dense-jump / batched
// kernel takes the remaining sweeps from there.  Its cost per sweep falls
// with the number of flips (each reads an n-site row), this kernel's does not
// (n^2 MMA work); on a dense n = 2048 QUBO the two cross between 96 and 256
// flips per replica and sweep (measured: sweep 1 takes 0.94 ms here against
// 2.73 ms in the jump kernel for 4096 replicas, sweep 2 0.32 ms against
// 0.83 ms).
//
// Warps 0..7 decide (warps 0..3 also move the fields of the next chunk from
// tensor memory into shared memory); warp 8 issues the copies and the MMAs.
// Every wait is bounded: one that runs out sets *status, the CTA stops at the
// next chunk, drains its copies and MMAs and writes nothing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kRT = 16;                 // replicas per CTA (MMA N): two CTAs share an SM
constexpr int kDecWarps = 8;            // deciding warps
constexpr int kHotThreads = (kDecWarps + 1) * 32;
constexpr int kStages = 4;              // ring of coupling tiles
constexpr int kAhead = kStages - 2;     // tiles in flight ahead of the MMAs
constexpr int kHotMaxChunks = 16;       // n <= 2048: nch x 32 accumulator columns <= 512
constexpr uint32_t kTile = 128 * 128;   // one int8 tile
constexpr uint32_t kBTile = kRT * 128;  // one tile of spin changes
constexpr int kSwWords = 32 * ((kHotMaxChunks + 7) / 8);  // spin words per replica
constexpr long long kHotDrain = 1ll << 26;

// dynamic shared memory layout (bytes)
constexpr uint32_t kOffRing = 0;
constexpr uint32_t kOffDiag = kOffRing + kStages * kTile;
constexpr uint32_t kOffB = kOffDiag + 2 * kTile;
constexpr uint32_t kOffF = kOffB + 2 * kBTile;               // [kRT][128] FP32 fields of the chunk
constexpr uint32_t kOffSw = kOffF + kRT * 128 * 4;           // [kRT][kSwWords] spin words
constexpr uint32_t kOffBar = kOffSw + kRT * kSwWords * 4;    // mbarriers
constexpr int kNumBars = 2 * kStages + 2 + 1 + 2;            // full, empty, diag, ready, done
constexpr uint32_t kOffMisc = kOffBar + kNumBars * 8;
constexpr size_t kHotSmem = kOffMisc + 64;
static_assert(2 * (kHotSmem + 1024) <= 228 * 1024, "two CTAs per SM");

struct HotArgs {
  const int8_t* digits;   // one int8 digit per coupling, tiled (oj_k_field_tc.cu)
  const int64_t* dtoff;
  const int32_t* uexp;
  const float* h;
  const int64_t* hoff;
  const int32_t* n;
  const int32_t* reads;
  const int64_t* soff;
  int8_t* spins;
  float* F;               // fields in and out, [reads][npad] per instance
  const int64_t* foff;
  const int64_t* eoff;    // replica offset of each instance (kstop index)
  const int32_t* items;   // [nitems][2]: instance, replica tile
  int nitems;
  const float* betas;
  int64_t nsweeps;
  ojd::Keys keys;
  uint32_t sweep0, inst0, rep0;
  int32_t* kstop;         // per replica: the sweep (from 0) the sweep kernel continues at
  int flip_floor;         // a tile leaves after a sweep with fewer flips per replica than this (-1: n/16)
  unsigned long long* flips;
  int* status;
  long long wait_limit;
};

__device__ __forceinline__ int sw_word(int c, int l) { return 32 * (c >> 3) + l; }
__device__ __forceinline__ int sw_shift(int c) { return 4 * (c & 7); }

__device__ __forceinline__ uint32_t canon(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15));
}

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
  // K-major, no swizzle: LBO 128 bytes (K-adjacent core matrices), SBO 1024 (8-row groups)
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46);
}

// s8 x s8 -> s32, K-major A and B, M = 128, N = kRT
__device__ __forceinline__ uint32_t idesc_i8() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kRT >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t da, uint64_t db) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, 1, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          dtmem),
      "l"(da), "l"(db), "r"(idesc_i8()));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   ojd::smem_u32(bar))
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

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const int32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}

// one TMEM row of a chunk: the kRT replicas' accumulators of this lane's site
static_assert(kRT == 16, "the TMEM row accessors move 16 columns");
__device__ __forceinline__ void tmem_ld_rt(uint32_t taddr, int32_t (&v)[kRT]) { tmem_ld16(taddr, v); }
__device__ __forceinline__ void tmem_st_rt(uint32_t taddr, const int32_t (&v)[kRT]) { tmem_st16(taddr, v); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__global__ void __launch_bounds__(kHotThreads, 2) hot_tc_kernel(HotArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int item = blockIdx.x;
  if (item >= a.nitems) return;  // the whole CTA
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = a.items[2 * item], rt = a.items[2 * item + 1];
  const int n = a.n[m], R = a.reads[m];
  const int nch = (n + 127) >> 7, npad = nch << 7;
  if (nch < 2 || nch > kHotMaxChunks) return;  // the host sends only 128 < n <= 2048
  const int r0 = rt * kRT;
  const uint32_t cols = nch * kRT <= 64 ? 64 : (nch * kRT <= 128 ? 128 : (nch * kRT <= 256 ? 256 : 512));
  unsigned char* ring = sm + kOffRing;
  unsigned char* diag = sm + kOffDiag;
  unsigned char* Bt = sm + kOffB;
  float* fsm = reinterpret_cast<float*>(sm + kOffF);
  uint32_t* swsm = reinterpret_cast<uint32_t*>(sm + kOffSw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kOffBar);
  uint64_t* full = bar;                    // [kStages]
  uint64_t* empty = bar + kStages;         // [kStages]
  uint64_t* dfull = bar + 2 * kStages;     // [2] diagonal tile of chunk-step q in buffer q % 2
  uint64_t* ready = dfull + 2;             // fields of the next chunk complete
  uint64_t* done = ready + 1;              // [2] every MMA of chunk-step q (B tile q % 2 free)
  uint32_t* misc = reinterpret_cast<uint32_t*>(sm + kOffMisc);
  uint32_t* tslot = misc;                  // TMEM base
  // abort flags by chunk-step parity: a wait of chunk-step q that runs out sets
  // ab[q & 1] before the step's closing barrier (the deciding warps) or
  // ab[(q + 1) & 1] after it (the MMA warp); every thread reads ab[q & 1]
  // after the barrier, so all leave at the same step
  volatile int* ab = reinterpret_cast<volatile int*>(misc + 1);
  unsigned int* sweep_flips = misc + 3;    // [2] flips of the sweep (by parity)
  uint64_t* fin = reinterpret_cast<uint64_t*>(misc + 6);  // 8-byte aligned: completion of every MMA
  int* jnext = reinterpret_cast<int*>(misc + 8);           // [2] next replica of the chunk step (by parity)
  const int8_t* dig = a.digits + a.dtoff[m];
  const float scale = ldexpf(1.0f, a.uexp[m]);   // 2^e: products stay exact
  const float inv_scale = ldexpf(1.0f, -a.uexp[m]);
  const float* hm = a.h + a.hoff[m];
  float* Fm = a.F + a.foff[m];
  int8_t* sp = a.spins + a.soff[m];
  const uint32_t tag = ((a.inst0 + (uint32_t)m) << 8) | ojd::TAG_BATCH;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(ojd::smem_u32(tslot)),
                 "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < kNumBars; ++q) ojd::mbar_init(bar + q, 1);
    ojd::mbar_init(fin, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    ab[0] = ab[1] = 0;
    sweep_flips[0] = sweep_flips[1] = 0u;
    jnext[0] = jnext[1] = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;

  // ---- initial state: accumulators from the FP32 fields (exact), spin bits
  if (warp < 4) {
    for (int c = 0; c < nch; ++c) {
      const int s = 128 * c + 32 * warp + lane;
      const float hf = hm[s];  // zero past n
      int32_t v[kRT];
#pragma unroll
      for (int j = 0; j < kRT; ++j) {
        const int r = r0 + j;
        const float f = r < R ? Fm[(size_t)r * npad + s] : hf;
        v[j] = __float2int_rn(__fmul_rn(__fsub_rn(f, hf), inv_scale));
      }
      tmem_st_rt(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(c * kRT), v);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }
  if (warp < kDecWarps) {
    for (int j = warp; j < kRT; j += kDecWarps) {
      const int r = r0 + j;
      for (int c8 = 0; c8 < nch; c8 += 8) {
        uint32_t w = 0u;
        if (r < R)
          for (int c = c8; c < nch && c < c8 + 8; ++c)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int i = 128 * c + 4 * lane + e;
              if (i < n && sp[(size_t)r * n + i] < 0) w |= 1u << (sw_shift(c) + e);
            }
        swsm[j * kSwWords + sw_word(c8, lane)] = w;
      }
    }
  }
  // copies / MMAs: tile g of the stream is chunk-step q = g / nch, t = g % nch:
  // J[(c + 1 + t) % nch][c] with c = q % nch (the next chunk's tile first)
  const long long gmax = a.nsweeps * (long long)nch * nch;
  long long g_issued = 0;   // tiles whose copies were issued (warp 8, lane 0)
  auto tile_src = [&](long long g) {
    const long long q = g / nch;
    const int t = (int)(g % nch), c = (int)(q % nch), cp = (c + 1 + t) % nch;
    return dig + ((size_t)cp * nch + c) * kTile;
  };
  auto issue_tile = [&](long long g) {  // its stage is free
    const int s = (int)(g % kStages);
    ojd::mbar_expect_tx(full + s, kTile);
    ojd::bulk_copy(ring + (size_t)s * kTile, tile_src(g), kTile, full + s);
  };
  auto issue_diag = [&](long long q) {  // buffer q % 2 is free
    const int c = (int)(q % nch), b = (int)(q & 1);
    ojd::mbar_expect_tx(dfull + b, kTile);
    ojd::bulk_copy(diag + (size_t)b * kTile, dig + ((size_t)c * nch + c) * kTile, kTile, dfull + b);
  };
  const bool mma_thread = warp == kDecWarps && lane == 0;
  if (mma_thread) {
    for (; g_issued < kAhead && g_issued < gmax; ++g_issued) issue_tile(g_issued);
    issue_diag(0);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  unsigned long long nflip = 0;
  long long q = 0;          // chunk-step
  long long g_cons = 0;     // tiles consumed by the MMA thread
  long long q_diag = 0;     // last chunk-step whose diagonal tile was copied
  int64_t kend = 0;         // sweeps done (0 while running)
  bool aborted = false;
  for (int64_t k = 0; k < a.nsweeps && !kend && !aborted; ++k) {
    const float beta2 = 2.0f * __ldg(a.betas + k);
    const uint32_t kk = a.sweep0 + (uint32_t)k;
    for (int c = 0; c < nch; ++c, ++q) {
      const int b = (int)(q & 1);
      if (warp < kDecWarps) {
        // fields of chunk c into shared memory (FP32, exact)
        if (warp < 4) {
          if (q > 0 && !ojd::mbar_wait(ready, (uint32_t)((q - 1) & 1), a.wait_limit)) ab[q & 1] = 1;
          tc_fence_after();
          int32_t v[kRT];
          tmem_ld_rt(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(c * kRT), v);
          const int s = 32 * warp + lane;
          const float hf = hm[128 * c + s];
#pragma unroll
          for (int j = 0; j < kRT; ++j) fsm[j * 128 + s] = __fadd_rn(hf, __fmul_rn(__int2float_rn(v[j]), scale));
        }
        if (!ojd::mbar_wait(dfull + b, (uint32_t)((q >> 1) & 1), a.wait_limit)) ab[q & 1] = 1;
        if (q >= 2 && !ojd::mbar_wait(done + b, (uint32_t)(((q - 2) >> 1) & 1), a.wait_limit)) ab[q & 1] = 1;
        named_sync(1, kDecWarps * 32);
        // the next chunk step's replica counter (its last users passed the
        // closing barrier of the previous step)
        if (tid == 0) jnext[(q + 1) & 1] = 0;
        // decide chunk c: each warp takes the next replica of the tile until
        // none is left (a warp whose replicas flip little takes more)
        const unsigned char* dg = diag + (size_t)b * kTile;
        unsigned char* Bq = Bt + (size_t)b * kBTile;
        const uint32_t inside = 0xFu >> (4 - min(max(n - 128 * c - 4 * lane, 0), 4));
        unsigned int wflips = 0;
        for (;;) {
          int j = 0;
          if (lane == 0) j = atomicAdd(jnext + (q & 1), 1);
          j = __shfl_sync(0xffffffffu, j, 0);
          if (j >= kRT) break;
          const int r = r0 + j;
          uint32_t* swj = swsm + j * kSwWords;
          const uint32_t myw0 = (swj[sw_word(c, lane)] >> sw_shift(c)) & 0xFu;
          uint32_t myw = myw0;
          if (r < R) {
            float4 fc = reinterpret_cast<const float4*>(fsm + j * 128)[lane];
            bool go;
            {
              // a chunk none of whose sites has beta*dE below the largest -ln u
              // keeps its state and draws nothing
              const float fv[4] = {fc.x, fc.y, fc.z, fc.w};
              uint32_t can = 0u;
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const float bf = __fmul_rn(beta2, fv[e]);
                if ((((myw >> e) & 1u) ? bf : -bf) < ojd::kNegLogMax) can |= 1u << e;
              }
              go = __any_sync(0xffffffffu, (can & inside) != 0u);
            }
            if (go) {
              const ojd::u4 x = ojd::philox((uint32_t)(32 * c + lane), kk, a.rep0 + (uint32_t)r, tag, a.keys);
              float L[4];
              L[0] = ojd::neglog(x.x);
              L[1] = ojd::neglog(x.y);
              L[2] = ojd::neglog(x.z);
              L[3] = ojd::neglog(x.w);
              uint32_t open = inside;
              for (;;) {
                const float fv[4] = {fc.x, fc.y, fc.z, fc.w};
                uint32_t mask = 0u;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                  const float bf = __fmul_rn(beta2, fv[e]);
                  if ((((myw >> e) & 1u) ? bf : -bf) < L[e]) mask |= 1u << e;
                }
                mask &= open;
                const uint32_t lanes = __ballot_sync(0xffffffffu, mask != 0u);
                if (!lanes) break;
                const int ls = __ffs(lanes) - 1;
                const uint32_t pk = __shfl_sync(0xffffffffu, mask | (myw << 4), ls);
                const int es = __ffs(pk & 0xFu) - 1;
                const float coef = ((pk >> (4 + es)) & 1u) ? 2.0f : -2.0f;
                const int il = 4 * ls + es;  // chunk-local site
                // row il of the diagonal tile = column il (J symmetric): this lane's four sites
                const uint32_t q4 = *reinterpret_cast<const uint32_t*>(dg + canon(il, 4 * lane));
                fc.x = __fmaf_rn(coef, __fmul_rn(__int2float_rn((int)(int8_t)(q4 & 0xFFu)), scale), fc.x);
                fc.y = __fmaf_rn(coef, __fmul_rn(__int2float_rn((int)(int8_t)((q4 >> 8) & 0xFFu)), scale), fc.y);
                fc.z = __fmaf_rn(coef, __fmul_rn(__int2float_rn((int)(int8_t)((q4 >> 16) & 0xFFu)), scale), fc.z);
                fc.w = __fmaf_rn(coef, __fmul_rn(__int2float_rn((int)(int8_t)(q4 >> 24)), scale), fc.w);
                if (lane == ls) myw ^= 1u << es;
                ++wflips;
                open = inside & (0xFu << min(max(il + 1 - 4 * lane, 0), 4));
              }
            }
          }
          // spin changes of this replica's chunk: +2 (from -1), -2 (from +1), 0
          const uint32_t ch = myw ^ myw0;
          uint32_t ds = 0u;
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if ((ch >> e) & 1u) ds |= (((myw0 >> e) & 1u) ? 0x02u : 0xFEu) << (8 * e);
          *reinterpret_cast<uint32_t*>(Bq + canon(j, 4 * lane)) = ds;
          if (ch) {
            uint32_t& wd = swj[sw_word(c, lane)];
            wd = (wd & ~(0xFu << sw_shift(c))) | (myw << sw_shift(c));
          }
        }
        if (lane == 0 && wflips) {
          atomicAdd(sweep_flips + (k & 1), wflips);
          nflip += wflips;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
      }
      named_sync(2, kHotThreads);
      tc_fence_after();
      if (ab[q & 1]) {
        aborted = true;
        break;
      }
      const bool last = c == nch - 1;
      bool stop = false;
      if (last) {
        const unsigned int sf = *reinterpret_cast<volatile unsigned int*>(sweep_flips + (k & 1));
        const long long floor_m = a.flip_floor >= 0 ? a.flip_floor : (n >> 4);
        stop = k + 1 >= a.nsweeps || (long long)sf < floor_m * min(kRT, R - r0);
      }
      if (mma_thread) {
        if (!stop) {
          issue_diag(q + 1);  // its buffer was last read by chunk-step q - 1
          q_diag = q + 1;
        }
        // the chunk's spin changes into every field: acc[c'] += J[c', c] ds
        for (int t = 0; t < nch; ++t) {
          const long long g = q * nch + t;
          const int s = (int)(g % kStages);
          // keep kAhead copies in flight: tile g + kAhead goes to the stage of
          // tile g - 2, whose MMAs were issued two tiles ago
          const long long gn = g + kAhead;
          if (gn == g_issued && gn < gmax && !(stop && gn >= (q + 1) * nch)) {
            const long long gold = gn - kStages;
            if (gold < 0 || ojd::mbar_wait(empty + (int)(gn % kStages), (uint32_t)((gold / kStages) & 1), a.wait_limit)) {
              issue_tile(gn);
              ++g_issued;
            } else {
              ab[(q + 1) & 1] = 1;
            }
          }
          if (!ojd::mbar_wait(full + s, (uint32_t)((g / kStages) & 1), a.wait_limit)) {
            ab[(q + 1) & 1] = 1;
            break;
          }
          ++g_cons;
          tc_fence_after();
          const int cp = (c + 1 + t) % nch;
          const uint32_t a0 = ojd::smem_u32(ring + (size_t)s * kTile), b0 = ojd::smem_u32(Bt + (size_t)b * kBTile);
#pragma unroll
          for (int kq = 0; kq < 4; ++kq)
            mma_i8(tbase + (uint32_t)(cp * kRT), desc_kmajor(a0 + kq * 256), desc_kmajor(b0 + kq * 256));
          mma_commit(empty + s);
          if (t == 0) mma_commit(ready);
        }
        mma_commit(done + b);
      }
      if (last) {
        if (tid == 0) sweep_flips[(k + 1) & 1] = 0u;
        if (stop) {
          kend = k + 1;
          ++q;
          break;
        }
      }
    }
  }
  // ---- drain (MMA thread): every MMA issued, every copy issued
  bool drained = true;
  if (mma_thread) {
    mma_commit(fin);
    drained &= ojd::mbar_wait(fin, 0u, kHotDrain);
    for (long long g = g_cons; g < g_issued; ++g)
      drained &= ojd::mbar_wait(full + (int)(g % kStages), (uint32_t)((g / kStages) & 1), kHotDrain);
    // the diagonal tile copied for the step after the last one the warps read
    if (aborted && q_diag >= q) drained &= ojd::mbar_wait(dfull + (int)(q_diag & 1), (uint32_t)((q_diag >> 1) & 1), kHotDrain);
    if (!drained) ab[0] = ab[1] = 1;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  aborted = aborted || ab[0] || ab[1];
  // ---- write-back: FP32 fields, spins and the sweep to continue from
  if (!aborted) {
    if (warp < 4) {
      for (int c = 0; c < nch; ++c) {
        int32_t v[kRT];
        tmem_ld_rt(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(c * kRT), v);
        const int s = 128 * c + 32 * warp + lane;
        const float hf = hm[s];
#pragma unroll
        for (int j = 0; j < kRT; ++j) {
          const int r = r0 + j;
          if (r < R) Fm[(size_t)r * npad + s] = __fadd_rn(hf, __fmul_rn(__int2float_rn(v[j]), scale));
        }
      }
    }
    if (warp < kDecWarps) {
      for (int j = warp; j < kRT; j += kDecWarps) {
        const int r = r0 + j;
        if (r >= R) continue;
        const uint32_t* swj = swsm + j * kSwWords;
        for (int c = 0; c < nch; ++c) {
          const uint32_t w = swj[sw_word(c, lane)] >> sw_shift(c);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int i = 128 * c + 4 * lane + e;
            if (i < n) sp[(size_t)r * n + i] = ((w >> e) & 1u) ? (int8_t)-1 : (int8_t)1;
          }
        }
        if (lane == 0) a.kstop[a.eoff[m] + r] = (int32_t)kend;
      }
    }
    if (lane == 0 && nflip && a.flips) atomicAdd(a.flips, nflip);
  } else if (tid == 0 && a.status) {
    atomicExch(a.status, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(cols));
}

// OJ_HOT_FLOOR fixes the hand-over floor (flips per replica and sweep) for
// every instance; by default it is n/16 of each instance.
int hot_floor() {
  if (const char* env = std::getenv("OJ_HOT_FLOOR")) {
    const int v = std::atoi(env);
    if (v >= 0) return v;
  }
  return -1;
}

}  // namespace

bool hot_tc_applies(const oj_batch* b) {
  if (const char* env = std::getenv("OJ_HOT"))
    if (env[0] == '0') return false;
  if (!b->exact_fields || b->ndig != 1 || b->count == 0) return false;
  for (int m = 0; m < b->count; ++m)
    if (b->n[m] > 128 && b->n[m] <= 128 * kHotMaxChunks) return true;
  return false;
}

void hot_tc_items(const oj_batch* b, const int32_t* reads, const std::vector<int>& order,
                  std::vector<int32_t>& items) {
  items.clear();
  for (int m : order) {
    const int n = b->n[m];
    if (n <= 128 || n > 128 * kHotMaxChunks) continue;
    for (int rt = 0; rt * kRT < reads[m]; ++rt) {
      items.push_back(m);
      items.push_back(rt);
    }
  }
}

cudaError_t launch_hot_tc(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff, int8_t* spins,
                          float* F, const int64_t* d_foff, const int64_t* d_eoff, const int32_t* d_items,
                          int nitems, const float* betas, int64_t nsweeps, RngBase rb, uint32_t inst0,
                          int32_t* kstop, int* d_status, long long wait_limit, cudaStream_t st) {
  if (nitems <= 0 || nsweeps <= 0) return cudaSuccess;
  HotArgs a;
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
  a.eoff = d_eoff;
  a.items = d_items;
  a.nitems = nitems;
  a.betas = betas;
  a.nsweeps = nsweeps;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.inst0 = inst0;
  a.rep0 = rb.rep0;
  a.kstop = kstop;
  a.flip_floor = hot_floor();
  a.flips = rb.flips;
  a.status = d_status;
  a.wait_limit = wait_limit >= 0 ? wait_limit : kHotDrain;
  cudaError_t e = cudaFuncSetAttribute(hot_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHotSmem);
  if (e != cudaSuccess) return e;
  hot_tc_kernel<<<nitems, kHotThreads, kHotSmem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace oj
