// Batched dense SA over many instances of uneven size in one persistent launch.
//
// Work item = (instance m, group of up to W replicas of m, W = warps per CTA
// of the launch variant: 4, 8, 16 or 32; with 32 all reads of a 32-read
// instance share one SM and its L1 for the J rows).  Items
// are ordered by decreasing n (longest first) and handed out through an atomic
// counter, so the CTAs resident on the SMs keep pulling the next largest item
// until the queue is empty.  One warp runs one replica: its FP32 local fields
// live in the warp's slice of shared memory, laid out in 128-site chunks with
// lane l owning sites 4l..4l+3 of every chunk (one float4 per lane), and its
// spins are bits in shared memory: lane l's word g holds chunks 8g..8g+7, bit
// 4(c mod 8)+e set when site 128c+4l+e is -1.
//
// Update order and acceptance are the reference's sequential single-spin flip
// (include/openjij/updater/single_spin_flip.hpp:66-95): sites 0..n-1 in order,
// accept when dE <= 0 or beta*dE < -ln(u), dE = -2 s_i f_i, and on a flip every
// field moves by -2 s_i J_ij (f_j = fma(c, J_ij, f_j), c = -2 s_i: the product
// is exact, so this is the reference's dE += 4 s_i J_ij s_j rounded once).
// Within a chunk the warp evaluates the acceptance of all 128 sites at once from
// the current fields, jumps to the first accepted site, applies that flip and
// re-evaluates the sites after it: sites that do not flip leave the state
// unchanged, so this is the sequential sweep, with one step per flip instead
// of one per site; a flip applies its whole coupling row to the warp's fields
// at once.  The uniform of site i, sweep k, replica r of instance m is
// Philox((i >> 2, k, r, m << 8 | TAG_BATCH))[i & 3], r the replica's global
// index (rep0 + index within the instance).
//
// J is FP32, row-major with rows padded to a multiple of 128 columns (zeros),
// read through L1 one float4 per lane on every accepted flip, or from an FP16
// copy (8 bytes per lane) when FP16 holds every coupling exactly; small
// instances' rows are staged in shared memory (one bulk copy per work item),
// and batches of instances of at
// most 128 sites run sa_batch1_kernel (fields and spin bits in registers).
// The fields come from the tensor-core field kernel (oj_k_field_tc.cu),
// launched just before, through a global buffer of reads x padded n floats per
// instance; for couplings that are not exact in FP32 sums a run is cut into
// segments at multiples of the recompute interval and the fields are computed
// anew between segments (the sweep kernel then stores its final fields back,
// so that the field kernel can measure their drift).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "oj_device.cuh"
#include "oj_internal.h"

namespace oj {
namespace {

constexpr int kBatchWarps = 8;
constexpr int kBatchMaxN = 4096;
constexpr int kMaxChunks = kBatchMaxN / 128;

struct BatchArgs {
  const float* J;          // concatenated padded rows
  const float* h;          // concatenated padded fields
  const int64_t* joff;     // [count] offset of instance m's J (floats)
  const int64_t* hoff;     // [count] offset of instance m's h (floats)
  const int32_t* n;        // [count]
  const int32_t* reads;    // [count]
  const int64_t* soff;     // [count] offset of instance m's spins (bytes)
  const int32_t* items;    // [nitems][2] (instance, replica group), longest instance first
  int nitems;
  int count;               // instances in the batch
  int* counter;            // work-queue head, zero at launch
  int8_t* spins;
  const float* betas;
  int64_t nsweeps;
  ojd::Keys keys;
  uint32_t sweep0;
  uint32_t inst0;          // global index of instance 0
  uint32_t rep0;           // global index of each instance's replica 0
  int fstride;             // fields per warp in shared memory (multiple of 128)
  int swstride;            // spin words per warp: 32 per eight chunks
  const __half* J16;       // J as FP16 (same offsets), when every value is exact in FP16
  const float* F;          // initial fields, [reads][npad] per instance (tensor-core field kernel)
  const int64_t* foff;     // [count] offset of instance m's fields (floats)
  float* Fw;               // when set, each replica's final fields are stored here (same layout)
  double* E;               // FP64 energies from the final fields, or null (exact-field batches)
  const int64_t* eoff;     // [count] offset of instance m's energies
  unsigned long long* flips;  // accepted-flip counter, or null
  int* status;             // set when a bounded wait runs out
  long long wait_limit;    // iterations of the staging wait
  const int32_t* kstart;   // per replica (eoff[m] + r): the first sweep to run, or null (0)
  // one-chunk kernel: the fields set anew from the grid integers q (int32,
  // [n][128] at joff[m], element [i][j] = q_ji) before every global sweep that
  // is a multiple of recompute (0: never), as the tensor-core field kernel sets
  // them; with drift, the largest |f - f_exact| over those points and the end
  // of the run goes there (float bits) and the final fields are the exact ones
  const int32_t* Q;
  const int32_t* uexp;
  int recompute;
  unsigned int* drift;
};

constexpr long long kStageDrainLimit = 1ll << 26;

// Copies an instance's coupling rows (bytes, a multiple of 16, both addresses
// 16-byte aligned) into shared memory with one bulk copy that thread 0 issues
// and every thread of the CTA waits for.  Returns false in every thread when
// a thread's wait ran out (the copy is then waited for with the drain limit
// and *status is set): the CTA leaves the item.
__device__ __forceinline__ bool stage_rows(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                           uint32_t& phase, const BatchArgs& a) {
  if (threadIdx.x == 0) {
    ojd::mbar_expect_tx(bar, bytes);
    ojd::bulk_copy(dst, src, bytes, bar);
  }
  bool ok = ojd::mbar_wait(bar, phase, a.wait_limit);
  if (!ok) {
    ojd::mbar_wait(bar, phase, kStageDrainLimit);
    if (a.status) atomicExch(a.status, 1);
  }
  phase ^= 1u;
  return !__syncthreads_or(!ok);
}

// The CTA's staging barrier, once per launch.
__device__ __forceinline__ void stage_init(uint64_t* bar) {
  if (threadIdx.x == 0) {
    ojd::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// Spin bits of chunk c of lane l: four bits of word 32*(c/8) + l.
__device__ __forceinline__ int sw_word(int c, int l) { return 32 * (c >> 3) + l; }
__device__ __forceinline__ int sw_shift(int c) { return 4 * (c & 7); }

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
// four FP16 couplings widened to FP32 (exact)
__device__ __forceinline__ float4 ldg4h(const __half* p) {
  const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
  return make_float4(a.x, a.y, b.x, b.y);
}

// A flip row's four couplings of one lane, from global memory (through L1)
// or from the copy of the instance's couplings in shared memory (SJ).
template <bool SJ>
__device__ __forceinline__ float4 row4(const float* p) {
  if constexpr (SJ) return *reinterpret_cast<const float4*>(p);
  else return ldg4(p);
}
template <bool SJ>
__device__ __forceinline__ float4 row4h(const __half* p) {
  if constexpr (SJ) {
    const uint2 u = *reinterpret_cast<const uint2*>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
  } else {
    return ldg4h(p);
  }
}

// The couplings of an instance are staged in shared memory (SJ) when the
// batch's largest block of n rows x npad columns takes at most this many bytes.
constexpr size_t kBatchSmemJBytes = 96 * 1024;

// GROUP: chunks of a flip row whose loads are in flight together (more costs
// registers).  H: the flip rows come from the FP16 copy of J (half the L2
// bytes per flip).  SJ: every work item first copies its instance's couplings
// (FP32 or FP16 rows, as H says) into shared memory after the warps' fields and
// spin words, and the flips read their rows there (small instances: no L2
// round trip per flip).
template <int W, int MINB, int GROUP, bool H, bool SJ>
__global__ void __launch_bounds__(W * 32, MINB) sa_batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) float shb[];
  __shared__ int item_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* f = shb + (size_t)warp * a.fstride;  // this warp's fields, float4 per lane per chunk
  uint32_t* sw = reinterpret_cast<uint32_t*>(shb + (size_t)W * a.fstride) +
                 (size_t)warp * a.swstride;  // spin words [chunk / 8][lane]
  // the staged couplings (SJ): after every warp's fields and spin words
  char* jsh = reinterpret_cast<char*>(shb + (size_t)W * a.fstride + (size_t)W * a.swstride);
  __shared__ __align__(8) uint64_t stage_bar;
  uint32_t stage_phase = 0u;
  if (SJ) stage_init(&stage_bar);
  unsigned long long nflip = 0;  // lane 0 counts the warp's flips
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item_sh = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = item_sh;
    if (item >= a.nitems) break;
    const int m = a.items[2 * item];
    if ((unsigned)m >= (unsigned)a.count) continue;  // a corrupt table entry is skipped, never followed
    const int r = a.items[2 * item + 1] * W + warp;
    const int n = a.n[m];
    const bool active = r < a.reads[m];  // warps past the instance's reads wait for the next item
    const int nch = (n + 127) >> 7;
    const int npad = nch << 7;
    const float* J = a.J + a.joff[m];
    int8_t* gs = a.spins + a.soff[m] + (size_t)(active ? r : 0) * n;
    if (SJ) {
      // n rows of npad couplings by one bulk copy; every warp of the CTA waits
      // for it before any leaves for an inactive replica
      const void* src = H ? static_cast<const void*>(a.J16 + a.joff[m]) : static_cast<const void*>(J);
      if (!stage_rows(jsh, src, (uint32_t)(n * npad * (H ? 2 : 4)), &stage_bar, stage_phase, a)) continue;
    }
    const float* Jr = SJ ? reinterpret_cast<const float*>(jsh) : J;
    const __half* Jr16 = SJ ? reinterpret_cast<const __half*>(jsh) : (H ? a.J16 + a.joff[m] : nullptr);
    // spins -> bits
    if (active)
      for (int c8 = 0; c8 < nch; c8 += 8) {
        uint32_t w = 0u;
        for (int c = c8; c < nch && c < c8 + 8; ++c)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int i = 128 * c + 4 * lane + e;
            if (i < n && gs[i] < 0) w |= 1u << (sw_shift(c) + e);
          }
        sw[sw_word(c8, lane)] = w;
      }
    if (!active) continue;  // no block-wide barrier until the next item
    __syncwarp();
    // the fields f_j = h_j + sum_i J_ij s_i come from the tensor-core field kernel
    {
      const float* Fr = a.F + a.foff[m] + (size_t)r * npad;
      for (int c = 0; c < nch; ++c) reinterpret_cast<float4*>(f)[32 * c + lane] = ldg4(Fr + 128 * c + 4 * lane);
    }
    __syncwarp();
    const uint32_t tag = ((a.inst0 + (uint32_t)m) << 8) | ojd::TAG_BATCH;
    const uint32_t rg = a.rep0 + (uint32_t)r;
    // this lane's sites of the last chunk that exist (site index below n), as
    // a 4-bit mask; every site of the other chunks exists
    const uint32_t inside_last = 0xFu >> (4 - min(max(n - 128 * (nch - 1) - 4 * lane, 0), 4));
    const int64_t kfirst = a.kstart ? (int64_t)a.kstart[a.eoff[m] + r] : 0;
    for (int64_t k = kfirst; k < a.nsweeps; ++k) {
      const float beta2 = 2.0f * __ldg(a.betas + k);
      const uint32_t kk = a.sweep0 + (uint32_t)k;
      for (int c = 0; c < nch; ++c) {
        const uint32_t inside = c == nch - 1 ? inside_last : 0xFu;
        {
          // a chunk none of whose sites has beta*dE below the largest -ln u
          // keeps its state: its uniforms are not drawn (the stream is
          // counter-based, so nothing after it moves)
          const float4 f4 = reinterpret_cast<const float4*>(f)[32 * c + lane];
          const float fv[4] = {f4.x, f4.y, f4.z, f4.w};
          const uint32_t myw = sw[sw_word(c, lane)] >> sw_shift(c);
          uint32_t can = 0u;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float bf = __fmul_rn(beta2, fv[e]);
            if ((((myw >> e) & 1u) ? bf : -bf) < ojd::kNegLogMax) can |= 1u << e;
          }
          if (!__any_sync(0xffffffffu, (can & inside) != 0u)) continue;
        }
        const ojd::u4 x = ojd::philox((uint32_t)(32 * c + lane), kk, rg, tag, a.keys);
        float L[4];
        L[0] = ojd::neglog(x.x);
        L[1] = ojd::neglog(x.y);
        L[2] = ojd::neglog(x.z);
        L[3] = ojd::neglog(x.w);
        // this lane's sites that exist and are not yet decided in this chunk
        // (chunk-local index at or past the last flip's + 1)
        uint32_t open = inside;
        for (;;) {
          const float4 f4 = reinterpret_cast<const float4*>(f)[32 * c + lane];
          const float fv[4] = {f4.x, f4.y, f4.z, f4.w};
          const uint32_t myw = sw[sw_word(c, lane)] >> sw_shift(c);
          uint32_t mask = 0u;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const bool neg = (myw >> e) & 1u;
            // beta*dE with dE = -+2 f: (2 beta) f is the same number (scaling by
            // 2 is exact).  dE <= 0 accepts without a draw; as -ln u > 0 for
            // every u and beta is finite and >= 0, beta*dE < -ln u covers that
            // case too
            const float bf = __fmul_rn(beta2, fv[e]);
            if ((neg ? bf : -bf) < L[e]) mask |= 1u << e;
          }
          mask &= open;
          const uint32_t lanes = __ballot_sync(0xffffffffu, mask != 0u);
          if (!lanes) break;
          const int ls = __ffs(lanes) - 1;
          const uint32_t ms = __shfl_sync(0xffffffffu, mask, ls);
          const int es = __ffs(ms) - 1;
          const uint32_t ws = sw[sw_word(c, ls)];
          const bool neg = (ws >> (sw_shift(c) + es)) & 1u;
          const float coef = neg ? 2.0f : -2.0f;
          const int i = 128 * c + 4 * ls + es;
          const float* Ji = Jr + (size_t)i * npad + 4 * lane;
          const __half* Ji16 = Jr16 + (size_t)i * npad + 4 * lane;
          // the row in groups of GROUP chunks whose loads are in flight together
#pragma unroll
          for (int c0 = 0; c0 < kMaxChunks; c0 += GROUP) {
            if (c0 >= nch) break;
            float4 v[GROUP];
#pragma unroll
            for (int q = 0; q < GROUP; ++q)
              if (c0 + q < nch) v[q] = H ? row4h<SJ>(Ji16 + 128 * (c0 + q)) : row4<SJ>(Ji + 128 * (c0 + q));
#pragma unroll
            for (int q = 0; q < GROUP; ++q)
              if (c0 + q < nch) {
                float4 g = reinterpret_cast<const float4*>(f)[32 * (c0 + q) + lane];
                g.x = __fmaf_rn(coef, v[q].x, g.x);
                g.y = __fmaf_rn(coef, v[q].y, g.y);
                g.z = __fmaf_rn(coef, v[q].z, g.z);
                g.w = __fmaf_rn(coef, v[q].w, g.w);
                reinterpret_cast<float4*>(f)[32 * (c0 + q) + lane] = g;
              }
          }
          __syncwarp();
          if (lane == ls) sw[sw_word(c, ls)] = ws ^ (1u << (sw_shift(c) + es));
          if (lane == 0) ++nflip;
          const int pos = 4 * ls + es + 1;  // chunk-local index of the first site not yet decided
          open = inside & (0xFu << min(max(pos - 4 * lane, 0), 4));
          __syncwarp();
        }
      }
    }
    if (a.Fw) {
      float* Fr = a.Fw + a.foff[m] + (size_t)r * npad;
      for (int c = 0; c < nch; ++c)
        *reinterpret_cast<float4*>(Fr + 128 * c + 4 * lane) = reinterpret_cast<const float4*>(f)[32 * c + lane];
    }
    if (a.E) {
      // exact fields: E = 1/2 sum_i s_i (f_i + h_i), every term and partial sum
      // exact in FP64, so the result is the FP64 energy in any order
      const float* h = a.h + a.hoff[m];
      double e = 0.0;
      for (int c = 0; c < nch; ++c) {
        const float4 f4 = reinterpret_cast<const float4*>(f)[32 * c + lane];
        const float4 h4 = ldg4(h + 128 * c + 4 * lane);
        const float fv[4] = {f4.x, f4.y, f4.z, f4.w}, hv[4] = {h4.x, h4.y, h4.z, h4.w};
        const uint32_t w = sw[sw_word(c, lane)] >> sw_shift(c);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double t = (double)fv[q] + (double)hv[q];
          if (128 * c + 4 * lane + q < n) e += ((w >> q) & 1u) ? -t : t;
        }
      }
      for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
      if (lane == 0) a.E[a.eoff[m] + r] = 0.5 * e;
    }
    for (int c = 0; c < nch; ++c) {
      const uint32_t w = sw[sw_word(c, lane)] >> sw_shift(c);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int i = 128 * c + 4 * lane + e;
        if (i < n) gs[i] = ((w >> e) & 1u) ? (int8_t)-1 : (int8_t)1;
      }
    }
    __syncwarp();
  }
  ojd::add_flips(a.flips, nflip);
}

// Batches whose instances have at most 128 sites (one chunk): the sweep of
// sa_batch_kernel with each lane's four fields and spin bits in registers for
// the whole run and the instance's coupling rows (FP32, or FP16 when H) staged
// in shared memory by every work item, so that a flip is a ballot, a shuffle,
// one shared-memory row load and four FMAs.  Same random stream, acceptance
// test, skipping of chunks that cannot flip and FMA order, so the same bits.
// The exact fields of this lane's four sites (4 lane .. 4 lane + 3) of a
// one-chunk instance: f_j = fp32(fp64(h_j) + 2^e sum_i q_ji s_i), the sum in
// int64 (exact), the same operations as the tensor-core field kernel's
// epilogue, so the same values.  wd: this lane's spin bits (set: -1).
__device__ __forceinline__ float4 exact_fields1(const int32_t* __restrict__ Qm, int n, uint32_t wd, double scale,
                                                const float4 h4) {
  const int lane = threadIdx.x & 31;
  long long acc[4] = {0, 0, 0, 0};
  // two source lanes (8 rows) a pass, their row loads issued together; |q| <=
  // 2^26, so the 8-row partial sums fit int32
  for (int L0 = 0; 4 * L0 < n; L0 += 2) {
    int4 q[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int i = 4 * L0 + t;
      q[t] = i < n ? __ldg(reinterpret_cast<const int4*>(Qm + (size_t)i * 128) + lane) : make_int4(0, 0, 0, 0);
    }
    int p[4] = {0, 0, 0, 0};
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const uint32_t w = __shfl_sync(0xffffffffu, wd, (L0 + l) & 31);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int4 v = q[4 * l + e];  // zero past n
        const int sg = ((w >> e) & 1u) ? -1 : 1;
        p[0] += sg * v.x;
        p[1] += sg * v.y;
        p[2] += sg * v.z;
        p[3] += sg * v.w;
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[e] += p[e];
  }
  const float hv[4] = {h4.x, h4.y, h4.z, h4.w};
  float f[4];
#pragma unroll
  for (int e = 0; e < 4; ++e)
    f[e] = __double2float_rn(__dadd_rn((double)hv[e], __dmul_rn(__ll2double_rn(acc[e]), scale)));
  return make_float4(f[0], f[1], f[2], f[3]);
}

// Largest |f - g| over this lane's sites below n.
__device__ __forceinline__ float field_gap(const float4 f, const float4 g, int n) {
  const int lane = threadIdx.x & 31;
  const float a[4] = {f.x, f.y, f.z, f.w}, b[4] = {g.x, g.y, g.z, g.w};
  float d = 0.0f;
#pragma unroll
  for (int e = 0; e < 4; ++e)
    if (4 * lane + e < n) d = fmaxf(d, fabsf(a[e] - b[e]));
  return d;
}

template <int W, bool H>
__global__ void __launch_bounds__(W * 32) sa_batch1_kernel(BatchArgs a) {
  extern __shared__ __align__(16) float shb[];  // [n][128] couplings of the item's instance
  __shared__ int item_sh;
  __shared__ __align__(8) uint64_t stage_bar;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t stage_phase = 0u;
  stage_init(&stage_bar);
  unsigned long long nflip = 0;  // lane 0 counts the warp's flips
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item_sh = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = item_sh;
    if (item >= a.nitems) break;
    const int m = a.items[2 * item];
    if ((unsigned)m >= (unsigned)a.count) continue;  // a corrupt table entry is skipped, never followed
    const int n = a.n[m];
    if (n > 128) continue;  // the host launches this kernel only for n <= 128
    const int r = a.items[2 * item + 1] * W + warp;
    {
      // n rows of 128 couplings by one bulk copy, waited for by every warp of
      // the CTA before any leaves for an inactive replica
      const void* src = H ? static_cast<const void*>(a.J16 + a.joff[m]) : static_cast<const void*>(a.J + a.joff[m]);
      if (!stage_rows(shb, src, (uint32_t)(n * 128 * (H ? 2 : 4)), &stage_bar, stage_phase, a)) continue;
    }
    if (r >= a.reads[m]) continue;  // warps past the instance's reads wait for the next item
    int8_t* gs = a.spins + a.soff[m] + (size_t)r * n;
    uint32_t wd = 0u;  // bit e: site 4*lane + e is -1
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = 4 * lane + e;
      if (i < n && gs[i] < 0) wd |= 1u << e;
    }
    float4 fc = ldg4(a.F + a.foff[m] + (size_t)r * 128 + 4 * lane);
    const uint32_t inside = 0xFu >> (4 - min(max(n - 4 * lane, 0), 4));
    const float* Js = shb + 4 * lane;
    const __half* Js16 = reinterpret_cast<const __half*>(shb) + 4 * lane;
    const uint32_t tag = ((a.inst0 + (uint32_t)m) << 8) | ojd::TAG_BATCH;
    const uint32_t rg = a.rep0 + (uint32_t)r;
    const int32_t* Qm = a.Q ? a.Q + a.joff[m] : nullptr;
    const double qscale = Qm ? ldexp(1.0, a.uexp[m]) : 0.0;
    const float4 h4q = Qm ? ldg4(a.h + a.hoff[m] + 4 * lane) : make_float4(0.f, 0.f, 0.f, 0.f);
    float dmax = 0.0f;
    for (int64_t k = 0; k < a.nsweeps; ++k) {
      const float beta2 = 2.0f * __ldg(a.betas + k);
      if (Qm && k > 0 && (a.sweep0 + (uint32_t)k) % (uint32_t)a.recompute == 0u) {
        const float4 fx = exact_fields1(Qm, n, wd, qscale, h4q);
        if (a.drift) dmax = fmaxf(dmax, field_gap(fc, fx, n));
        fc = fx;
      }
      {
        // no site below the largest -ln u: the chunk keeps its state
        const float fv[4] = {fc.x, fc.y, fc.z, fc.w};
        uint32_t can = 0u;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float bf = __fmul_rn(beta2, fv[e]);
          if ((((wd >> e) & 1u) ? bf : -bf) < ojd::kNegLogMax) can |= 1u << e;
        }
        if (!__any_sync(0xffffffffu, (can & inside) != 0u)) continue;
      }
      const ojd::u4 x = ojd::philox((uint32_t)lane, a.sweep0 + (uint32_t)k, rg, tag, a.keys);
      float L[4];
      L[0] = ojd::neglog(x.x);
      L[1] = ojd::neglog(x.y);
      L[2] = ojd::neglog(x.z);
      L[3] = ojd::neglog(x.w);
      uint32_t open = inside;  // sites that exist and are not yet decided in this sweep
      for (;;) {
        const float fv[4] = {fc.x, fc.y, fc.z, fc.w};
        uint32_t mask = 0u;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float bf = __fmul_rn(beta2, fv[e]);
          if ((((wd >> e) & 1u) ? bf : -bf) < L[e]) mask |= 1u << e;
        }
        mask &= open;
        const uint32_t lanes = __ballot_sync(0xffffffffu, mask != 0u);
        if (!lanes) break;
        const int ls = __ffs(lanes) - 1;
        // the first accepting lane's mask and spin bits
        const uint32_t pk = __shfl_sync(0xffffffffu, mask | (wd << 4), ls);
        const int es = __ffs(pk & 0xFu) - 1;
        const float coef = ((pk >> (4 + es)) & 1u) ? 2.0f : -2.0f;
        const int i = 4 * ls + es;
        const float4 v = H ? row4h<true>(Js16 + 128 * i) : row4<true>(Js + 128 * i);
        fc.x = __fmaf_rn(coef, v.x, fc.x);
        fc.y = __fmaf_rn(coef, v.y, fc.y);
        fc.z = __fmaf_rn(coef, v.z, fc.z);
        fc.w = __fmaf_rn(coef, v.w, fc.w);
        if (lane == ls) wd ^= 1u << es;
        if (lane == 0) ++nflip;
        open = inside & (0xFu << min(max(i + 1 - 4 * lane, 0), 4));
      }
    }
    if (Qm && a.drift) {
      // the drift check after the last sweep; the exact fields are kept
      const float4 fx = exact_fields1(Qm, n, wd, qscale, h4q);
      dmax = fmaxf(dmax, field_gap(fc, fx, n));
      fc = fx;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
      if (lane == 0 && dmax > 0.0f) atomicMax(a.drift, __float_as_uint(dmax));
    }
    if (a.Fw) *reinterpret_cast<float4*>(a.Fw + a.foff[m] + (size_t)r * 128 + 4 * lane) = fc;
    if (a.E) {
      // exact fields: E = 1/2 sum_i s_i (f_i + h_i), as in sa_batch_kernel
      const float4 h4 = ldg4(a.h + a.hoff[m] + 4 * lane);
      const float fv[4] = {fc.x, fc.y, fc.z, fc.w}, hv[4] = {h4.x, h4.y, h4.z, h4.w};
      double e = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double t = (double)fv[q] + (double)hv[q];
        if (4 * lane + q < n) e += ((wd >> q) & 1u) ? -t : t;
      }
      for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
      if (lane == 0) a.E[a.eoff[m] + r] = 0.5 * e;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = 4 * lane + e;
      if (i < n) gs[i] = ((wd >> e) & 1u) ? (int8_t)-1 : (int8_t)1;
    }
  }
  ojd::add_flips(a.flips, nflip);
}

// FP64 energy of every replica: E = sum_{i<j} J_ij s_i s_j + sum_i h_i s_i
// (dense.hpp:176-192) from the FP64 augmented matrix.  One CTA per (instance,
// 32 replicas), instances largest first: the spins are staged as one word per
// site (bit = replica), a lane accumulates its replica, warps take rows
// round-robin, read each row segment once (coalesced, through a per-warp
// shared buffer, next segment prefetched) and apply it to all 32 replicas;
// partial sums are combined in a fixed order, so the result does not depend on
// timing.
__global__ void __launch_bounds__(256) batch_energy_kernel(const double* __restrict__ J64,
                                                           const int64_t* __restrict__ j64off,
                                                           const int32_t* __restrict__ n_arr,
                                                           const int32_t* __restrict__ reads,
                                                           const int64_t* __restrict__ soff,
                                                           const int64_t* __restrict__ eoff,
                                                           const int32_t* __restrict__ order,
                                                           const int8_t* __restrict__ spins, double* __restrict__ out,
                                                           int64_t nrep) {
  __shared__ uint32_t wsh[kBatchMaxN + 32];
  __shared__ double rowbuf[8][32];
  __shared__ double part[8][32];
  const int m = order[blockIdx.x];
  const int r0 = 32 * blockIdx.y;
  const int R = reads[m];
  if (r0 >= R) return;
  const int n = n_arr[m];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int8_t* s = spins + soff[m];
  for (int j = threadIdx.x; j < n + 32; j += blockDim.x) {
    uint32_t w = 0u;
    if (j < n)
      for (int q = 0; q < 32 && r0 + q < R; ++q)
        if (s[(size_t)(r0 + q) * n + j] < 0) w |= 1u << q;
    wsh[j] = w;
  }
  __syncthreads();
  const double* A = J64 + j64off[m];  // augmented (n+1)^2, row-major
  const int split = blockIdx.z, nsplit = gridDim.z;  // rows i with (i / 8) % nsplit == split
  double acc = 0.0;
  for (int i = 8 * split + warp; i < n; i += 8 * nsplit) {
    const double* Ai = A + (size_t)i * (n + 1);
    const uint32_t wi = wsh[i];
    double p[4] = {0.0, 0.0, 0.0, 0.0};
    int j0 = i + 1;
    double a = j0 + lane < n ? __ldg(Ai + j0 + lane) : 0.0;
    for (; j0 < n; j0 += 32) {
      const double an = j0 + 32 + lane < n ? __ldg(Ai + j0 + 32 + lane) : 0.0;  // next segment
      __syncwarp();
      rowbuf[warp][lane] = a;  // zero past the end of the row
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const double v = rowbuf[warp][q];
        const uint32_t flip = ((wi ^ wsh[j0 + q]) >> lane) & 1u;  // s_i != s_j in this replica
        p[q & 3] += flip ? -v : v;
      }
      a = an;
    }
    const double hv = __ldg(Ai + n);
    acc += ((p[0] + p[1]) + (p[2] + p[3])) + (((wi >> lane) & 1u) ? -hv : hv);
  }
  part[warp][lane] = acc;
  __syncthreads();
  if (warp == 0 && r0 + lane < R) {
    double e = 0.0;
    for (int w = 0; w < 8; ++w) e += part[w][lane];
    out[(size_t)split * nrep + eoff[m] + r0 + lane] = e;  // this row split's part
  }
}

// Sums the row splits' parts of every replica's energy, split 0 first.
__global__ void batch_energy_sum_kernel(const double* __restrict__ parts, int nsplit, int64_t nrep,
                                        double* __restrict__ out) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrep) return;
  double e = 0.0;
  for (int k = 0; k < nsplit; ++k) e += parts[(size_t)k * nrep + r];
  out[r] = e;
}

}  // namespace

int batch_max_sites() { return kBatchMaxN; }
int batch_warps() { return kBatchWarps; }

// Launch variants: warps per CTA x minimum CTAs per SM (register budget).
// 45 = 4 warps, 102 registers, 8 chunks at a time (more CTAs per SM when the
//      fields' shared memory limits residency);
// 82 = 8 warps, 128 registers, a flip row's loads 16 chunks at a time;
// 83 = 8 warps, 80 registers; 84 = 8 warps, 64; 162 = 16 warps, 64; 321 = 32 warps, 64
// (4 chunks at a time).
int batch_min_warps() { return 4; }

int batch_variant_warps(int variant) {
  switch (variant) {
    case 45: return 4;
    case 162: return 16;
    case 321: return 32;
    default: return 8;
  }
}

bool batch_variant_valid(int variant) {
  return variant == 45 || variant == 82 || variant == 83 || variant == 84 || variant == 162 || variant == 321;
}

// largest n whose fields fit the variant: W warps x (FP32 fields + spin
// words) within the 227 KB of shared memory per CTA
int batch_variant_max_n(int variant) {
  switch (variant) {
    case 321: return 1664;
    case 162: return 3456;
    default: return kBatchMaxN;
  }
}

int batch_default_variant() {
  if (const char* env = std::getenv("OJ_BATCH_VARIANT")) {
    const int v = std::atoi(env);
    if (batch_variant_valid(v)) return v;
  }
  return 83;
}

template <int W, int MINB, int GROUP>
cudaError_t launch_variant(const BatchArgs& a, int nitems, int sm_count, cudaStream_t st, bool h, size_t jbytes) {
  const bool sj = jbytes > 0;
  auto kern = h ? (sj ? sa_batch_kernel<W, MINB, GROUP, true, true> : sa_batch_kernel<W, MINB, GROUP, true, false>)
                : (sj ? sa_batch_kernel<W, MINB, GROUP, false, true> : sa_batch_kernel<W, MINB, GROUP, false, false>);
  // FP32 fields + spin words per warp, then the staged couplings
  const size_t smem = (size_t)W * ((size_t)a.fstride * 4 + (size_t)a.swstride * 4) + jbytes;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::max(1, std::min(nitems, per_sm * sm_count));
  kern<<<grid, W * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <int W>
cudaError_t launch_one_chunk(const BatchArgs& a, int max_n, int nitems, int sm_count, cudaStream_t st, bool h) {
  auto kern = h ? sa_batch1_kernel<W, true> : sa_batch1_kernel<W, false>;
  const size_t smem = (size_t)max_n * 128 * (h ? 2 : 4);  // the staged couplings
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::max(1, std::min(nitems, per_sm * sm_count));
  kern<<<grid, W * 32, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_batch_sweeps(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff,
                                const int32_t* d_items, int nitems, int* d_counter, int8_t* spins,
                                const float* betas, int64_t nsweeps, RngBase rb, uint32_t inst0, int sm_count,
                                cudaStream_t st, int* launches, int variant, float* d_fields,
                                const int64_t* d_foff, double* d_energies, const int64_t* d_eoff,
                                bool write_fields, int* d_status, long long wait_limit,
                                const int32_t* kstart, int recompute, unsigned int* d_drift) {
  if (variant == 0) variant = batch_default_variant();
  if (!batch_variant_valid(variant) || b->max_n > batch_variant_max_n(variant)) return cudaErrorInvalidValue;
  if (b->count == 0 || nitems <= 0 || nsweeps <= 0) return cudaSuccess;
  const int fstride = std::max(128, (b->max_n + 127) / 128 * 128);
  BatchArgs a;
  a.J = b->d_J.as<float>();
  a.h = b->d_h.as<float>();
  a.joff = b->d_joff.as<int64_t>();
  a.hoff = b->d_hoff.as<int64_t>();
  a.n = b->d_n.as<int32_t>();
  a.reads = d_reads;
  a.soff = d_soff;
  a.items = d_items;
  a.nitems = nitems;
  a.count = b->count;
  a.counter = d_counter;
  a.spins = spins;
  a.betas = betas;
  a.nsweeps = nsweeps;
  a.keys = ojd::make_keys(rb.k0, rb.k1);
  a.sweep0 = rb.sweep0;
  a.inst0 = inst0;
  a.rep0 = rb.rep0;
  a.fstride = fstride;
  a.swstride = 32 * ((fstride / 128 + 7) / 8);
  a.J16 = b->j16 ? b->d_J16.as<__half>() : nullptr;
  a.F = d_fields;
  a.foff = d_foff;
  a.Fw = write_fields ? d_fields : nullptr;
  a.E = b->exact_fields ? d_energies : nullptr;
  a.eoff = d_eoff;
  a.flips = rb.flips;
  a.status = d_status;
  a.wait_limit = wait_limit >= 0 ? wait_limit : kStageDrainLimit;
  a.kstart = kstart;
  const bool own = recompute > 0 && b->max_n <= 128 && b->d_q32.ptr && !b->exact_fields;
  a.Q = own ? b->d_q32.as<int32_t>() : nullptr;
  a.uexp = own ? b->d_uexp.as<int32_t>() : nullptr;
  a.recompute = own ? recompute : 0;
  a.drift = own ? d_drift : nullptr;
  cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  if (b->max_n <= 128) {
    // one chunk per instance: fields and spin bits in registers (same warps
    // per CTA as the variant, so the same work items)
    switch (batch_variant_warps(variant)) {
      case 4: e = launch_one_chunk<4>(a, b->max_n, nitems, sm_count, st, b->j16); break;
      case 16: e = launch_one_chunk<16>(a, b->max_n, nitems, sm_count, st, b->j16); break;
      case 32: e = launch_one_chunk<32>(a, b->max_n, nitems, sm_count, st, b->j16); break;
      default: e = launch_one_chunk<8>(a, b->max_n, nitems, sm_count, st, b->j16); break;
    }
    if (e == cudaSuccess && launches) ++*launches;
    return e;
  }
  // the largest instance's couplings in shared memory when they are small
  size_t jbytes = (size_t)b->max_n * (size_t)fstride * (b->j16 ? 2 : 4);
  if (jbytes > kBatchSmemJBytes) jbytes = 0;
  switch (variant) {
    case 45: e = launch_variant<4, 5, 8>(a, nitems, sm_count, st, b->j16, jbytes); break;
    case 82: e = launch_variant<8, 2, 16>(a, nitems, sm_count, st, b->j16, jbytes); break;
    case 83: e = launch_variant<8, 3, 4>(a, nitems, sm_count, st, b->j16, jbytes); break;
    case 84: e = launch_variant<8, 4, 4>(a, nitems, sm_count, st, b->j16, jbytes); break;
    case 162: e = launch_variant<16, 2, 4>(a, nitems, sm_count, st, b->j16, jbytes); break;
    default: e = launch_variant<32, 1, 4>(a, nitems, sm_count, st, b->j16, jbytes); break;
  }
  if (e == cudaSuccess && launches) ++*launches;
  return e;
}

cudaError_t launch_sa_batch(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff,
                            const int32_t* d_items, int nitems, int* d_counter, int8_t* spins, const float* betas,
                            int64_t nsweeps, RngBase rb, uint32_t inst0, int sm_count, cudaStream_t st,
                            int* launches, int variant, float* d_fields, const int64_t* d_foff,
                            const FieldCall& fc, double* d_energies, const int64_t* d_eoff) {
  if (b->count == 0 || nitems <= 0) return cudaSuccess;
  cudaError_t e = launch_field_tc(b, d_reads, d_soff, spins, d_fields, d_foff, fc.items, fc.nitems, fc.NT, false,
                                  fc.drift, fc.status, fc.wait_limit, st);
  if (e != cudaSuccess) return e;
  if (launches) ++*launches;
  return launch_batch_sweeps(b, d_reads, d_soff, d_items, nitems, d_counter, spins, betas, nsweeps, rb, inst0,
                             sm_count, st, launches, variant, d_fields, d_foff, d_energies, d_eoff, false, fc.status,
                             fc.wait_limit);
}

int batch_energy_splits(const oj_batch* b, int max_reads, int sm_count) {
  // rows split over CTAs until the grid covers the SMs several times (8 rows per
  // warp pass, so a split keeps at least 64 rows)
  const int64_t base = (int64_t)b->count * ((max_reads + 31) / 32);
  int k = 1;
  while (k < 16 && base * k < 6LL * sm_count && 64 * 2 * k <= b->max_n) k *= 2;
  return k;
}

cudaError_t launch_batch_energy(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff,
                                const int64_t* d_eoff, const int32_t* d_order, int max_reads, const int8_t* spins,
                                double* out, cudaStream_t st, int nsplit, double* parts, int64_t nrep) {
  if (b->count == 0 || max_reads == 0) return cudaSuccess;
  if (nsplit < 1 || (nsplit > 1 && !parts)) return cudaErrorInvalidValue;
  dim3 grid(b->count, (max_reads + 31) / 32, nsplit);
  batch_energy_kernel<<<grid, 256, 0, st>>>(b->d_J64.as<double>(), b->d_j64off.as<int64_t>(), b->d_n.as<int32_t>(),
                                            d_reads, d_soff, d_eoff, d_order, spins, nsplit > 1 ? parts : out, nrep);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || nsplit == 1) return e;
  batch_energy_sum_kernel<<<(unsigned)((nrep + 255) / 256), 256, 0, st>>>(parts, nsplit, nrep, out);
  return cudaGetLastError();
}

}  // namespace oj
