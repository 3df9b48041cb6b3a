// Device-side building blocks shared by every sweep kernel: the Philox4x32-10
// counter-based generator and the -ln(u) acceptance variate.
//
// Random stream definitions (key = (seed & 0xffffffff, seed >> 32)):
//   SA, colour-class and sequential dense kernels:
//     u(r, k, i)    = Philox((i, k, r >> 2, TAG_SA))[r & 3]
//   SQA colour-class kernel:
//     u(r, t, k, i) = Philox((i, k, r, ((t>>3)<<9) | ((t&1)<<8) | TAG_SQA))[(t>>1) & 3]
//   bit-packed SA kernel (32 replicas per word, group g):
//     W_l(g, k, i)  = Philox((i, k, g, ((l>>2)<<8) | TAG_SA_MSC))[l & 3],  l = 0..31
//   bit-packed SQA kernel (T slices per word, slice group q = 0, 1, 2):
//     W_l(r, q, k, i) = Philox((i, k, r, ((l>>2)<<16) | (q<<8) | TAG_SQA_MSC))[l & 3]
//   slice-split bit-packed SQA kernel (replica group g, half q = 0 even / 1 odd):
//     W_l(g, q, k, i) = Philox((i, k, g, ((l>>2)<<16) | (q<<8) | TAG_SQA_SPLIT))[l & 3]
//   Swendsen-Wang (bond e, cluster root c):
//     u(r, k, e)   = Philox((e >> 2, k, r, TAG_SW_BOND))[e & 3]
//     coin(r, k, c) = Philox((c >> 2, k, r, TAG_SW_FLIP))[c & 3] & 1
//   batched dense SA kernel (instance m, replica r of that instance):
//     u(m, r, k, i) = Philox((i >> 2, k, r, (m << 8) | TAG_BATCH))[i & 3]
// with r the replica, t the Trotter slice, k the sweep (one_mc_step repeats
// included) and i the site.  Results are therefore independent of how the
// replicas are spread over CTAs, clusters or GPUs.
#pragma once
#include <cstdint>

namespace ojd {

constexpr uint32_t TAG_SA = 0x5Au;
constexpr uint32_t TAG_SQA = 0xA5u;
constexpr uint32_t TAG_SA_MSC = 0x3Cu;
constexpr uint32_t TAG_SQA_MSC = 0xC3u;
constexpr uint32_t TAG_SQA_SPLIT = 0x69u;
constexpr uint32_t TAG_BATCH = 0x96u;
constexpr uint32_t TAG_SW_BOND = 0xB1u;
constexpr uint32_t TAG_SW_FLIP = 0xB2u;

struct u4 {
  uint32_t x, y, z, w;
};

// Adds the warp's accepted flips (the sum of v over its lanes) to *ctr with
// one atomic; every lane of the warp calls it, ctr may be null.
__device__ __forceinline__ void add_flips(unsigned long long* ctr, unsigned long long v) {
  if (!ctr) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, v);
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): per round
// (c0,c1,c2,c3) <- (hi(M1*c2)^c1^k0, lo(M1*c2), hi(M0*c0)^c3^k1, lo(M0*c0)),
// key bumped by the Weyl constants between rounds.
__device__ __forceinline__ u4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                     uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    // one 32x32->64 wide multiply gives both halves of each product
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    c0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    c1 = (uint32_t)p1;
    c2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c3 = (uint32_t)p0;
  }
  return u4{c0, c1, c2, c3};
}

// Philox key schedule (the ten round keys), precomputed on the host and
// passed as a kernel parameter so that every round reads its key from the
// constant bank instead of adding the Weyl increment.
struct Keys {
  uint32_t k0[10];
  uint32_t k1[10];
};

inline Keys make_keys(uint32_t k0, uint32_t k1) {
  Keys K;
  for (int r = 0; r < 10; ++r) {
    K.k0[r] = k0;
    K.k1[r] = k1;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return K;
}

__device__ __forceinline__ u4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const Keys& K) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    c0 = (uint32_t)(p1 >> 32) ^ c1 ^ K.k0[r];
    c1 = (uint32_t)p1;
    c2 = (uint32_t)(p0 >> 32) ^ c3 ^ K.k1[r];
    c3 = (uint32_t)p0;
  }
  return u4{c0, c1, c2, c3};
}

__device__ __forceinline__ uint32_t pick(const u4& v, int j) {
  return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

// -ln(u), u = (2*(x>>9)+1) * 2^-24 in (0,1).  u = m*2^e with m reduced to
// [sqrt(1/2), sqrt(2)]; ln m = t + t^2 Q(t), t = m - 1, Q a degree-6
// polynomial fitted by least squares at Chebyshev nodes to (ln(1+t) - t)/t^2
// (error below 6e-8, no division).  Each step is a single IEEE
// round-to-nearest operation (explicit _rn intrinsics, no contraction), so
// host code doing the same operations reproduces the bits.
//
// The range reduction uses integer steps that give exactly the values of the
// arithmetic definition (u = float(2k+1) * 2^-24; m = the mantissa in [1,2),
// halved with e + 1 when above 0x1.6a09e6p+0; float(e)) in fewer instructions:
//   * 0x3F800000 | k is the float 1 + k 2^-23 (one funnel shift of x), and
//     adding -(1 - 2^-24) gives (2k+1) 2^-24 exactly (the sum is representable);
//   * with b' = bits(u) - 0x3F3504F4 (0x3504F4: the first mantissa above
//     0x1.6a09e6p+0), b' >> 23 (arithmetic) is e and (b' & 0x7FFFFF) +
//     0x3F3504F4 the bits of m, the halving included;
//   * float(e) = float(0x4B400000 + e) - 1.5 * 2^23 (exact for |e| < 2^22).
// The largest value neglog takes (at u = 2^-24): a site whose beta*dE is at
// least this is rejected whatever its uniform.
constexpr float kNegLogMax = 0x1.0a2b24p+4f;

__device__ __forceinline__ float neglog(uint32_t x) {
  const float u = __fadd_rn(__uint_as_float(__funnelshift_r(x, 0x7Fu, 9)), -0x1.fffffep-1f);
  const uint32_t b = __float_as_uint(u) - 0x3F3504F4u;
  const float m = __uint_as_float((b & 0x007FFFFFu) + 0x3F3504F4u);
  const float ef = __fsub_rn(__int_as_float(0x4B400000 + ((int)b >> 23)), 0x1.8p23f);
  const float t = __fsub_rn(m, 1.0f);
  const float t2 = __fmul_rn(t, t);
  float q = -0x1.8e99cep-4f;
  q = __fmaf_rn(q, t, 0x1.4c9576p-3f);
  q = __fmaf_rn(q, t, -0x1.6420eep-3f);
  q = __fmaf_rn(q, t, 0x1.979cccp-3f);
  q = __fmaf_rn(q, t, -0x1.ff1d5ep-3f);
  q = __fmaf_rn(q, t, 0x1.5558fcp-2f);
  q = __fmaf_rn(q, t, -0x1.0000ecp-1f);
  const float lnm = __fmaf_rn(t2, q, t);
  const float lnu = __fmaf_rn(ef, 0x1.62e430p-1f, lnm);
  return -lnu;
}

// Shared-memory mbarriers and 1-D bulk copies (global -> this CTA's shared
// memory, no multicast).  Every wait is bounded by an iteration count.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t ph, long long limit) {
  for (long long it = 0; it < limit; ++it) {
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

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

// bytes a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

}  // namespace ojd
