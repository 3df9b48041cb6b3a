// ORACLE — test infrastructure only.  Nothing in the product (openjij_b200/)
// links, imports or calls this file; tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py use it as the checker.
//
// Two independent CPU programs live here:
//
//  (1) A plain C++17 restatement of OpenJij's CPU single-spin-flip path, FP64,
//      with the reference's own random stream (Xorshift + libstdc++
//      distributions).  It follows, line by line:
//        include/openjij/utility/random.hpp:39-87          Xorshift
//        include/openjij/graph/graph.hpp:54-65              gen_spin
//        include/openjij/system/classical_ising.hpp:87-90   reset_dE
//        include/openjij/updater/single_spin_flip.hpp:66-95 classical sweep
//        include/openjij/system/transverse_ising.hpp:165-186 reset_dE (SQA)
//        include/openjij/updater/single_spin_flip.hpp:127-258 SQA sweep
//        include/openjij/utility/schedule_list.hpp:165-207  schedules
//        include/openjij/result/get_solution.hpp:39-84      get_solution
//        include/openjij/graph/dense.hpp:176-192            energy
//      Pinned by the reference's own known-answer tests
//      (tests/test_cxx.py:224-275,419-469; tests/cxxtest/sampler/quadraitc.hpp).
//      Only difference from the reference: reset_dE sums rows in index order,
//      where Eigen uses SIMD partial sums; identical for dyadic couplings.
//
//  (2) A replay of the B200 kernels' update order and counter-based random
//      stream (Philox4x32-10, Salmon et al., SC'11), FP32 fields, used to check
//      the kernels spin-for-spin.  It shares no code with the product: Philox,
//      the -ln(u) function and the greedy colouring are written again here.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cfloat>
#include <climits>
#include <random>
#include <vector>
#include <algorithm>
#include <functional>
#include <thread>
#include <atomic>

#if defined(__FP_FAST_FMAF) || defined(__FMA__)
#define ORC_FMAF(a, b, c) __builtin_fmaf((a), (b), (c))
#else
#define ORC_FMAF(a, b, c) std::fmaf((a), (b), (c))
#endif

namespace {

// ---------------------------------------------------------------------------
// (1) reference restatement
// ---------------------------------------------------------------------------

// random.hpp:39-87.  result_type is uint_fast32_t (8 bytes on x86-64 Linux),
// min()=0, max()=UINT_MAX; x, y, z fixed and the seed (truncated to unsigned)
// in w.
class Xorshift {
 public:
  using result_type = uint_fast32_t;
  static constexpr unsigned min() { return 0u; }
  static constexpr unsigned max() { return UINT_MAX; }
  explicit Xorshift(unsigned s) : w(s) {}
  unsigned operator()() {
    unsigned t = x ^ (x << 11);
    x = y;
    y = z;
    z = w;
    return w = (w ^ (w >> 19)) ^ (t ^ (t >> 8));
  }

 private:
  unsigned x = 123456789u, y = 362436069u, z = 521288629u, w;
};

// Symmetric augmented matrix ((n+1) x (n+1), h in row/column n, 1 in the
// corner) as CSR, exactly what Dense/CSRSparse::get_interactions() return.
struct Aug {
  int n;
  const int64_t* indptr;
  const int32_t* indices;
  const double* data;
};

template <class Eng>
std::vector<int> gen_spin(Eng& eng, int n) {  // graph.hpp:54-65
  std::vector<int> s(n);
  std::uniform_int_distribution<> uid(0, 1);
  for (auto& e : s) e = 2 * uid(eng) - 1;
  return s;
}

// classical_ising.hpp:87-90: dE = -2 s (J s)
void reset_dE(const Aug& g, const std::vector<double>& s, std::vector<double>& dE) {
  dE.assign(g.n + 1, 0.0);
  for (int i = 0; i <= g.n; ++i) {
    double acc = 0.0;
    for (int64_t p = g.indptr[i]; p < g.indptr[i + 1]; ++p) acc += g.data[p] * s[g.indices[p]];
    dE[i] = -2.0 * s[i] * acc;
  }
}

// single_spin_flip.hpp:66-95
template <class Eng>
void sa_update(const Aug& g, std::vector<double>& s, std::vector<double>& dE, Eng& eng, double beta) {
  auto urd = std::uniform_real_distribution<>(0, 1.0);
  const int n = g.n;
  for (int i = 0; i < n; ++i) {
    if (dE[i] <= 0 || std::exp(-beta * dE[i]) > urd(eng)) {
      const double si4 = 4 * s[i];
      for (int64_t p = g.indptr[i]; p < g.indptr[i + 1]; ++p) {
        const int j = g.indices[p];
        dE[j] += si4 * (g.data[p] * s[j]);
      }
      dE[i] *= -1;
      s[i] *= -1;
    }
    s[n] = 1;
  }
}

// Trotter spins stored slice-major: S[t*(n+1) + i]; dummy row i=n is 1.
// transverse_ising.hpp:165-186 / 537-558
void reset_dE_sqa(const Aug& g, int T, const std::vector<double>& S, std::vector<double>& dE) {
  const int n1 = g.n + 1;
  dE.assign((size_t)n1 * T, 0.0);
  for (int t = 0; t < T; ++t)
    for (int i = 0; i < n1; ++i) {
      double acc = 0.0;
      for (int64_t p = g.indptr[i]; p < g.indptr[i + 1]; ++p)
        acc += g.data[p] * S[(size_t)t * n1 + g.indices[p]];
      dE[(size_t)t * n1 + i] = -2 * S[(size_t)t * n1 + i] * acc;
    }
}

// single_spin_flip.hpp:196-251 (do_calc)
void sqa_do_calc(const Aug& g, int T, std::vector<double>& S, std::vector<double>& dE,
                 const std::vector<double>& rp, double beta, double s, int i, int t, double B) {
  const int n1 = g.n + 1;
  auto at = [&](int ii, int tt) -> double& { return S[(size_t)tt * n1 + ii]; };
  const int tp = (t + 1 + T) % T, tm = (t - 1 + T) % T;
  double dEtrot = -2 * at(i, t) * (at(i, tp) + at(i, tm));
  double dEv = s * (beta / T) * dE[(size_t)t * n1 + i] + B * dEtrot;
  if (dEv < 0 || std::exp(-dEv) > rp[(size_t)t * n1 + i]) {
    const double si4 = 4 * at(i, t);
    for (int64_t p = g.indptr[i]; p < g.indptr[i + 1]; ++p) {
      const int j = g.indices[p];
      dE[(size_t)t * n1 + j] += si4 * (g.data[p] * at(j, t));
    }
    dE[(size_t)t * n1 + i] *= -1;
    at(i, t) *= -1;
  }
}

// single_spin_flip.hpp:127-193
template <class Eng>
void sqa_update(const Aug& g, int T, std::vector<double>& S, std::vector<double>& dE,
                std::vector<double>& rp, Eng& eng, double beta, double gamma, double s) {
  const int n = g.n, n1 = n + 1;
  auto urd = std::uniform_real_distribution<>(0, 1.0);
  double B = (1 / 2.) * log(tanh(beta * gamma * (1.0 - s) / (double)(size_t)T));
  for (int t = 0; t < T; ++t)
    for (int i = 0; i < n; ++i) rp[(size_t)t * n1 + i] = urd(eng);
  const int upper = (T % 2 != 0) ? T - 1 : T;
  for (int t = 0; t < upper; t += 2)
    for (int i = 0; i < n; ++i) sqa_do_calc(g, T, S, dE, rp, beta, s, i, t, B);
  for (int t = 1; t < T; t += 2)
    for (int i = 0; i < n; ++i) sqa_do_calc(g, T, S, dE, rp, beta, s, i, t, B);
  if (T % 2 != 0) {
    const int t = T - 1;
    for (int i = 0; i < n; ++i) sqa_do_calc(g, T, S, dE, rp, beta, s, i, t, B);
  }
}

// ---------------------------------------------------------------------------
// (2) replay of the B200 kernels
// ---------------------------------------------------------------------------

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
// increments 0x9E3779B9 / 0xBB67AE85, 10 rounds.
struct P4 {
  uint32_t v[4];
};
P4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
  }
  return P4{{c0, c1, c2, c3}};
}

constexpr uint32_t TAG_SA = 0x5Au;       // c3 of the generic / dense SA stream
constexpr uint32_t TAG_SQA = 0xA5u;      // low byte of c3 of the SQA stream
constexpr uint32_t TAG_SA_MSC = 0x3Cu;   // low byte of c3 of the bit-packed SA stream
constexpr uint32_t TAG_SQA_MSC = 0xC3u;    // low byte of c3 of the bit-packed SQA stream
constexpr uint32_t TAG_SQA_SPLIT = 0x69u;  // low byte of c3 of the slice-split SQA stream
constexpr uint32_t TAG_BATCH = 0x96u;      // low byte of c3 of the batched dense SA stream
constexpr uint32_t TAG_SW_BOND = 0xB1u;    // Swendsen-Wang bond draws
constexpr uint32_t TAG_SW_FLIP = 0xB2u;    // Swendsen-Wang cluster coins

inline float f_of(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}
inline uint32_t b_of(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  return b;
}

// -ln(u) for u = (2*(x>>9)+1) * 2^-24, by m*2^e reduction to [sqrt(1/2),
// sqrt(2)] and ln m = t + t^2 Q(t), t = m - 1, Q a degree-6 polynomial fitted
// by least squares at Chebyshev nodes to (ln(1+t) - t) / t^2 (no division;
// error below 6e-8).  Every step is one IEEE round-to-nearest operation, so
// this and the device copy give the same bits.
float neglog(uint32_t x) {
  const uint32_t k = x >> 9;
  const float u = (float)(2u * k + 1u) * 0x1p-24f;
  const uint32_t b = b_of(u);
  int e = (int)(b >> 23) - 127;
  float m = f_of((b & 0x007FFFFFu) | 0x3F800000u);
  if (m > 0x1.6a09e6p+0f) {
    m = m * 0.5f;
    e += 1;
  }
  const float t = m - 1.0f;
  const float t2 = t * t;
  float q = -0x1.8e99cep-4f;
  q = ORC_FMAF(q, t, 0x1.4c9576p-3f);
  q = ORC_FMAF(q, t, -0x1.6420eep-3f);
  q = ORC_FMAF(q, t, 0x1.979cccp-3f);
  q = ORC_FMAF(q, t, -0x1.ff1d5ep-3f);
  q = ORC_FMAF(q, t, 0x1.5558fcp-2f);
  q = ORC_FMAF(q, t, -0x1.0000ecp-1f);
  const float lnm = ORC_FMAF(t2, q, t);
  const float lnu = ORC_FMAF((float)e, 0x1.62e430p-1f, lnm);
  return -lnu;
}

// Greedy first-fit colouring in index order over a neighbour list.
std::vector<int> greedy_colour(int n, const int64_t* rp, const int32_t* ci) {
  std::vector<int> col(n, -1);
  std::vector<int> seen;
  for (int i = 0; i < n; ++i) {
    seen.assign(seen.size(), 0);
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
      const int j = ci[p];
      if (j < i && col[j] >= 0) {
        if ((size_t)col[j] >= seen.size()) seen.resize(col[j] + 1, 0);
        seen[col[j]] = 1;
      }
    }
    int c = 0;
    while ((size_t)c < seen.size() && seen[c]) ++c;
    col[i] = c;
    if ((size_t)c >= seen.size()) seen.resize(c + 1, 0);
  }
  return col;
}

// The colouring the colour-class kernels use: two colours for a bipartite
// graph (two_colour), else the greedy colouring above, with its classes evened
// out.  With target t = ceil(n / ncol), each pass goes over
// the sites 0..n-1 and puts a site whose class holds more than t sites into
// the smallest-index colour whose class holds fewer than t sites and none of
// the site's neighbours; passes stop after one without a move, or after 8.
// A bipartite graph takes two colours: site 0 of every component (the
// smallest index) gets colour 0 and the rest alternate along a breadth-first
// search; false if an odd cycle shows up.
bool two_colour(int n, const int64_t* rp, const int32_t* ci, std::vector<int>& col) {
  col.assign(n, -1);
  std::vector<int> queue;
  for (int s = 0; s < n; ++s) {
    if (col[s] >= 0) continue;
    col[s] = 0;
    queue.assign(1, s);
    for (size_t h = 0; h < queue.size(); ++h) {
      const int u = queue[h];
      for (int64_t p = rp[u]; p < rp[u + 1]; ++p) {
        const int v = ci[p];
        if (col[v] < 0) {
          col[v] = 1 - col[u];
          queue.push_back(v);
        } else if (col[v] == col[u]) {
          return false;
        }
      }
    }
  }
  return true;
}

std::vector<int> kernel_colour(int n, const int64_t* rp, const int32_t* ci) {
  std::vector<int> col;
  if (!two_colour(n, rp, ci, col)) col = greedy_colour(n, rp, ci);
  int ncol = 0;
  for (int c : col) ncol = std::max(ncol, c + 1);
  if (ncol < 2) return col;
  const int t = (n + ncol - 1) / ncol;
  std::vector<int> cnt(ncol, 0);
  for (int c : col) ++cnt[c];
  for (int pass = 0; pass < 8; ++pass) {
    int moves = 0;
    for (int i = 0; i < n; ++i) {
      if (cnt[col[i]] <= t) continue;
      std::vector<char> used(ncol, 0);
      for (int64_t p = rp[i]; p < rp[i + 1]; ++p) used[col[ci[p]]] = 1;
      for (int c = 0; c < ncol; ++c) {
        if (cnt[c] >= t || used[c]) continue;
        --cnt[col[i]];
        ++cnt[c];
        col[i] = c;
        ++moves;
        break;
      }
    }
    if (moves == 0) break;
  }
  return col;
}

// Site neighbour lists (excluding the diagonal and the dummy column n) in CSR
// column order, and h_i, both rounded to FP32 — the data the kernels hold.
struct Nbr {
  int n;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<float> val;
  std::vector<float> h;
};
Nbr make_nbr(const Aug& g) {
  Nbr b;
  b.n = g.n;
  b.rp.assign(g.n + 1, 0);
  b.h.assign(g.n, 0.f);
  for (int i = 0; i < g.n; ++i) {
    for (int64_t p = g.indptr[i]; p < g.indptr[i + 1]; ++p) {
      const int j = g.indices[p];
      if (j == g.n) {
        b.h[i] = (float)g.data[p];
      } else if (j != i && g.data[p] != 0.0) {
        b.ci.push_back(j);
        b.val.push_back((float)g.data[p]);
      }
    }
    b.rp[i + 1] = (int64_t)b.ci.size();
  }
  return b;
}

template <class F>
void parallel_for(int count, int threads, F&& f) {
  if (threads <= 1 || count <= 1) {
    for (int i = 0; i < count; ++i) f(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < std::min(threads, count); ++t)
    pool.emplace_back([&]() {
      for (int i = next++; i < count; i = next++) f(i);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// ----- building blocks exposed for known-answer tests -----------------------

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  P4 r = philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

float orc_neglog(uint32_t x) { return neglog(x); }
// the largest -ln u over every input (k = x >> 9 takes 2^23 values)
float orc_neglog_max() {
  float m = 0.0f;
  for (uint32_t k = 0; k < (1u << 23); ++k) m = std::max(m, neglog(k << 9));
  return m;
}

void orc_greedy_colour(int n, const int64_t* rp, const int32_t* ci, int32_t* out) {
  auto c = greedy_colour(n, rp, ci);
  for (int i = 0; i < n; ++i) out[i] = c[i];
}

void orc_kernel_colour(int n, const int64_t* rp, const int32_t* ci, int32_t* out) {
  auto c = kernel_colour(n, rp, ci);
  for (int i = 0; i < n; ++i) out[i] = c[i];
}

// engine: 0 = Xorshift (openjij compile_config.hpp:45), 1 = std::mt19937
void orc_gen_spin(uint64_t seed, int n, int engine, int8_t* out) {
  std::vector<int> s;
  if (engine == 0) {
    Xorshift e((unsigned)seed);
    s = gen_spin(e, n);
  } else {
    std::mt19937 e((std::mt19937::result_type)seed);
    s = gen_spin(e, n);
  }
  for (int i = 0; i < n; ++i) out[i] = (int8_t)s[i];
}

// `count` consecutive gen_spin() draws from one engine (the reference's
// Trotter initialisation in tests/cxxtest/sampler/quadraitc.hpp:84-87).
void orc_gen_spin_seq(uint64_t seed, int n, int count, int engine, int8_t* out) {
  auto run = [&](auto& e) {
    for (int c = 0; c < count; ++c) {
      auto s = gen_spin(e, n);
      for (int i = 0; i < n; ++i) out[(size_t)c * n + i] = (int8_t)s[i];
    }
  };
  if (engine == 0) {
    Xorshift e((unsigned)seed);
    run(e);
  } else {
    std::mt19937 e((std::mt19937::result_type)seed);
    run(e);
  }
}

// schedule_list.hpp:165-181
void orc_classical_schedule(double beta_min, double beta_max, int64_t num_call, double* out) {
  double r = std::pow(beta_max / beta_min, 1.0 / static_cast<double>(num_call - 1));
  double beta = beta_min;
  for (int64_t k = 0; k < num_call; ++k) {
    out[k] = beta;
    beta *= r;
  }
}

// schedule_list.hpp:193-207
void orc_transverse_schedule(int64_t num_call, double* out_s) {
  double ds = 1.0 / static_cast<double>(num_call - 1);
  double s = 0;
  for (int64_t k = 0; k < num_call; ++k) {
    out_s[k] = s;
    s += ds;
  }
}

// dense.hpp:176-192 / csr_sparse.hpp:139-155 (upper triangle, minus the corner)
double orc_energy(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                  const int8_t* spins) {
  double e = 0.0;
  for (int i = 0; i <= n; ++i) {
    const double si = i < n ? spins[i] : 1.0;
    double acc = 0.0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      const int j = indices[p];
      if (j < i) continue;
      acc += data[p] * (j < n ? spins[j] : 1.0);
    }
    e += si * acc;
  }
  return e - 1.0;
}

// Reference SA (one read): spins in/out [n]; schedule of (beta_k, mcs_k).
// engine: 0 Xorshift, 1 mt19937.
void orc_ref_sa(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                int8_t* spins, const double* betas, const int64_t* mcs, int64_t nsched,
                uint64_t seed, int engine) {
  Aug g{n, indptr, indices, data};
  std::vector<double> s(n + 1), dE;
  for (int i = 0; i < n; ++i) s[i] = spins[i];
  s[n] = 1;
  reset_dE(g, s, dE);
  auto run = [&](auto& eng) {
    for (int64_t k = 0; k < nsched; ++k)
      for (int64_t m = 0; m < mcs[k]; ++m) sa_update(g, s, dE, eng, betas[k]);
  };
  if (engine == 0) {
    Xorshift e((unsigned)seed);
    run(e);
  } else {
    std::mt19937 e((std::mt19937::result_type)seed);
    run(e);
  }
  for (int i = 0; i < n; ++i) spins[i] = (int8_t)(s[i] * s[n]);  // get_solution.hpp:45-46
}

// Many independent reference reads on all host threads, read r seeded with
// seeds[r] and started from spins[r*n...].  Used as the timed CPU baseline.
void orc_ref_sa_many(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                     int num_reads, int8_t* spins, const double* betas, const int64_t* mcs,
                     int64_t nsched, const uint64_t* seeds, int threads) {
  parallel_for(num_reads, threads, [&](int r) {
    orc_ref_sa(n, indptr, indices, data, spins + (size_t)r * n, betas, mcs, nsched, seeds[r], 0);
  });
}

// Reference SQA (one read): trotter spins in/out [T][n]; schedule (beta_k, s_k,
// mcs_k).  out_best: the get_solution() slice (get_solution.hpp:59-84).
void orc_ref_sqa(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                 int T, int8_t* tspins, double gamma, const double* betas, const double* ss,
                 const int64_t* mcs, int64_t nsched, uint64_t seed, int engine,
                 int8_t* out_best) {
  Aug g{n, indptr, indices, data};
  const int n1 = n + 1;
  std::vector<double> S((size_t)n1 * T), dE, rp((size_t)n1 * T, 0.0);
  for (int t = 0; t < T; ++t) {
    for (int i = 0; i < n; ++i) S[(size_t)t * n1 + i] = tspins[(size_t)t * n + i];
    S[(size_t)t * n1 + n] = 1;
  }
  reset_dE_sqa(g, T, S, dE);
  auto run = [&](auto& eng) {
    for (int64_t k = 0; k < nsched; ++k)
      for (int64_t m = 0; m < mcs[k]; ++m) sqa_update(g, T, S, dE, rp, eng, betas[k], gamma, ss[k]);
  };
  if (engine == 0) {
    Xorshift e((unsigned)seed);
    run(e);
  } else {
    std::mt19937 e((std::mt19937::result_type)seed);
    run(e);
  }
  for (int t = 0; t < T; ++t)
    for (int i = 0; i < n; ++i) tspins[(size_t)t * n + i] = (int8_t)S[(size_t)t * n1 + i];
  // get_solution: slice with minimum s^T J s (full symmetric J), first wins.
  int best = 0;
  double emin = DBL_MAX;
  for (int t = 0; t < T; ++t) {
    double e = 0.0;
    for (int i = 0; i < n1; ++i) {
      double acc = 0.0;
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) acc += data[p] * S[(size_t)t * n1 + indices[p]];
      e += S[(size_t)t * n1 + i] * acc;
    }
    if (e < emin) {
      best = t;
      emin = e;
    }
  }
  if (out_best)
    for (int i = 0; i < n; ++i) out_best[i] = (int8_t)S[(size_t)best * n1 + i];
}

void orc_ref_sqa_many(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                      int num_reads, int T, int8_t* tspins, double gamma, const double* betas,
                      const double* ss, const int64_t* mcs, int64_t nsched, const uint64_t* seeds,
                      int threads) {
  parallel_for(num_reads, threads, [&](int r) {
    orc_ref_sqa(n, indptr, indices, data, T, tspins + (size_t)r * T * n, gamma, betas, ss, mcs,
                nsched, seeds[r], 0, nullptr);
  });
}

// ----- replays of the GPU kernels ------------------------------------------

// Generic colour-class SA (sparse) and sequential dense SA share one stream:
// u(r, k, i) = Philox(ctr = (i, k, r>>2, TAG_SA), key = seed)[r & 3].
// mode 0: colour-class order (greedy colouring), fields gathered every attempt
//         in neighbour order starting from h_i;
// mode 1: sequential order i = 0..n-1 with FP32 fields kept incrementally
//         (initial f_i = h_i + sum_j J_ij s_j, j ascending).
// betas_f: one FP32 beta per sweep (schedule already expanded).
void orc_replay_sa(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                   int R, int8_t* spins, const float* betas_f, int64_t nsweeps, uint64_t seed,
                   int mode, int threads, uint32_t rep0, uint32_t sweep0) {
  Aug g{n, indptr, indices, data};
  Nbr b = make_nbr(g);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int> col = kernel_colour(n, b.rp.data(), b.ci.data());
  int ncol = 0;
  for (int c : col) ncol = std::max(ncol, c + 1);
  std::vector<std::vector<int>> by_col(ncol);
  for (int i = 0; i < n; ++i) by_col[col[i]].push_back(i);
  // dense row-major FP32 J for mode 1
  std::vector<float> Jd;
  if (mode == 1) {
    Jd.assign((size_t)n * n, 0.f);
    for (int i = 0; i < n; ++i)
      for (int64_t p = b.rp[i]; p < b.rp[i + 1]; ++p) Jd[(size_t)i * n + b.ci[p]] = b.val[p];
  }
  parallel_for(R, threads, [&](int r) {
    int8_t* s = spins + (size_t)r * n;
    const uint32_t rg = rep0 + (uint32_t)r;  // global replica index
    auto draw = [&](int i, int64_t k) {
      P4 q = philox((uint32_t)i, sweep0 + (uint32_t)k, rg >> 2, TAG_SA, k0, k1);
      return q.v[rg & 3];
    };
    if (mode == 0) {
      for (int64_t k = 0; k < nsweeps; ++k) {
        const float beta = betas_f[k];
        for (int c = 0; c < ncol; ++c)
          for (int i : by_col[c]) {
            float f = b.h[i];
            for (int64_t p = b.rp[i]; p < b.rp[i + 1]; ++p)
              f = f + (s[b.ci[p]] > 0 ? b.val[p] : -b.val[p]);
            const float dE = s[i] > 0 ? -2.0f * f : 2.0f * f;
            const float L = neglog(draw(i, k));
            if (dE <= 0.0f || beta * dE < L) s[i] = (int8_t)-s[i];
          }
      }
    } else {
      std::vector<float> f(n);
      for (int i = 0; i < n; ++i) {
        float acc = b.h[i];
        for (int j = 0; j < n; ++j) {
          const float J = Jd[(size_t)i * n + j];
          acc = acc + (s[j] > 0 ? J : -J);
        }
        f[i] = acc;
      }
      for (int64_t k = 0; k < nsweeps; ++k) {
        const float beta = betas_f[k];
        for (int i = 0; i < n; ++i) {
          const float dE = s[i] > 0 ? -2.0f * f[i] : 2.0f * f[i];
          const float L = neglog(draw(i, k));
          if (dE <= 0.0f || beta * dE < L) {
            const float c = s[i] > 0 ? -2.0f : 2.0f;
            const float* Ji = &Jd[(size_t)i * n];
            for (int j = 0; j < n; ++j) f[j] = f[j] + c * Ji[j];
            s[i] = (int8_t)-s[i];
          }
        }
      }
    }
  });
}

// Generic SQA replay.  Stream: u(r, t, k, i) = Philox(ctr = (i, k, r,
// ((t>>3)<<9) | ((t&1)<<8) | TAG_SQA), key = seed)[(t>>1) & 3], so one Philox
// call serves the four slices t = 8a+p, 8a+p+2, 8a+p+4, 8a+p+6 of one parity.  Order per sweep: slice groups
// {even t < upper}, {odd t}, {T-1 if T odd} (single_spin_flip.hpp:163-192);
// inside a group, colour classes of the spatial graph.  coef_a[k] = s*beta/T,
// coef_b[k] = 0.5*log(tanh(beta*gamma*(1-s)/T)), both FP32, per sweep.
void orc_replay_sqa(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                    int R, int T, int8_t* tspins, const float* coef_a, const float* coef_b,
                    int64_t nsweeps, uint64_t seed, int threads) {
  Aug g{n, indptr, indices, data};
  Nbr b = make_nbr(g);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int> col = kernel_colour(n, b.rp.data(), b.ci.data());
  int ncol = 0;
  for (int c : col) ncol = std::max(ncol, c + 1);
  std::vector<std::vector<int>> by_col(ncol);
  for (int i = 0; i < n; ++i) by_col[col[i]].push_back(i);
  const int upper = (T % 2 != 0) ? T - 1 : T;
  std::vector<std::vector<int>> groups(3);
  for (int t = 0; t < upper; t += 2) groups[0].push_back(t);
  for (int t = 1; t < T; t += 2) groups[1].push_back(t);
  if (T % 2 != 0) groups[2].push_back(T - 1);
  parallel_for(R, threads, [&](int r) {
    int8_t* S = tspins + (size_t)r * T * n;
    for (int64_t k = 0; k < nsweeps; ++k) {
      const float a = coef_a[k], B = coef_b[k];
      for (auto& grp : groups)
        for (int c = 0; c < ncol; ++c)
          for (int t : grp)
            for (int i : by_col[c]) {
              int8_t* St = S + (size_t)t * n;
              float f = b.h[i];
              for (int64_t p = b.rp[i]; p < b.rp[i + 1]; ++p)
                f = f + (St[b.ci[p]] > 0 ? b.val[p] : -b.val[p]);
              const float dEsp = St[i] > 0 ? -2.0f * f : 2.0f * f;
              const int tp = (t + 1) % T, tm = (t - 1 + T) % T;
              const int ssum = S[(size_t)tp * n + i] + S[(size_t)tm * n + i];
              const float dEtrot = (float)(-2 * St[i] * ssum);
              const float dE = a * dEsp + B * dEtrot;
              P4 q = philox((uint32_t)i, (uint32_t)k, (uint32_t)r,
                            (((uint32_t)t >> 3) << 9) | (((uint32_t)t & 1u) << 8) | TAG_SQA,
                            k0, k1);
              const float L = neglog(q.v[(t >> 1) & 3]);
              if (dE < L) St[i] = (int8_t)-St[i];
            }
    }
  });
}

// Bit-packed (multi-spin coded) SA replay for regular graphs with couplings
// +-c and h = 0.  Word (g, i) bit j = 1 iff replica 32g+j has s_i = -1.
// Per sweep k, per colour class, per site i, per group g:
//   unsat_l = b_i ^ b_j(l) ^ (J_ij(l) > 0 ? ~0 : 0); u = popcount per bit;
//   dE = 2c(d - 2u); bits with 2u >= d flip; the others flip iff
//   U < thr[k][d-2u] (32-bit compare), U's bit (31-l) of bit j taken from
//   word l of W(i, k, g) = Philox(ctr = (i, k, g, (l/4 << 8) | TAG_SA_MSC))[l%4].
//   always[k] bit m set: class m accepts unconditionally (beta == 0).
// thr: [nsweeps][dmax+1] u32 (index m), always: [nsweeps] u32.
void orc_replay_sa_msc(int n, const int64_t* indptr, const int32_t* indices, const double* data,
                       int G, uint32_t* words /*[G][n]*/, const uint32_t* thr, int dmax,
                       const uint32_t* always, int64_t nsweeps, uint64_t seed, int threads) {
  Aug g{n, indptr, indices, data};
  Nbr b = make_nbr(g);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int> col = kernel_colour(n, b.rp.data(), b.ci.data());
  int ncol = 0;
  for (int c : col) ncol = std::max(ncol, c + 1);
  std::vector<std::vector<int>> by_col(ncol);
  for (int i = 0; i < n; ++i) by_col[col[i]].push_back(i);
  parallel_for(G, threads, [&](int gi) {
    uint32_t* w = words + (size_t)gi * n;
    for (int64_t k = 0; k < nsweeps; ++k) {
      const uint32_t* th = thr + (size_t)k * (dmax + 1);
      for (int c = 0; c < ncol; ++c)
        for (int i : by_col[c]) {
          const int d = (int)(b.rp[i + 1] - b.rp[i]);
          const uint32_t wi = w[i];
          // per-bit unsatisfied count
          int cnt[32] = {0};
          for (int64_t p = b.rp[i]; p < b.rp[i + 1]; ++p) {
            const uint32_t jm = b.val[p] > 0 ? 0xFFFFFFFFu : 0u;
            const uint32_t un = wi ^ w[b.ci[p]] ^ jm;
            for (int j = 0; j < 32; ++j) cnt[j] += (un >> j) & 1u;
          }
          uint32_t flip = 0;
          uint32_t Wl[32];
          bool have = false;
          for (int j = 0; j < 32; ++j) {
            const int m = d - 2 * cnt[j];
            if (m <= 0 || ((always[k] >> m) & 1u)) {
              flip |= 1u << j;
              continue;
            }
            if (!have) {
              for (int q = 0; q < 8; ++q) {
                P4 r4 = philox((uint32_t)i, (uint32_t)k, (uint32_t)gi,
                               ((uint32_t)q << 8) | TAG_SA_MSC, k0, k1);
                for (int l = 0; l < 4; ++l) Wl[4 * q + l] = r4.v[l];
              }
              have = true;
            }
            uint32_t U = 0;
            for (int l = 0; l < 32; ++l) U |= ((Wl[l] >> j) & 1u) << (31 - l);
            if (U < th[m]) flip |= 1u << j;
          }
          w[i] = wi ^ flip;
        }
    }
  });
}

// Thresholds of the bit-packed SA kernel, computed with the host libm exactly
// as the product does: thr[k][m] = min(2^32-1, floor(exp(-beta_k*2c*m)*2^32)),
// m = 1..dmax; always[k] bit m set when exp(...) >= 1 (beta_k == 0).
void orc_msc_thresholds(const float* betas_f, int64_t nsweeps, double c, int dmax, uint32_t* thr,
                        uint32_t* always) {
  for (int64_t k = 0; k < nsweeps; ++k) {
    always[k] = 0;
    thr[(size_t)k * (dmax + 1)] = 0;
    for (int m = 1; m <= dmax; ++m) {
      const double p = std::exp(-(double)betas_f[k] * 2.0 * c * (double)m);
      const double t = std::floor(std::ldexp(p, 32));
      uint32_t v;
      if (p >= 1.0) {
        always[k] |= 1u << m;
        v = 0xFFFFFFFFu;
      } else {
        v = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
      }
      thr[(size_t)k * (dmax + 1) + m] = v;
    }
  }
}

// Per-sweep SQA coefficients as the product computes them (host libm):
// a = s*(beta/T), b = 0.5*log(tanh(beta*gamma*(1-s)/T))  (single_spin_flip.hpp:147-148,216-217)
void orc_sqa_coefficients(const double* betas, const double* ss, int64_t count, double gamma, int T,
                          float* a, float* b) {
  for (int64_t k = 0; k < count; ++k) {
    a[k] = (float)(ss[k] * (betas[k] / (double)(size_t)T));
    b[k] = (float)((1 / 2.) * std::log(std::tanh(betas[k] * gamma * (1.0 - ss[k]) / (double)(size_t)T)));
  }
}

// Bit-packed SQA replay (regular graph, couplings +-c, h = 0, T <= 32).
// Word (r, i) bit t = 1 iff slice t of replica r has s_i = -1.  Order: per
// sweep k, slice groups {even t < T - T%2}, {odd t}, {T-1 if T odd} (grp 0, 1,
// 2), per colour class, per site i of the class, every slice t of the group:
//   u = unsatisfied bonds of (i, t); kk = Trotter neighbours t+-1 (mod T) with
//   the same spin; class m = 3u + kk;
//   always[k] bit m -> flip; live[k] bit m -> flip iff U < thr[k][m], where U's
//   bit (31 - l) is bit t of W_l = Philox(ctr = (i, k, r, (l/4) << 16 | grp << 8
//   | TAG_SQA_MSC))[l % 4]; otherwise no flip.
// The slices of one group are decided from the word before the group's update
// (they are never Trotter neighbours of each other, except t = 0 and T-1 with
// T odd, which sit in different groups).
// thr: [nsweeps][(dmax+1)*3], mode: [nsweeps][2] = (always, live).
void orc_replay_sqa_msc(int n, const int64_t* indptr, const int32_t* indices, const double* data, int R,
                        int T, uint32_t* words /*[R][n]*/, const uint32_t* thr, const uint32_t* mode, int dmax,
                        int64_t nsweeps, uint64_t seed, int threads) {
  Aug g{n, indptr, indices, data};
  Nbr b = make_nbr(g);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int> col = kernel_colour(n, b.rp.data(), b.ci.data());
  int ncol = 0;
  for (int c : col) ncol = std::max(ncol, c + 1);
  std::vector<std::vector<int>> by_col(ncol);
  for (int i = 0; i < n; ++i) by_col[col[i]].push_back(i);
  const int upper = (T % 2 != 0) ? T - 1 : T;
  std::vector<std::vector<int>> groups(3);
  for (int t = 0; t < upper; t += 2) groups[0].push_back(t);
  for (int t = 1; t < T; t += 2) groups[1].push_back(t);
  if (T % 2 != 0) groups[2].push_back(T - 1);
  const int NC = (dmax + 1) * 3;
  parallel_for(R, threads, [&](int r) {
    uint32_t* w = words + (size_t)r * n;
    for (int64_t k = 0; k < nsweeps; ++k) {
      const uint32_t* th = thr + (size_t)k * NC;
      const uint32_t always = mode[2 * k], live = mode[2 * k + 1];
      for (int grp = 0; grp < 3; ++grp) {
        if (groups[grp].empty()) continue;
        for (int c = 0; c < ncol; ++c)
          for (int i : by_col[c]) {
            const uint32_t wi = w[i];
            uint32_t Wl[32];
            for (int q = 0; q < 8; ++q) {
              P4 r4 = philox((uint32_t)i, (uint32_t)k, (uint32_t)r,
                             ((uint32_t)q << 16) | ((uint32_t)grp << 8) | TAG_SQA_MSC, k0, k1);
              for (int l = 0; l < 4; ++l) Wl[4 * q + l] = r4.v[l];
            }
            uint32_t flip = 0;
            for (int t : groups[grp]) {
              const int bi = (wi >> t) & 1;
              int u = 0;
              for (int64_t p = b.rp[i]; p < b.rp[i + 1]; ++p) {
                const int bj = (w[b.ci[p]] >> t) & 1;
                // J s_i s_j > 0: unsatisfied; s_i s_j = +1 iff the bits agree
                const bool same = bi == bj;
                if ((b.val[p] > 0) == same) ++u;
              }
              const int tp = (t + 1) % T, tm = (t - 1 + T) % T;
              const int kk = (((wi >> tp) & 1) == (uint32_t)bi) + (((wi >> tm) & 1) == (uint32_t)bi);
              const int m = 3 * u + kk;
              if ((always >> m) & 1u) {
                flip |= 1u << t;
              } else if ((live >> m) & 1u) {
                uint32_t U = 0;
                for (int l = 0; l < 32; ++l) U |= ((Wl[l] >> t) & 1u) << (31 - l);
                if (U < th[m]) flip |= 1u << t;
              }
            }
            w[i] = wi ^ flip;
          }
      }
    }
  });
}

// Thresholds of the bit-packed SQA kernel from the per-sweep FP32 coefficients
// (a, B): for class m = 3u + kk, dE = a*float(2c(dmax-2u)) + B*float(4-4kk)
// (FP32, products and sum each rounded once); dE <= 0 -> always; NaN -> never;
// else thr = min(2^32-1, floor(exp(-dE)*2^32)), live when thr > 0.
void orc_sqa_msc_thresholds(const float* coef_a, const float* coef_b, int64_t nsweeps, double c, int dmax,
                            uint32_t* thr, uint32_t* mode) {
  const int NC = (dmax + 1) * 3;
  for (int64_t k = 0; k < nsweeps; ++k) {
    uint32_t always = 0, live = 0;
    for (int u = 0; u <= dmax; ++u)
      for (int kk = 0; kk < 3; ++kk) {
        const int m = 3 * u + kk;
        const float dEsp = (float)(2.0 * c * (double)(dmax - 2 * u));
        const float dEtrot = (float)(4 - 4 * kk);
        const float p1 = coef_a[k] * dEsp;
        const float p2 = coef_b[k] * dEtrot;
        const float dE = p1 + p2;
        uint32_t v = 0;
        if (dE != dE) {
          v = 0;
        } else if (dE <= 0.0f) {
          always |= 1u << m;
        } else {
          const double t = std::floor(std::ldexp(std::exp(-(double)dE), 32));
          v = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
          if (v) live |= 1u << m;
        }
        thr[(size_t)k * NC + m] = v;
      }
    mode[2 * k] = always;
    mode[2 * k + 1] = live;
  }
}

// Slice-split bit-packed SQA replay (regular graph, couplings +-c, h = 0, even
// T <= 64), on spins [R][T][n].  H = T/2, P = largest power of two with
// P*H <= 32; replica r belongs to group g = r / P and its slice t to bit
// b = (r % P)*H + t/2 of half q = t % 2.  Order: per sweep k, half q = 0 (even
// slices) then q = 1 (odd slices), per colour class, per site i of the class,
// every slice t of the half:
//   u = unsatisfied bonds of (i, t); kk = Trotter neighbours t+-1 (mod T) with
//   the same spin; class m = 3u + kk;
//   always[k] bit m -> flip; live[k] bit m -> flip iff U < thr[k][m], where U's
//   bit (31 - l) is bit b of W_l = Philox(ctr = (i, k, g, (l/4) << 16 | q << 8 |
//   TAG_SQA_SPLIT))[l % 4]; otherwise no flip.
// The slices of one half are not Trotter neighbours of each other, so updating
// them one after another equals deciding them together.
void orc_replay_sqa_split(int n, const int64_t* indptr, const int32_t* indices, const double* data, int R,
                          int T, int8_t* tspins /*[R][T][n]*/, const uint32_t* thr, const uint32_t* mode,
                          int dmax, int64_t nsweeps, uint64_t seed, int threads) {
  Aug g{n, indptr, indices, data};
  Nbr b = make_nbr(g);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int> col = kernel_colour(n, b.rp.data(), b.ci.data());
  int ncol = 0;
  for (int c : col) ncol = std::max(ncol, c + 1);
  std::vector<std::vector<int>> by_col(ncol);
  for (int i = 0; i < n; ++i) by_col[col[i]].push_back(i);
  const int H = T / 2;
  int P = 1;
  while (2 * P * H <= 32) P *= 2;
  const int NC = (dmax + 1) * 3;
  const int G = (R + P - 1) / P;
  parallel_for(G, threads, [&](int gi) {
    for (int64_t k = 0; k < nsweeps; ++k) {
      const uint32_t* th = thr + (size_t)k * NC;
      const uint32_t always = mode[2 * k], live = mode[2 * k + 1];
      for (int q = 0; q < 2; ++q)
        for (int c = 0; c < ncol; ++c)
          for (int i : by_col[c]) {
            uint32_t Wl[32];
            for (int qq = 0; qq < 8; ++qq) {
              P4 r4 = philox((uint32_t)i, (uint32_t)k, (uint32_t)gi,
                             ((uint32_t)qq << 16) | ((uint32_t)q << 8) | TAG_SQA_SPLIT, k0, k1);
              for (int l = 0; l < 4; ++l) Wl[4 * qq + l] = r4.v[l];
            }
            for (int p = 0; p < P; ++p) {
              const int r = gi * P + p;
              if (r >= R) break;
              int8_t* S = tspins + (size_t)r * T * n;
              for (int t = q; t < T; t += 2) {
                const int bit = p * H + t / 2;
                const int si = S[(size_t)t * n + i];
                int u = 0;
                for (int64_t e = b.rp[i]; e < b.rp[i + 1]; ++e)
                  if (b.val[e] * si * S[(size_t)t * n + b.ci[e]] > 0) ++u;
                const int tp = (t + 1) % T, tm = (t - 1 + T) % T;
                const int kk = (S[(size_t)tp * n + i] == si) + (S[(size_t)tm * n + i] == si);
                const int m = 3 * u + kk;
                bool flip = false;
                if ((always >> m) & 1u) {
                  flip = true;
                } else if ((live >> m) & 1u) {
                  uint32_t U = 0;
                  for (int l = 0; l < 32; ++l) U |= ((Wl[l] >> bit) & 1u) << (31 - l);
                  flip = U < th[m];
                }
                if (flip) S[(size_t)t * n + i] = (int8_t)-si;
              }
            }
          }
    }
  });
}

// Batched dense SA replay.  Instance m has n[m] spins and its augmented
// (n+1)^2 FP64 matrix at J_aug + offset[m]; the dynamics use FP32 J and h.
// Each replica r of instance m runs the sequential sweep of mode 1 above
// (sites 0..n-1, accept when dE <= 0 or beta*dE < -ln(u), fields moved by
// c*J_ij with c = -2 s_i) with u(m, r, k, i) = Philox(ctr = (i >> 2, k, r,
// (inst0 + m) << 8 | TAG_BATCH))[i & 3].  spins: the instances' [reads[m]][n[m]]
// blocks concatenated.
void orc_replay_sa_batch(int count, const int32_t* n_arr, const int64_t* offset, const double* J_aug,
                         const int32_t* reads, int8_t* spins, const float* betas_f, int64_t nsweeps,
                         uint64_t seed, uint32_t inst0, int threads, float* fields_out, uint32_t rep0,
                         uint32_t sweep0, int recompute, float* drift_out) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int64_t> soff(count + 1, 0), roff(count + 1, 0);
  std::vector<int> rm, rr;  // flattened (instance, replica)
  for (int m = 0; m < count; ++m) {
    soff[m + 1] = soff[m] + (int64_t)reads[m] * n_arr[m];
    roff[m + 1] = roff[m] + reads[m];
    for (int r = 0; r < reads[m]; ++r) {
      rm.push_back(m);
      rr.push_back(r);
    }
  }
  parallel_for((int)rm.size(), threads, [&](int qx) {
    const int m = rm[qx], r = rr[qx], n = n_arr[m];
    const int64_t n1 = n + 1;
    const double* A = J_aug + offset[m];
    std::vector<float> J((size_t)n * n), h(n), f(n), fq(n);
    float amax = 0.0f;
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) {
        J[(size_t)i * n + j] = (float)A[i * n1 + j];
        amax = std::max(amax, std::fabs(J[(size_t)i * n + j]));
      }
      h[i] = (float)A[i * n1 + n];
    }
    // The field definition of the tensor-core field kernel: J on the grid
    // 2^e, e = E - 26 with 2^(E-1) <= max|J| < 2^E, q = J / 2^e rounded half
    // to even; f_j = fp32(fp64(h_j) + 2^e * sum_i q_ij s_i), the sum exact.
    int E = 0;
    if (amax > 0.0f) std::frexp((double)amax, &E);
    const int e = amax > 0.0f ? E - 26 : 0;
    std::vector<int64_t> q((size_t)n * n);
    for (size_t t = 0; t < q.size(); ++t) q[t] = (int64_t)std::nearbyint(std::ldexp((double)J[t], -e));
    int8_t* s = spins + soff[m] + (size_t)r * n;
    auto qfield = [&](std::vector<float>& out) {
      for (int j = 0; j < n; ++j) {
        int64_t acc = 0;
        const int64_t* qj = &q[(size_t)j * n];  // J symmetric: row j holds column j
        for (int i = 0; i < n; ++i) acc += s[i] > 0 ? qj[i] : -qj[i];
        out[j] = (float)((double)h[j] + std::ldexp((double)acc, e));
      }
    };
    float drift = 0.0f;
    auto recompute_now = [&]() {
      qfield(fq);
      for (int j = 0; j < n; ++j) {
        drift = std::max(drift, std::fabs(fq[j] - f[j]));
        f[j] = fq[j];
      }
    };
    qfield(f);
    const uint32_t tag = ((inst0 + (uint32_t)m) << 8) | TAG_BATCH;
    for (int64_t k = 0; k < nsweeps; ++k) {
      const uint32_t g = sweep0 + (uint32_t)k;
      // fields anew before every global sweep that is a multiple of the interval
      if (recompute > 0 && k > 0 && g % (uint32_t)recompute == 0) recompute_now();
      const float beta = betas_f[k];
      for (int i = 0; i < n; ++i) {
        const float dE = s[i] > 0 ? -2.0f * f[i] : 2.0f * f[i];
        const P4 u = philox((uint32_t)(i >> 2), g, rep0 + (uint32_t)r, tag, k0, k1);
        const float L = neglog(u.v[i & 3]);
        if (dE <= 0.0f || beta * dE < L) {
          const float c = s[i] > 0 ? -2.0f : 2.0f;
          const float* Ji = &J[(size_t)i * n];
          for (int j = 0; j < n; ++j) f[j] = f[j] + c * Ji[j];
          s[i] = (int8_t)-s[i];
        }
      }
    }
    // the incrementally updated FP32 fields at the end (same layout as spins)
    if (fields_out)
      for (int j = 0; j < n; ++j) fields_out[soff[m] + (size_t)r * n + j] = f[j];
    // the drift at the recompute points and against the final spins' fields
    if (drift_out) {
      qfield(fq);
      for (int j = 0; j < n; ++j) drift = std::max(drift, std::fabs(fq[j] - f[j]));
      drift_out[roff[m] + r] = drift;
    }
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Swendsen-Wang
// ---------------------------------------------------------------------------

// Reference Swendsen-Wang (include/openjij/updater/swendsen_wang.hpp:43-182 with
// include/openjij/utility/union_find.hpp): one read, spins in/out [n], the
// dummy spin n starts at +1, result s_i * s_n (get_solution.hpp:45-46).
namespace {
struct RefUnionFind {  // union_find.hpp: union by rank, path compression
  std::vector<size_t> parent, rank;
  explicit RefUnionFind(size_t n) : parent(n), rank(n, 0) {
    for (size_t i = 0; i < n; ++i) parent[i] = i;
  }
  size_t find(size_t node) {
    size_t base = node, p = parent[node];
    while (p != node) {
      node = p;
      p = parent[node];
    }
    const size_t root = p;
    node = parent[base];
    while (root != node) {
      parent[base] = root;
      base = node;
      node = parent[base];
    }
    return root;
  }
  void unite(size_t x, size_t y) {
    size_t rx = find(x), ry = find(y);
    if (rx == ry) return;
    if (rank[rx] > rank[ry]) {
      parent[ry] = rx;
    } else {
      parent[rx] = ry;
      if (rank[rx] == rank[ry]) ++rank[ry];
    }
  }
};

template <class Eng>
void ref_sw_update(const Aug& g, std::vector<double>& s, Eng& eng, double beta) {
  auto urd = std::uniform_real_distribution<>(0, 1.0);
  const size_t N = (size_t)g.n + 1;
  RefUnionFind uf(N);
  for (size_t node = 0; node < N; ++node)
    for (int64_t p = g.indptr[node]; p < g.indptr[node + 1]; ++p) {
      const size_t adj = (size_t)g.indices[p];
      const double J = g.data[p];
      if (node >= adj) continue;
      if (J * s[node] * s[adj] > 0) continue;
      const double rate = std::max(0.0, 1.0 - std::exp(-2.0 * beta * std::abs(J)));
      if (urd(eng) < rate) uf.unite(node, adj);
    }
  std::vector<std::vector<size_t>> members(N);
  for (size_t node = 0; node < N; ++node) members[uf.find(node)].push_back(node);
  std::vector<size_t> roots = uf.parent;  // get_roots(): sorted unique parents
  std::sort(roots.begin(), roots.end());
  roots.erase(std::unique(roots.begin(), roots.end()), roots.end());
  for (size_t c : roots)
    if (urd(eng) < 0.5)
      for (size_t i : members[c]) s[i] *= -1;
}
}  // namespace

extern "C" {

void orc_ref_sw(int n, const int64_t* indptr, const int32_t* indices, const double* data, int8_t* spins,
                const double* betas, const int64_t* mcs, int64_t nsched, uint64_t seed) {
  Aug g{n, indptr, indices, data};
  std::vector<double> s(n + 1);
  for (int i = 0; i < n; ++i) s[i] = spins[i];
  s[n] = 1;
  Xorshift e((unsigned)seed);
  for (int64_t k = 0; k < nsched; ++k)
    for (int64_t m = 0; m < mcs[k]; ++m) ref_sw_update(g, s, e, betas[k]);
  for (int i = 0; i < n; ++i) spins[i] = (int8_t)(s[i] * s[n]);
}

void orc_ref_sw_many(int n, const int64_t* indptr, const int32_t* indices, const double* data, int num_reads,
                     int8_t* spins, const double* betas, const int64_t* mcs, int64_t nsched, const uint64_t* seeds,
                     int threads) {
  parallel_for(num_reads, threads, [&](int r) {
    orc_ref_sw(n, indptr, indices, data, spins + (size_t)r * n, betas, mcs, nsched, seeds[r]);
  });
}

// Replay of the B200 Swendsen-Wang kernel.  Bonds: (i, j), i < j, over the
// neighbour lists in CSR column order, then (i, n) for every h_i != 0, indexed
// e = 0, 1, ... in that order; |J| and the sign from the FP64 couplings, |J|
// rounded to FP32.  Per sweep k (betas_f[k] FP32): bond e is kept when it is
// satisfied (J s_i s_j < 0, s_n = +1) and neglog(u_e) < (2*beta)*|J| (FP32
// products), u_e = Philox(ctr = (e >> 2, k, r, TAG_SW_BOND))[e & 3]; clusters
// of the kept bonds; a cluster's label is its smallest site; every cluster
// other than the one holding n flips when bit 0 of Philox(ctr = (c >> 2, k, r,
// TAG_SW_FLIP))[c & 3] is set (c the label).
void orc_replay_sw(int n, const int64_t* indptr, const int32_t* indices, const double* data, int R,
                   int8_t* spins, const float* betas_f, int64_t nsweeps, uint64_t seed, int threads) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  std::vector<int> bi, bj;
  std::vector<float> bw;
  std::vector<char> bpos;
  for (int i = 0; i < n; ++i)
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      const int j = indices[p];
      if (j == i || j == n || data[p] == 0.0 || j < i) continue;
      bi.push_back(i);
      bj.push_back(j);
      bw.push_back((float)std::fabs(data[p]));
      bpos.push_back(data[p] > 0);
    }
  for (int i = 0; i < n; ++i)
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p)
      if (indices[p] == n && data[p] != 0.0) {
        bi.push_back(i);
        bj.push_back(n);
        bw.push_back((float)std::fabs(data[p]));
        bpos.push_back(data[p] > 0);
      }
  const size_t ne = bi.size();
  parallel_for(R, threads, [&](int r) {
    int8_t* s = spins + (size_t)r * n;
    std::vector<int> comp(n + 1);
    std::function<int(int)> root = [&](int x) {
      while (comp[x] != x) x = comp[x];
      return x;
    };
    for (int64_t k = 0; k < nsweeps; ++k) {
      for (int i = 0; i <= n; ++i) comp[i] = i;
      const float beta2 = 2.0f * betas_f[k];
      for (size_t e = 0; e < ne; ++e) {
        const int si = s[bi[e]], sj = bj[e] < n ? s[bj[e]] : 1;
        const bool aligned = si * sj > 0;
        if (aligned == (bool)bpos[e]) continue;  // unsatisfied (or J s_i s_j > 0)
        const P4 q = philox((uint32_t)(e >> 2), (uint32_t)k, (uint32_t)r, TAG_SW_BOND, k0, k1);
        if (!(neglog(q.v[e & 3]) < beta2 * bw[e])) continue;
        int a = root(bi[e]), b = root(bj[e]);
        if (a == b) continue;
        if (a < b) std::swap(a, b);
        comp[a] = b;  // the larger label under the smaller: a cluster's label is its smallest site
      }
      const int rn = root(n);
      for (int i = 0; i < n; ++i) {
        const int c = root(i);
        if (c == rn) continue;
        const P4 q = philox((uint32_t)c >> 2, (uint32_t)k, (uint32_t)r, TAG_SW_FLIP, k0, k1);
        if (q.v[c & 3] & 1u) s[i] = (int8_t)-s[i];
      }
    }
  });
}

}  // extern "C"