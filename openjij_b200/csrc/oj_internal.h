// Internal host-side structures of libojb200: the context, the uploaded graph
// with its host analysis (colouring, bimodality, partition plans) and the
// kernel launchers.  Not part of the public C ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/openjij_b200.h"

namespace oj {

// Host-side fault injection for tests (oj_ctx_inject_fault): while it is >= 0,
// every device allocation counts it down, and the one that finds it at zero
// fails as if the device were out of memory (no allocation is attempted).
inline std::atomic<long long>& alloc_fail_countdown() {
  static std::atomic<long long> c{-1};
  return c;
}

// Grow-only device buffer owned by a context or graph.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (alloc_fail_countdown().load() >= 0 && alloc_fail_countdown().fetch_sub(1) == 0)
      return cudaErrorMemoryAllocation;  // the buffer keeps its old contents and size
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

// Partition of the sites of a regular +-c graph over the CTAs of one thread
// block cluster, used by the bit-packed SA kernel.  Each CTA (part p) keeps the
// words of its own sites and a halo copy of remote neighbours in shared memory.
// Local slots: [0, nloc) own sites sorted by (colour, boundary, site) where a
// boundary site has a neighbour in another part; [nloc, nloc+nhalo) halo sites
// sorted by (colour, site).
struct MscPlan {
  int P = 0;       // CTAs per cluster
  int D = 0;       // degree (regular graph)
  int ncol = 0;
  int slots = 0;   // max over parts of nloc + nhalo
  int nlocmax = 0;
  int hmax = 0;
  DevBuf tables;   // one allocation; the pointers below index into it
  // part-major arrays
  int32_t* gidx = nullptr;   // [P][slots] global site of each slot (-1 = pad)
  int32_t* coff = nullptr;   // [P][ncol+1] colour offsets of own sites
  int32_t* cb = nullptr;     // [P][ncol] first boundary slot of each colour (interior first)
  int32_t* hoff = nullptr;   // [P][ncol+1] colour offsets into the refresh list
  uint32_t* hsrc = nullptr;  // [P][hmax] (owner part << 16) | owner slot
  uint16_t* hdst = nullptr;  // [P][hmax] local halo slot
  uint16_t* nbr = nullptr;   // [P][nlocmax][D] local slots of the neighbours
  uint16_t* jm = nullptr;    // [P][nlocmax] bit l set when J(site, nbr l) > 0
  // push lists (bit-packed SA): own slot s of part p is copied, after each
  // update, to the halo slots pent[poff[p][s] .. poff[p][s+1]) of the parts
  // that read it, as (reader part << 16) | reader halo slot
  int pmax = 0;
  int32_t* poff = nullptr;   // [P][nlocmax+1]
  uint32_t* pent = nullptr;  // [P][pmax]
};

// Launch shape of a tunable kernel; 0 = the kernel's default choice.
struct Shape {
  int cluster = 0;  // CTAs per thread block cluster
  int threads = 0;  // threads per CTA
  int variant = 0;  // register-budget variant (batched kernel)
};

// Tiled couplings of the tensor-core dense kernel: J in BF16 (and the BF16
// remainder J - bf16(J) for non-exact couplings) as the MMA B tiles of every
// (32-spin block, CTA column range), FP32 32x32 in-block tiles and padded h.
struct TcPlan {
  int P = 0, ncta = 0, bpc = 0, nblk = 0;
  bool exact = true;
  DevBuf bt_hi, bt_lo, jblk, h, status;
};

}  // namespace oj

struct oj_graph {
  int device = 0;
  int n = 0;
  // symmetric augmented CSR exactly as received (FP64), for energies
  std::vector<int64_t> aug_indptr;
  std::vector<int32_t> aug_indices;
  std::vector<double> aug_data;
  // neighbour lists without diagonal, dummy column and zeros (CSR column order)
  std::vector<int32_t> rp, ci;
  std::vector<double> val64;
  std::vector<float> val;
  std::vector<double> h64;
  std::vector<float> h;
  std::vector<int32_t> colour, order, coff;  // greedy colouring; sites sorted by colour
  oj_graph_info info{};
  bool regular = false;
  // device copies
  oj::DevBuf d_rp, d_ci, d_val, d_h, d_val64, d_h64, d_order, d_coff;
  oj::DevBuf d_dense;  // FP32 dense J (n x n), created on first use
  std::unique_ptr<oj::MscPlan> msc;
  std::unique_ptr<oj::TcPlan> tc;
  oj::DevBuf sqa_nbr, sqa_jm;  // bit-packed SQA tables: [n][D] neighbours (u16), [n] J>0 masks
  std::map<uint64_t, oj::Shape> tuned;  // autotuned launch shapes by (kernel, replicas, slices)
  std::unique_ptr<oj_batch> single;     // this graph as a one-instance batch (dense jump kernel, energies)
  oj::DevBuf single_tab;                // its per-call tables: reads, order, replica and energy offsets
  int64_t sw_ne = -1;                   // Swendsen-Wang bond count (-1: list not built)
  oj::DevBuf sw_tables;                 // its bond list: i, j, |J|, sign
  ~oj_graph();
};

// A batch of dense instances for the batched SA kernel: FP32 J with rows
// padded to a multiple of 128 columns and FP32 h (the dynamics), and the FP64
// augmented matrices as received (the energies).
struct oj_batch {
  int device = 0;
  int count = 0;
  int max_n = 0;
  std::vector<int32_t> n;
  oj::DevBuf d_J, d_h, d_J64, d_joff, d_hoff, d_j64off, d_n;
  oj::DevBuf d_J16;   // J as FP16 when every coupling's FP32 value is exactly an FP16 value (flip rows)
  bool j16 = false;
  bool exact_fields = false;  // FP32 fields exact: energies from the fields (sweep kernel epilogue)
  // J * 2^p is int8 (exact fields and every scaled coupling in [-127, 127]):
  // the fields are then one int8 digit per coupling
  bool j8 = false;
  float j8_scale = 1.0f;  // 2^-p
  int tuned_variant = 0;  // autotuned register-budget variant, 0 = not tuned
  // the couplings as int8 digits on a per-instance grid 2^uexp, tiled for the
  // tensor-core field kernel (oj_k_field_tc.cu): ndig digits per coupling
  oj::DevBuf d_dig, d_dtoff, d_uexp;
  int ndig = 0;
  // batches of one-chunk instances (max_n <= 128) with four digits: the grid
  // integers q as int32, [n][128] at joff[m] (element [i][j] = q_ji), for the
  // recompute inside sa_batch1_kernel
  oj::DevBuf d_q32;
  ~oj_batch();
};

struct oj_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  std::string noalloc_error;  // why the allocation-free entry point could not be set up ("" = ready)
  oj::DevBuf spins, words, params, energies, best, aux, batch, fields, eparts;
  oj::DevBuf counters;  // device counters of a run: accepted flips (u64), field drift (float bits), status
  oj::DevBuf fitems;    // work items of the tensor-core field and hot-sweep kernels
  oj::DevBuf kstart;    // per replica: the sweep the sweep kernel continues at after the hot-sweep kernel
  int recompute = 16;   // full field recompute every this many sweeps (real couplings; 0 = never)
  long long wait_limit = -1;  // iterations of the field kernel's pipeline waits (< 0: the default)
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // the launch sequence of a batched / dense-jump run (field kernel, hot-sweep
  // kernel, the sweep launches between recomputes) is captured as a CUDA graph
  // on gstream, ordered after and before `stream` by gev, and replayed; the
  // executable graph is kept and updated in place by the next run's capture
  cudaStream_t gstream = nullptr;
  cudaEvent_t gev[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec = nullptr;
  // a slice-split SQA run from host buffers in two halves of replica groups,
  // the second on gstream, so that the copies of one half overlap the other's
  // kernel: pev[0] the preamble done on `stream`, pev[1] the second half's
  // kernel done, pev[2] the second half's copies done
  cudaEvent_t pev[3] = {nullptr, nullptr, nullptr};
};

namespace oj {

// Counter base of a run: Philox key and the global indices of the first sweep
// and the first replica, so that a run split over calls (first_sweep) or over
// GPUs (replica_offset) draws exactly the numbers of the unsplit run; and the
// device counter the annealing kernels add their accepted flips to (null: not
// counted).
struct RngBase {
  uint32_t k0, k1;
  uint32_t sweep0;
  uint32_t rep0;
  unsigned long long* flips = nullptr;
};

// ---- launchers (each returns cudaGetLastError() after the launch) ---------

cudaError_t launch_sa_colour(const oj_graph* g, int R, int8_t* spins, const float* betas,
                             int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches);
cudaError_t launch_sqa_colour(const oj_graph* g, int R, int T, int8_t* spins, const float2* coef,
                              int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches);
cudaError_t launch_sa_dense_plain(const oj_graph* g, int R, int8_t* spins, const float* betas,
                                  int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches);
cudaError_t launch_sa_msc(const oj_graph* g, int G, uint32_t* words, const uint32_t* thr,
                          const uint32_t* always, int64_t nsweeps, RngBase rb, cudaStream_t st,
                          int* launches, int threads = 0);
cudaError_t launch_sa_dense_tc(const oj_graph* g, int R, int8_t* spins, const float* betas, int64_t nsweeps,
                               RngBase rb, int recompute, cudaStream_t st, int* launches);
cudaError_t dense_tc_prepare(oj_graph* g, std::string* why);
cudaError_t launch_sqa_msc(const oj_graph* g, int R, int T, uint32_t* words, const uint32_t* thr,
                           const uint32_t* mode, int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches);
cudaError_t sqa_msc_prepare(oj_graph* g);
bool sqa_msc_fits(const oj_graph* g);
cudaError_t launch_sqa_pack(const int8_t* spins, int R, int T, int n, uint32_t* words, cudaStream_t st);
cudaError_t launch_sqa_unpack(const uint32_t* words, int R, int T, int n, int8_t* spins, cudaStream_t st);
int sqa_split_replicas_per_group(int T);
bool sqa_split_applies(const oj_graph* g, int T);
cudaError_t sqa_split_prepare(oj_graph* g, int G, int sm_count, std::string* why, int cluster = 0);
cudaError_t launch_sqa_split(const oj_graph* g, int G, int T, uint32_t* words, const uint32_t* thr,
                             const uint32_t* mode, int64_t nsweeps, RngBase rb, cudaStream_t st, int* launches,
                             int threads = 0);
cudaError_t launch_sqa_split_pack(const int8_t* spins, int R, int T, int n, int G, uint32_t* words,
                                  cudaStream_t st);
cudaError_t launch_sqa_split_unpack(const uint32_t* words, int R, int T, int n, int G, int8_t* spins,
                                    cudaStream_t st);
size_t sw_smem_bytes(int n);
int sw_max_sites();
cudaError_t sw_prepare(oj_graph* g);
cudaError_t launch_sw(const oj_graph* g, int R, int8_t* spins, const float* betas, int64_t nsweeps, RngBase rb,
                      uint32_t* scratch, int chunk, cudaStream_t st, int* launches);
int batch_max_sites();
int batch_warps();
int batch_variant_warps(int variant);
int batch_min_warps();  // fewest warps per CTA of any variant (most work items)
int batch_default_variant();
int batch_variant_max_n(int variant);  // largest instance a launch variant takes
// Tensor-core local fields of a batch (oj_k_field_tc.cu).
struct FieldCall {
  const int32_t* items = nullptr;  // device [nitems][3]: instance, site tile, replica tile
  int nitems = 0;
  int NT = 16;                     // replicas per tile
  unsigned int* drift = nullptr;   // max |F_new - F_old| (float bits) in compare mode
  int* status = nullptr;           // set when a bounded wait runs out
  long long wait_limit = 0;
  // the tensor-core kernel of the flip-heavy first sweeps (exact one-digit
  // batches, oj_k_hot_tc.cu): its work items and, per replica, the sweep the
  // sweep kernel continues at
  const int32_t* hot_items = nullptr;  // device [hot_nitems][2]: instance, replica tile
  int hot_nitems = 0;
  int32_t* kstart = nullptr;
  size_t nrep = 0;
};
bool hot_tc_applies(const oj_batch* b);
void hot_tc_items(const oj_batch* b, const int32_t* reads, const std::vector<int>& order,
                  std::vector<int32_t>& items);
cudaError_t launch_hot_tc(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff, int8_t* spins,
                          float* F, const int64_t* d_foff, const int64_t* d_eoff, const int32_t* d_items,
                          int nitems, const float* betas, int64_t nsweeps, RngBase rb, uint32_t inst0,
                          int32_t* kstop, int* d_status, long long wait_limit, cudaStream_t st);
// Fields on the tensor cores, then the sweeps (one segment, no recompute).
cudaError_t launch_sa_batch(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff,
                            const int32_t* d_items, int nitems, int* d_counter, int8_t* spins, const float* betas,
                            int64_t nsweeps, RngBase rb, uint32_t inst0, int sm_count, cudaStream_t st,
                            int* launches, int variant, float* d_fields, const int64_t* d_foff,
                            const FieldCall& fc, double* d_energies = nullptr, const int64_t* d_eoff = nullptr);
int field_tc_tile_replicas(const oj_batch* b, int max_reads);
void field_tc_items(const oj_batch* b, const int32_t* reads, const std::vector<int>& order, int NT,
                    std::vector<int32_t>& items);
cudaError_t launch_field_tc(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff, const int8_t* spins,
                            float* F, const int64_t* d_foff, const int32_t* d_items, int nitems, int NT, bool compare,
                            unsigned int* d_drift, int* d_status, long long wait_limit, cudaStream_t st);
cudaError_t field_tc_prepare(oj_batch* b, const std::vector<float>& J32, const std::vector<int64_t>& joff,
                             const std::vector<int8_t>* J8, int pmax);
// The batched sweep kernel alone (no fields): nsweeps sweeps from the fields in
// d_fields; with write_fields it stores its final fields back there.
cudaError_t launch_batch_sweeps(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff,
                                const int32_t* d_items, int nitems, int* d_counter, int8_t* spins,
                                const float* betas, int64_t nsweeps, RngBase rb, uint32_t inst0, int sm_count,
                                cudaStream_t st, int* launches, int variant, float* d_fields,
                                const int64_t* d_foff, double* d_energies, const int64_t* d_eoff,
                                bool write_fields, int* d_status, long long wait_limit,
                                const int32_t* kstart = nullptr, int recompute = 0, unsigned int* d_drift = nullptr);
cudaError_t launch_batch_energy(const oj_batch* b, const int32_t* d_reads, const int64_t* d_soff,
                                const int64_t* d_eoff, const int32_t* d_order, int max_reads, const int8_t* spins,
                                double* out, cudaStream_t st, int nsplit, double* parts, int64_t nrep);
int batch_energy_splits(const oj_batch* b, int max_reads, int sm_count);
cudaError_t launch_pack(const int8_t* spins, int R, int n, uint32_t* words, cudaStream_t st);
cudaError_t launch_unpack(const uint32_t* words, int R, int n, int8_t* spins, cudaStream_t st);
// Load the named kernels' code on the current device (CUDA loads modules
// lazily, which allocates device memory at a kernel's first use).
cudaError_t pack_preload();
cudaError_t msc_preload();
// Set-up of the allocation-free entry point on the current device: looks up
// its fixed scratch array's device address and loads the kernels it launches.
cudaError_t noalloc_prepare(int device);
// The device whose context page-locks the blocks of oj_host_alloc (the last
// one a context was created on); before any context, blocks are ordinary
// memory, so that allocating one never creates a context by itself.
void host_pin_device(int device);
int flip_stats_max_k();
cudaError_t launch_flip_stats(const oj_graph* g, int K, const int8_t* s, double thr, double* quad, double* lin,
                              unsigned long long* amin, cudaStream_t st);
cudaError_t launch_batch_flip_stats(const oj_batch* b, int K, const int8_t* s, const int64_t* soff, double thr,
                                    double* quad, double* lin, unsigned long long* amin, cudaStream_t st);
// FP64 energies of `count` spin vectors; the sites split over nsplit CTAs per
// 32 vectors (energy_splits), the partial sums in parts [nsplit][count] added
// in a fixed order (nsplit 1: no parts).
int energy_splits(const oj_graph* g, int count, int sm_count);
cudaError_t launch_energy(const oj_graph* g, int count, const int8_t* spins, double* out,
                          cudaStream_t st, int nsplit = 1, double* parts = nullptr);
cudaError_t launch_best_slice(const double* energies, int R, int T, int32_t* best, cudaStream_t st);

// Kernel limits used by the planner.
int sa_colour_max_smem_sites();
int msc_max_degree();
int msc_default_threads();
int split_default_threads();
cudaError_t msc_prepare(oj_graph* g, int P, std::string* why);
int msc_choose_cluster(const oj_graph* g, int G, int sm_count);

}  // namespace oj
