/*
 * openjij_b200 — C ABI of the B200 single-spin-flip annealing library.
 *
 * This is the drop-in boundary for OpenJij's SASampler / SQASampler hot path.
 * The reference has no C ABI: its path is the pybind11 module `cxxjij`
 * (openjij/main.cpp:27-227, openjij/declare.hpp) over header-only templates.
 * Each entry point below names the reference interface it replaces.  The
 * library's own pybind11 host (openjij_b200/csrc/cxxjij_host.cpp) keeps the
 * `cxxjij` Python surface and calls only these functions.
 *
 * Conventions
 *  - Every function returns oj_status (0 = OJ_OK) and never throws.
 *  - Spins are int8 in {-1, +1}.  SA layout [R][n], SQA layout [R][T][n].
 *  - Pointers are host pointers unless OJ_DEVICE_POINTERS is set in `flags`,
 *    in which case spins / energies are device pointers on the context's GPU.
 *  - Work is issued on the context's stream; with host pointers the call
 *    returns after the results are copied back.
 *  - One context per host thread (a context is not thread safe).
 */
#ifndef OPENJIJ_B200_H
#define OPENJIJ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t oj_status;
enum {
  OJ_OK = 0,
  OJ_ERR_ARG = 1,         /* invalid argument (reference: std::invalid_argument / runtime_error) */
  OJ_ERR_OOM = 2,         /* device or host allocation failed */
  OJ_ERR_CUDA = 3,        /* CUDA runtime error */
  OJ_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  OJ_ERR_BOUNDS = 5,      /* a device-side index check failed */
  OJ_ERR_UNSUPPORTED = 6, /* requested kernel cannot run this graph / size */
  OJ_ERR_NODEVICE = 7     /* no CUDA device / extension built without sm_100a */
};

/* flags */
#define OJ_DEVICE_POINTERS 0x1u
/* Autotune: on the first call for a (graph or batch, kernel, replicas, slices)
 * the tunable kernels (bit-packed SA, slice-split SQA, batched SA) time their
 * candidate launch shapes (cluster size, threads per CTA, register budget)
 * for a few sweeps on a copy of the call's own state and keep the fastest for
 * later calls.  Every shape gives the same spins; only the time differs.
 * Also enabled by the environment variable OJ_AUTOTUNE=1; OJ_AUTOTUNE=0 disables it
 * even when the flag is given (fixed launch shapes, e.g. for profiling). */
#define OJ_AUTOTUNE 0x2u
/* kernel selection (bits 4..7) */
#define OJ_KERNEL_SHIFT 4
#define OJ_KERNEL_MASK (0xFu << OJ_KERNEL_SHIFT)
#define OJ_KERNEL_AUTO (0u << OJ_KERNEL_SHIFT)
#define OJ_KERNEL_COLOUR (1u << OJ_KERNEL_SHIFT)     /* colour-class kernel, any sparse graph, FP32 */
#define OJ_KERNEL_DENSE_PLAIN (2u << OJ_KERNEL_SHIFT) /* sequential dense, one warp per replica, FP32 */
#define OJ_KERNEL_BITPACKED (3u << OJ_KERNEL_SHIFT)  /* 32 replicas per word, couplings +-c, h = 0 */
#define OJ_KERNEL_DENSE_TC (4u << OJ_KERNEL_SHIFT)   /* sequential dense, delayed tensor-core field updates */
#define OJ_KERNEL_SWENDSEN_WANG (6u << OJ_KERNEL_SHIFT) /* reported by oj_sw_run only */
#define OJ_KERNEL_DENSE_JUMP (5u << OJ_KERNEL_SHIFT) /* sequential dense, one warp per replica evaluating 128
                                                        sites at once and jumping between accepted flips
                                                        (the batched kernel on one instance), n <= 4096 */

typedef struct oj_ctx oj_ctx;
typedef struct oj_graph oj_graph;
typedef struct oj_batch oj_batch;

typedef struct oj_graph_info {
  int32_t n;              /* number of spins (dummy excluded) */
  int64_t nnz;            /* off-diagonal couplings (both triangles) */
  int32_t num_colours;    /* greedy colouring of the coupling graph */
  int32_t max_degree;
  int32_t min_degree;
  int32_t bimodal;        /* all |J_ij| equal, all h_i = 0 */
  int32_t integer_exact;  /* J_ij, h_i multiples of 1/2, |J| <= 256, |h| <= 2^21:
                            FP32 fields and BF16 couplings are exact */
  double coupling_abs;    /* |J| when bimodal */
} oj_graph_info;

typedef struct oj_run_stats {
  int32_t kernel;        /* OJ_KERNEL_* >> OJ_KERNEL_SHIFT actually used */
  int32_t launches;      /* kernels launched by the call */
  int64_t sweeps;        /* sweeps after expanding one_mc_step */
  double attempts;       /* spin-flip attempts = R * T * n * sweeps */
  float anneal_ms;       /* device time of the annealing kernel(s) */
  float total_ms;        /* device time of the whole call incl. copies */
  int32_t cluster;       /* CTAs per cluster of the annealing launch (tunable kernels, else 0) */
  int32_t threads;       /* threads per CTA of the annealing launch (tunable kernels, else 0) */
  int32_t variant;       /* register-budget variant (batched kernel, else 0) */
  int32_t tuned;         /* 1 when this call ran the autotuner */
  double accepted;       /* accepted single-spin flips over all replicas and sweeps (the bit-packed
                            kernels count every bit of their 32-replica words, padding replicas
                            included); -1 for Swendsen-Wang, whose cluster moves are not counted */
  double field_drift;    /* batched / dense-jump runs: the largest |f - f_exact| of the FP32
                            incremental fields over sites, replicas and the points where they are
                            recomputed (every oj_ctx_set_field_recompute sweeps) or checked (after
                            the last sweep), f_exact the tensor-core fields of the same spins
                            (within n 2^(E-27) of the FP64 field, E the exponent of max|J|);
                            0 when the couplings make the FP32 sums exact; -1 for other kernels */
} oj_run_stats;

const char* oj_version(void);
const char* oj_status_string(oj_status s);

/* Context: device, stream, reusable device workspace.  No reference
 * counterpart (the reference keeps state inside each system object). */
oj_status oj_ctx_create(int32_t device, oj_ctx** out);
oj_status oj_ctx_destroy(oj_ctx* ctx);
oj_status oj_ctx_set_stream(oj_ctx* ctx, void* cuda_stream);
oj_status oj_ctx_synchronize(oj_ctx* ctx);
const char* oj_ctx_last_error(const oj_ctx* ctx);

/* Full field recompute interval of the batched and dense-jump runs (the
 * reference's reset_dE, include/openjij/system/classical_ising.hpp:87-90, on
 * the tensor cores): for couplings whose FP32 field sums are not exact, the
 * fields are computed anew from the spins before every global sweep that is a
 * multiple of `sweeps` (default 16; 0 = only at the start of a call).  A run
 * split over calls at multiples of `sweeps` reproduces the unsplit run. */
oj_status oj_ctx_set_field_recompute(oj_ctx* ctx, int32_t sweeps);

/* Iterations after which the field kernel's pipeline waits give up (< 0: the
 * default, about a second).  A wait that gives up makes the kernel stop
 * issuing work, wait for its copies and MMAs in flight with the default limit,
 * free its tensor memory and return; the call reports OJ_ERR_TIMEOUT and the
 * context stays usable.  For tests of that path (0 gives up at once). */
oj_status oj_ctx_set_wait_limit(oj_ctx* ctx, int64_t iterations);

/* Host-side fault injection for tests of the error paths (no device fault is
 * made).  OJ_FAULT_ALLOC: the `after`-th device allocation from now (0 = the
 * next one) of any context of the process fails as if the device were out of
 * memory, so the call reports OJ_ERR_OOM; OJ_FAULT_NONE clears it. */
#define OJ_FAULT_NONE 0
#define OJ_FAULT_ALLOC 1
oj_status oj_ctx_inject_fault(oj_ctx* ctx, int32_t kind, int64_t after);

/* Page-locked host memory for spin buffers that stay on the host between
 * calls (the cxxjij systems keep theirs here): a run's copies in and out are
 * then single DMA transfers at the link's rate.  No counterpart in the
 * reference, whose systems hold their spins in ordinary Eigen members
 * (include/openjij/system/classical_ising.hpp:95 `spin`,
 * include/openjij/system/transverse_ising.hpp:198 `trotter_spins`).  Freed blocks are kept
 * in a process-wide cache (up to 2 GiB) for later requests of a similar size.
 * Blocks are page-locked through the device of the last context created in
 * the process and are usable from every context; before any oj_ctx_create
 * (so that no context is made on some default device), without a device,
 * when page-locked memory is refused, or with OJ_HOST_PINNED=0 in the
 * environment, a block is ordinary memory (every entry point takes either).  oj_host_alloc returns NULL only when no memory at all
 * can be had; free with oj_host_free only.  oj_host_is_pinned: 1 when p is a
 * page-locked block of this allocator. */
void* oj_host_alloc(size_t bytes);
void oj_host_free(void* p);
int32_t oj_host_is_pinned(const void* p);

/* Graph upload.  Replaces cxxjij.graph.Dense(num_spins).set_interaction_matrix
 * (openjij/declare.hpp:75-129; include/openjij/graph/dense.hpp:117-140) and
 * cxxjij.graph.CSRSparse(csr) (declare.hpp:195-217; csr_sparse.hpp:96-101).
 * Input is the symmetric augmented (n+1)x(n+1) matrix exactly as
 * get_interactions() returns it: J in [0,n)x[0,n), h in row/column n, 1 at
 * (n,n).  Diagonal J_ii must be zero (dense.hpp:127-131). */
oj_status oj_graph_create_dense(oj_ctx* ctx, int32_t n, const double* J_aug, oj_graph** out);
oj_status oj_graph_create_csr(oj_ctx* ctx, int32_t n, const int64_t* indptr,
                              const int32_t* indices, const double* data, oj_graph** out);
oj_status oj_graph_destroy(oj_graph* g);
oj_status oj_graph_query(const oj_graph* g, oj_graph_info* out);

/* Simulated annealing over R replicas.  Replaces the per-read loop
 * BaseSampler._cxxjij_sampling (openjij/sampler/sampler.py:116-140) around
 * Algorithm<SingleSpinFlip>::run(ClassicalIsing, rng, schedule)
 * (include/openjij/algorithm/algorithm.hpp:26-56,
 *  include/openjij/updater/single_spin_flip.hpp:66-95; binding
 *  openjij/declare.hpp:687-793).  The schedule is (betas[k], mcs[k]) for
 * k < num_sched, as ClassicalSchedule (schedule_list.hpp:121-127).
 * spins [R][n] in/out.  energies [R] (may be NULL): FP64 energy
 * sum_{i<j} J_ij s_i s_j + sum_i h_i s_i (dense.hpp:176-192).
 * Random numbers are a pure function of (seed, global sweep, global replica,
 * site): first_sweep is the global index of this call's first sweep and
 * replica_offset (a multiple of 32) the global index of replica 0, so a run
 * split over several calls or several GPUs reproduces the unsplit run. */
oj_status oj_sa_run(oj_ctx* ctx, const oj_graph* g, int32_t num_replicas, int8_t* spins,
                    const double* betas, const int32_t* mcs, int32_t num_sched, uint64_t seed,
                    int64_t first_sweep, int64_t replica_offset, uint32_t flags, double* energies,
                    oj_run_stats* stats);

/* Swendsen-Wang cluster annealing over R replicas.  Replaces
 * Algorithm<SwendsenWang>::run on a ClassicalIsing of a sparse graph
 * (include/openjij/updater/swendsen_wang.hpp:43-182, binding
 * openjij/main.cpp:144-154; SASampler's updater "swendsen wang",
 * openjij/sampler/sa_sampler.py:98-107).  Per sweep every satisfied bond
 * (h_i as a bond to a fixed dummy spin) is kept with probability
 * 1 - exp(-2 beta |J|) and every cluster not holding the dummy flips with
 * probability 1/2.  Arguments, schedule, counters and energies as oj_sa_run;
 * flags: OJ_DEVICE_POINTERS only.  One CTA per replica holds the union-find
 * forest in shared memory (n <= 45000) or, for larger graphs, in global
 * scratch of at most 1 GiB (replicas in chunks). */
oj_status oj_sw_run(oj_ctx* ctx, const oj_graph* g, int32_t num_replicas, int8_t* spins,
                    const double* betas, const int32_t* mcs, int32_t num_sched, uint64_t seed,
                    int64_t first_sweep, int64_t replica_offset, uint32_t flags, double* energies,
                    oj_run_stats* stats);

/* Discrete-time path-integral SQA over R replicas x T Trotter slices.
 * Replaces Algorithm<SingleSpinFlip>::run(TransverseIsing, rng, schedule)
 * (single_spin_flip.hpp:127-258; transverse_ising.hpp:54-224) with schedule
 * (betas[k], s[k], mcs[k]) as TransverseFieldSchedule (schedule_list.hpp:62-76).
 * T >= 2 (transverse_ising.hpp:78-81).  spins [R][T][n] in/out.
 * energies [R][T] (may be NULL): FP64 classical energy of each slice.
 * best_slice [R] (may be NULL): get_solution()'s slice, the first slice of
 * minimum energy (include/openjij/result/get_solution.hpp:59-84).
 * Kernels: OJ_KERNEL_COLOUR (any graph) or OJ_KERNEL_BITPACKED (regular
 * graph, couplings +-c, h = 0, degree <= 8): for even T <= 64 the even and
 * the odd slices of 32/(T/2) replicas (rounded down to a power of two) in two
 * 32-bit words per site; otherwise, for T <= 32, the T slices of one replica
 * in one word.  OJ_KERNEL_AUTO takes the bit-packed kernel when it applies. */
oj_status oj_sqa_run(oj_ctx* ctx, const oj_graph* g, int32_t num_replicas, int32_t num_slices,
                     int8_t* spins, double gamma, const double* betas, const double* s,
                     const int32_t* mcs, int32_t num_sched, uint64_t seed, int64_t first_sweep,
                     int64_t replica_offset, uint32_t flags, double* energies,
                     int32_t* best_slice, oj_run_stats* stats);

/* Allocation-free variant of oj_sa_run's bit-packed path, for callers that
 * cannot call cudaMalloc while they run (device memory already reserved by
 * another framework's allocator, or code that cannot accept cudaMalloc's
 * implicit device synchronisation).  No counterpart in the reference.
 * Runs the same kernel and random stream as oj_sa_run with OJ_KERNEL_BITPACKED,
 * so results are identical for the same arguments.  All per-call scratch lives
 * in one fixed 16 MiB device array inside the library (held by every GPU that
 * loads it until exit): words (ceil(R/32) * n * 4 B) plus thresholds
 * (sweeps * (degree+1) * 4 B) plus sweeps * 4 B must fit, else OJ_ERR_ARG.
 * spins: DEVICE pointer [R][n] on the context's device, in/out (a host
 * pointer or another device's memory -> OJ_ERR_ARG).  The graph must be
 * regular with couplings +-c, h = 0, and must have run oj_sa_run once (which
 * builds its site partition), else OJ_ERR_UNSUPPORTED.  The call is
 * asynchronous on the context's stream and cannot be captured into a CUDA
 * graph (a capturing stream -> OJ_ERR_UNSUPPORTED: the thresholds are copied
 * from a buffer that lives only during the call).  oj_ctx_create places the array on
 * the context's device and loads the kernels this entry point launches, so the
 * call itself allocates no device memory; calls overlapping on one GPU share
 * the array and race. */
oj_status oj_sa_run_bitpacked_noalloc(oj_ctx* ctx, const oj_graph* g, int32_t num_replicas, int8_t* spins,
                                      const double* betas, const int32_t* mcs, int32_t num_sched,
                                      uint64_t seed, int64_t first_sweep, int64_t replica_offset);

/* FP64 energies of R spin vectors [R][n].  Replaces Dense::energy /
 * CSRSparse::energy (dense.hpp:176-192, csr_sparse.hpp:139-155). */
oj_status oj_energy(oj_ctx* ctx, const oj_graph* g, int32_t num_replicas, const int8_t* spins,
                    uint32_t flags, double* energies);

/* Statistics behind SASampler's automatic beta range (sa_sampler.py:876-965,
 * which forms them with a dense matrix product and np.abs over the whole
 * augmented matrix).  For K (1..8) spin configurations spins[n][K] (+-1):
 *   dE_quad[n][K] = -2 s_i^c sum_{j<n} J_ij s_j^c   (coupling part of a flip)
 *   dE_lin[n][K]  = h_i s_i^c                       (field part)
 *   *abs_min      = smallest |entry| > threshold of the augmented matrix
 *                   (couplings, fields and the corner); +inf if there is none.
 * Host pointers; FP64; sums in the warp's order (exact for integer couplings). */
oj_status oj_graph_flip_stats(oj_ctx* ctx, const oj_graph* g, int32_t K, const int8_t* spins, double threshold,
                              double* dE_quad, double* dE_lin, double* abs_min);

/* A batch of dense instances of uneven size for oj_sa_run_batched.  Instance
 * k has n[k] spins (0 <= n[k] <= 4096) and its augmented (n[k]+1)^2 matrix,
 * row-major exactly as graph.Dense.get_interactions() returns it (J with zero
 * diagonal, h in row/column n[k], 1 in the corner; dense.hpp:117-140), at
 * J_aug + offset[k].  Invalid matrices -> OJ_ERR_ARG.  The reference has no
 * batch object: each instance is its own graph::Dense. */
oj_status oj_batch_create_dense(oj_ctx* ctx, int32_t count, const int32_t* n, const int64_t* offset,
                                const double* J_aug, oj_batch** out);
oj_status oj_batch_destroy(oj_batch* b);

/* oj_graph_flip_stats for every instance of a batch: spins, dE_quad and dE_lin
 * are the instances' [n[k]][K] blocks back to back, abs_min[count] (the
 * minimum over instance k's augmented matrix, corner included). */
oj_status oj_batch_flip_stats(oj_ctx* ctx, const oj_batch* b, int32_t K, const int8_t* spins, double threshold,
                              double* dE_quad, double* dE_lin, double* abs_min);

/* Simulated annealing of every instance of a batch in one persistent kernel
 * launch.  Replaces a loop of SASampler.sample calls over instances
 * (openjij/sampler/sa_sampler.py:137-329), each a per-read loop of
 * Algorithm<SingleSpinFlip>::run (algorithm.hpp:26-56,
 * single_spin_flip.hpp:66-95) on a graph::Dense.  reads[k] replicas of
 * instance k; spins concatenated instance by instance, [reads[k]][n[k]] each,
 * in/out; energies [sum reads] FP64 (may be NULL).  One schedule (betas[j],
 * mcs[j]) for all instances.  first_sweep as in oj_sa_run; instance_offset is
 * the global index of instance 0 (random numbers are a pure function of seed,
 * global instance, replica, sweep and site, so a batch split over calls or
 * GPUs reproduces the whole).  flags: OJ_DEVICE_POINTERS, OJ_AUTOTUNE. */
oj_status oj_sa_run_batched(oj_ctx* ctx, const oj_batch* b, const int32_t* reads, int8_t* spins,
                            const double* betas, const int32_t* mcs, int32_t num_sched, uint64_t seed,
                            int64_t first_sweep, int64_t instance_offset, uint32_t flags, double* energies,
                            oj_run_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* OPENJIJ_B200_H */
