// Graph upload and host-side analysis: neighbour lists, greedy colouring,
// bimodality / integer-exactness checks and the device copies the kernels use.
//
// Input layout (both entry points): the symmetric augmented (n+1)x(n+1)
// matrix returned by the reference's get_interactions()
// (include/openjij/graph/dense.hpp:280-282, csr_sparse.hpp:183-185): J_ij in
// [0,n)x[0,n), h_i in row/column n, 1 at (n,n).  Validation follows
// Dense::set_interaction_matrix (dense.hpp:117-140): square, zero diagonal,
// corner 1; the matrix must be symmetric (what get_interactions() returns).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "oj_internal.h"

oj_batch::~oj_batch() {
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  d_J.release();
  d_J16.release();
  d_h.release();
  d_J64.release();
  d_joff.release();
  d_hoff.release();
  d_j64off.release();
  d_n.release();
  d_dig.release();
  d_dtoff.release();
  d_uexp.release();
  d_q32.release();
  if (cur >= 0 && cur != device) cudaSetDevice(cur);
}

oj_graph::~oj_graph() {
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  d_rp.release();
  d_ci.release();
  d_val.release();
  d_h.release();
  d_val64.release();
  d_h64.release();
  d_order.release();
  d_coff.release();
  d_dense.release();
  sqa_nbr.release();
  sqa_jm.release();
  single.reset();
  single_tab.release();
  sw_tables.release();
  if (msc) msc->tables.release();
  if (tc) {
    tc->bt_hi.release();
    tc->bt_lo.release();
    tc->jblk.release();
    tc->h.release();
    tc->status.release();
  }
  if (cur >= 0 && cur != device) cudaSetDevice(cur);
}

namespace oj {

std::vector<int32_t> greedy_colouring(int n, const std::vector<int32_t>& rp, const std::vector<int32_t>& ci,
                                      int* ncol_out) {
  std::vector<int32_t> col(n, -1);
  std::vector<int> stamp;
  int ncol = 0;
  for (int i = 0; i < n; ++i) {
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      const int j = ci[q];
      if (j < i) {
        const int c = col[j];
        if ((size_t)c >= stamp.size()) stamp.resize(c + 1, -1);
        stamp[c] = i;
      }
    }
    int c = 0;
    while ((size_t)c < stamp.size() && stamp[c] == i) ++c;
    col[i] = c;
    ncol = std::max(ncol, c + 1);
  }
  if (ncol_out) *ncol_out = ncol;
  return col;
}

// Two colours for a bipartite graph: the smallest site of every component gets
// colour 0 and the others alternate along a breadth-first search (on a graph
// the greedy colouring already 2-colours, this is that colouring); false when
// an odd cycle shows up.
bool two_colouring(int n, const std::vector<int32_t>& rp, const std::vector<int32_t>& ci,
                   std::vector<int32_t>& col) {
  col.assign(n, -1);
  std::vector<int32_t> queue;
  queue.reserve(n);
  for (int s = 0; s < n; ++s) {
    if (col[s] >= 0) continue;
    col[s] = 0;
    queue.assign(1, s);
    for (size_t h = 0; h < queue.size(); ++h) {
      const int u = queue[h];
      for (int q = rp[u]; q < rp[u + 1]; ++q) {
        const int v = ci[q];
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

// Evens out the classes of a proper colouring (the colour-class kernels run
// one class per phase with a barrier between phases, so the largest class
// sets the phase time).  target = ceil(n / ncol); a pass visits the sites in
// index order and moves a site whose class is above the target into the
// lowest colour whose class is below the target and holds none of its
// neighbours; passes repeat until one moves nothing (at most 8).  The
// colouring stays proper and keeps ncol classes.
void balance_colouring(int n, const std::vector<int32_t>& rp, const std::vector<int32_t>& ci, int ncol,
                       std::vector<int32_t>& col) {
  if (ncol < 2 || n == 0) return;
  const int target = (n + ncol - 1) / ncol;
  std::vector<int> size(ncol, 0), mark(ncol, -1);
  for (int i = 0; i < n; ++i) size[col[i]]++;
  for (int pass = 0; pass < 8; ++pass) {
    bool moved = false;
    for (int i = 0; i < n; ++i) {
      if (size[col[i]] <= target) continue;
      for (int q = rp[i]; q < rp[i + 1]; ++q) mark[col[ci[q]]] = i;
      for (int c = 0; c < ncol; ++c)
        if (size[c] < target && mark[c] != i) {
          size[col[i]]--;
          size[c]++;
          col[i] = c;
          moved = true;
          break;
        }
    }
    if (!moved) break;
  }
}

template <class T>
static cudaError_t upload(DevBuf& b, const std::vector<T>& v) {
  const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
  cudaError_t e = b.ensure(bytes);
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpy(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// Builds everything from the augmented CSR (rows sorted or not).
oj_status finish_graph(oj_ctx* ctx, oj_graph* g) {
  const int n = g->n;
  const auto& ip = g->aug_indptr;
  const auto& ix = g->aug_indices;
  const auto& dv = g->aug_data;
  // validation (dense.hpp:117-140)
  double corner = 0.0;
  for (int64_t q = ip[n]; q < ip[n + 1]; ++q)
    if (ix[q] == n) corner += dv[q];
  if (corner != 1.0) {
    ctx->last_error = "The right bottom element of interaction matrix must be unity.";
    return OJ_ERR_ARG;
  }
  g->rp.assign(n + 1, 0);
  g->h64.assign(n, 0.0);
  std::vector<std::pair<int, double>> row;
  for (int i = 0; i < n; ++i) {
    row.clear();
    for (int64_t q = ip[i]; q < ip[i + 1]; ++q) {
      const int j = ix[q];
      if (j < 0 || j > n) {
        ctx->last_error = "column index out of range";
        return OJ_ERR_ARG;
      }
      if (!std::isfinite(dv[q])) {
        ctx->last_error = "couplings and fields must be finite";
        return OJ_ERR_ARG;
      }
      if (j == n) {
        g->h64[i] += dv[q];
      } else if (j == i) {
        if (dv[q] != 0.0) {
          ctx->last_error = "The diagonal elements of interaction matrix must be zero.";
          return OJ_ERR_ARG;
        }
      } else if (dv[q] != 0.0) {
        row.emplace_back(j, dv[q]);
      }
    }
    if (!std::is_sorted(row.begin(), row.end())) std::sort(row.begin(), row.end());
    for (size_t a = 0; a < row.size(); ++a) {
      if (a + 1 < row.size() && row[a + 1].first == row[a].first) {
        row[a + 1].second += row[a].second;  // duplicate entries are summed (scipy semantics)
        continue;
      }
      g->ci.push_back(row[a].first);
      g->val64.push_back(row[a].second);
    }
    g->rp[i + 1] = (int32_t)g->ci.size();
  }
  // symmetry check: J_ij == J_ji.  The transpose, built by counting sort,
  // has its rows in ascending column order like the rows themselves, so the
  // matrix is symmetric exactly when both CSR arrays coincide.
  {
    const size_t nnz = g->ci.size();
    std::vector<int32_t> tp(n + 1, 0), tci(nnz);
    std::vector<double> tv(nnz);
    for (size_t q = 0; q < nnz; ++q) ++tp[g->ci[q] + 1];
    for (int i = 0; i < n; ++i) tp[i + 1] += tp[i];
    std::vector<int32_t> fill(tp.begin(), tp.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int q = g->rp[i]; q < g->rp[i + 1]; ++q) {
        const int32_t at = fill[g->ci[q]]++;
        tci[at] = i;
        tv[at] = g->val64[q];
      }
    if (tp != g->rp || tci != g->ci || tv != g->val64) {
      ctx->last_error = "interaction matrix must be symmetric (as returned by get_interactions())";
      return OJ_ERR_ARG;
    }
  }
  g->val.resize(g->val64.size());
  for (size_t q = 0; q < g->val64.size(); ++q) g->val[q] = (float)g->val64[q];
  g->h.resize(n);
  for (int i = 0; i < n; ++i) g->h[i] = (float)g->h64[i];
  // analysis
  oj_graph_info& inf = g->info;
  inf.n = n;
  inf.nnz = (int64_t)g->ci.size();
  int ncol = 0;
  if (two_colouring(n, g->rp, g->ci, g->colour)) {
    ncol = 0;
    for (int i = 0; i < n; ++i) ncol = std::max(ncol, g->colour[i] + 1);
  } else {
    g->colour = greedy_colouring(n, g->rp, g->ci, &ncol);
  }
  balance_colouring(n, g->rp, g->ci, ncol, g->colour);
  inf.num_colours = ncol;
  int dmax = 0, dmin = n > 0 ? 1 << 30 : 0;
  for (int i = 0; i < n; ++i) {
    const int d = g->rp[i + 1] - g->rp[i];
    dmax = std::max(dmax, d);
    dmin = std::min(dmin, d);
  }
  inf.max_degree = dmax;
  inf.min_degree = dmin;
  g->regular = n > 0 && dmax == dmin;
  bool bim = inf.nnz > 0;
  const double c = inf.nnz > 0 ? std::fabs(g->val64[0]) : 0.0;
  for (double v : g->val64) bim = bim && std::fabs(v) == c;
  for (double v : g->h64) bim = bim && v == 0.0;
  inf.bimodal = bim ? 1 : 0;
  inf.coupling_abs = bim ? c : 0.0;
  // J multiples of 1/2 with |J| <= 256 are exact in BF16; h multiples of 1/2
  // below 2^21 and every partial field sum stay exact in FP32.
  bool ie = true;
  auto half_int = [](double v, double lim) { return std::fabs(v) <= lim && std::floor(v * 2.0) == v * 2.0; };
  for (double v : g->val64) ie = ie && half_int(v, 256.0);
  for (double v : g->h64) ie = ie && half_int(v, 2097152.0);
  inf.integer_exact = ie ? 1 : 0;
  // sites grouped by colour
  g->coff.assign(ncol + 1, 0);
  for (int i = 0; i < n; ++i) g->coff[g->colour[i] + 1]++;
  for (int cc = 0; cc < ncol; ++cc) g->coff[cc + 1] += g->coff[cc];
  g->order.assign(n, 0);
  {
    std::vector<int32_t> fill(g->coff.begin(), g->coff.end() - 1);
    for (int i = 0; i < n; ++i) g->order[fill[g->colour[i]]++] = i;
  }
  // device copies
  cudaError_t e;
  if ((e = upload(g->d_rp, g->rp)) != cudaSuccess || (e = upload(g->d_ci, g->ci)) != cudaSuccess ||
      (e = upload(g->d_val, g->val)) != cudaSuccess || (e = upload(g->d_h, g->h)) != cudaSuccess ||
      (e = upload(g->d_val64, g->val64)) != cudaSuccess || (e = upload(g->d_h64, g->h64)) != cudaSuccess ||
      (e = upload(g->d_order, g->order)) != cudaSuccess || (e = upload(g->d_coff, g->coff)) != cudaSuccess) {
    ctx->last_error = std::string("graph upload: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? OJ_ERR_OOM : OJ_ERR_CUDA;
  }
  return OJ_OK;
}

cudaError_t ensure_dense(oj_graph* g) {
  if (g->d_dense.ptr) return cudaSuccess;
  const int n = g->n;
  std::vector<float> J((size_t)n * n, 0.0f);
  for (int i = 0; i < n; ++i)
    for (int q = g->rp[i]; q < g->rp[i + 1]; ++q) J[(size_t)i * n + g->ci[q]] = g->val[q];
  return upload(g->d_dense, J);
}

}  // namespace oj
