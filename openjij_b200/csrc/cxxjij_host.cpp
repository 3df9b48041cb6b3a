// pybind11 host module `cxxjij` of openjij_b200: OpenJij's cxxjij Python
// surface (graph / system / algorithm / utility / result) for the
// single-spin-flip path, with every sweep executed on the GPU through the C
// ABI of include/openjij_b200.h.
//
// Reference bindings mirrored here (names, arguments, errors):
//   openjij/declare.hpp:43-129   Graph, Dense          openjij/main.cpp:43-47
//   openjij/declare.hpp:195-217  CSRSparse
//   openjij/declare.hpp:131-193  Sparse               openjij/main.cpp:44
//   openjij/declare.hpp:273-405  Dir, Square, ChimeraDir, Chimera (main.cpp:40-48)
//   openjij/declare.hpp:409-438  ClassicalIsing        openjij/main.cpp:68-73
//   openjij/declare.hpp:585-641  TransverseIsing       openjij/main.cpp:80-85
//   openjij/declare.hpp:687-793  Algorithm_SingleSpinFlip_run (4 overloads),
//                                Algorithm_SwendsenWang_run (openjij/main.cpp:144-154)
//   openjij/declare.hpp:795-879  updater parameters, schedules, make_*_schedule_list
//   openjij/declare.hpp:881-888  get_solution
// Extensions: a system may hold R replicas (2-D initial spins, or 3-D Trotter
// spins); the whole batch anneals in one GPU call.
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#include "openjij_b200.h"

namespace py = pybind11;
using namespace pybind11::literals;

namespace {

// ---------------------------------------------------------------------------
// device context
// ---------------------------------------------------------------------------

std::mutex g_ctx_mu;
oj_ctx* g_ctx = nullptr;
int g_device = -1;

int default_device() {
  const char* env = std::getenv("OPENJIJ_B200_DEVICE");
  return env ? std::atoi(env) : 0;
}

oj_ctx* ctx() {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (!g_ctx) {
    const int dev = g_device >= 0 ? g_device : default_device();
    oj_ctx* c = nullptr;
    const oj_status s = oj_ctx_create(dev, &c);
    if (s != OJ_OK)
      throw std::runtime_error(std::string("openjij_b200: cannot open CUDA device ") + std::to_string(dev) +
                               ": " + oj_status_string(s));
    g_ctx = c;
    g_device = dev;
  }
  return g_ctx;
}

void check(oj_status s, const char* what) {
  if (s == OJ_OK) return;
  std::string msg = std::string(what) + ": " + oj_status_string(s);
  if (g_ctx) {
    const char* d = oj_ctx_last_error(g_ctx);
    if (d && *d) msg += std::string(": ") + d;
  }
  if (s == OJ_ERR_ARG) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

struct RunInfo {
  std::string kernel;
  int launches = 0;
  long long sweeps = 0;
  double attempts = 0;
  double anneal_ms = 0, total_ms = 0;
  double accepted = 0;
  double field_drift = -1.0;  // largest over the calls of the run (-1: not measured)
};
RunInfo g_last_run;

void record(const oj_run_stats& st) {
  static const char* names[] = {"auto", "colour", "dense_plain", "bitpacked", "dense_tc", "dense_jump",
                                "swendsen_wang"};
  g_last_run.kernel = (st.kernel >= 0 && st.kernel < 7) ? names[st.kernel] : "?";
  g_last_run.launches += st.launches;
  g_last_run.sweeps += st.sweeps;
  g_last_run.attempts += st.attempts;
  g_last_run.anneal_ms += st.anneal_ms;
  g_last_run.total_ms += st.total_ms;
  g_last_run.accepted = (st.accepted < 0 || g_last_run.accepted < 0) ? -1.0 : g_last_run.accepted + st.accepted;
  g_last_run.field_drift = std::max(g_last_run.field_drift, st.field_drift);
}

// ---------------------------------------------------------------------------
// reference random engine for gen_spin (include/openjij/utility/random.hpp:39-87)
// ---------------------------------------------------------------------------

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

// ---------------------------------------------------------------------------
// graphs
// ---------------------------------------------------------------------------

struct Graph {
  explicit Graph(size_t n) : n_(n) {}
  virtual ~Graph() = default;
  template <class Eng>
  std::vector<int> gen_spin(Eng& eng) const {  // include/openjij/graph/graph.hpp:54-65
    std::vector<int> s(n_);
    std::uniform_int_distribution<> uid(0, 1);
    for (auto& e : s) e = 2 * uid(eng) - 1;
    return s;
  }
  template <class Eng>
  std::vector<int> gen_binary(Eng& eng) const {
    std::vector<int> s(n_);
    std::uniform_int_distribution<> uid(0, 1);
    for (auto& e : s) e = uid(eng);
    return s;
  }
  size_t size() const { return n_; }
  size_t n_;
};

// Symmetric augmented matrix in CSR form plus the device copy built from it.
struct AugCSR {
  size_t n = 0;
  std::vector<int64_t> indptr;
  std::vector<int32_t> indices;
  std::vector<double> data;
};

struct DeviceGraph {
  oj_graph* h = nullptr;
  ~DeviceGraph() {
    if (h) oj_graph_destroy(h);
  }
};

// Energy E(s) = sum_{i<j} J_ij s_i s_j + sum_i h_i s_i (dense.hpp:176-192).
double aug_energy(const AugCSR& a, const std::vector<int>& s) {
  if (s.size() != a.n) throw std::out_of_range("Out of range in energy in graph.");
  double e = 0.0;
  for (size_t i = 0; i < a.n; ++i) {
    double acc = 0.0;
    for (int64_t p = a.indptr[i]; p < a.indptr[i + 1]; ++p) {
      const size_t j = (size_t)a.indices[p];
      if (j < i) continue;
      if (j == a.n)
        acc += a.data[p];
      else if (j > i)
        acc += a.data[p] * s[j];
    }
    e += s[i] * acc;
  }
  return e;
}

struct Dense : Graph {
  explicit Dense(size_t n) : Graph(n), J_((n + 1) * (n + 1), 0.0) { at(n, n) = 1.0; }
  double& at(size_t i, size_t j) { return J_[i * (n_ + 1) + j]; }
  double at(size_t i, size_t j) const { return J_[i * (n_ + 1) + j]; }
  // J(i, j): coupling for i != j, h_i for i == j (dense.hpp:213-260)
  double get(size_t i, size_t j) const {
    if (i >= n_ || j >= n_) throw std::out_of_range("index out of range");
    return i != j ? at(std::min(i, j), std::max(i, j)) : at(i, n_);
  }
  void set(size_t i, size_t j, double v) {
    if (i >= n_ || j >= n_) throw std::out_of_range("index out of range");
    if (i != j) {
      at(i, j) = v;
      at(j, i) = v;
    } else {
      at(i, n_) = v;
      at(n_, i) = v;
    }
    dev_.reset();
  }
  void set_interaction_matrix(py::array_t<double, py::array::c_style | py::array::forcecast> m) {
    if (m.ndim() != 2 || m.shape(0) != m.shape(1)) throw std::runtime_error("interaction.rows() != interaction.cols()");
    if ((size_t)m.shape(0) != n_ + 1) throw std::runtime_error("invalid matrix size.");
    auto v = m.unchecked<2>();
    for (size_t i = 0; i < n_; ++i)
      if (v(i, i) != 0) throw std::runtime_error("The diagonal elements of interaction matrix must be zero.");
    if (v(n_, n_) != 1) throw std::runtime_error("The right bottom element of interaction matrix must be unity.");
    for (size_t i = 0; i <= n_; ++i)  // selfadjointView<Upper>: the upper triangle defines the matrix
      for (size_t j = i; j <= n_; ++j) {
        at(i, j) = v(i, j);
        at(j, i) = v(i, j);
      }
    dev_.reset();
  }
  py::array_t<double> get_interactions() const {
    py::array_t<double> out({n_ + 1, n_ + 1});
    std::copy(J_.begin(), J_.end(), out.mutable_data());
    return out;
  }
  AugCSR aug() const {
    AugCSR a;
    a.n = n_;
    a.indptr.push_back(0);
    for (size_t i = 0; i <= n_; ++i) {
      for (size_t j = 0; j <= n_; ++j) {
        const double v = at(i, j);
        if (v != 0.0 || i == j) {
          a.indices.push_back((int32_t)j);
          a.data.push_back(v);
        }
      }
      a.indptr.push_back((int64_t)a.indices.size());
    }
    return a;
  }
  double energy(const std::vector<int>& s) const { return aug_energy(aug(), s); }
  oj_graph* device() const {
    if (!dev_) {
      auto d = std::make_shared<DeviceGraph>();
      check(oj_graph_create_dense(ctx(), (int32_t)n_, J_.data(), &d->h), "oj_graph_create_dense");
      dev_ = d;
    }
    return dev_->h;
  }
  std::vector<double> J_;
  mutable std::shared_ptr<DeviceGraph> dev_;
};

struct CSRSparse : Graph {
  // The reference stores selfadjointView<Upper>() of the given matrix
  // (csr_sparse.hpp:96-101): only the upper triangle (with h in column n) is read.
  explicit CSRSparse(const py::object& mat) : Graph(0) {
    py::object csr = mat.attr("tocsr")();
    py::tuple shape = csr.attr("shape");
    const size_t rows = shape[0].cast<size_t>(), cols = shape[1].cast<size_t>();
    if (rows != cols) throw std::runtime_error("interaction.rows() != interaction.cols()");
    if (rows == 0) throw std::runtime_error("invalid matrix size.");
    n_ = rows - 1;
    auto ip = py::array_t<int64_t, py::array::forcecast>(csr.attr("indptr"));
    auto ix = py::array_t<int64_t, py::array::forcecast>(csr.attr("indices"));
    auto dv = py::array_t<double, py::array::forcecast>(csr.attr("data"));
    std::vector<std::vector<std::pair<int32_t, double>>> rowsv(rows);
    auto ipu = ip.unchecked<1>();
    auto ixu = ix.unchecked<1>();
    auto dvu = dv.unchecked<1>();
    for (size_t i = 0; i < rows; ++i)
      for (int64_t p = ipu(i); p < ipu(i + 1); ++p) {
        const size_t j = (size_t)ixu(p);
        const double v = dvu(p);
        if (j < i || v == 0.0) continue;
        rowsv[i].emplace_back((int32_t)j, v);
        if (j != i) rowsv[j].emplace_back((int32_t)i, v);
      }
    a_.n = n_;
    a_.indptr.push_back(0);
    for (size_t i = 0; i < rows; ++i) {
      auto& r = rowsv[i];
      std::sort(r.begin(), r.end());
      for (size_t q = 0; q < r.size(); ++q) {
        if (q + 1 < r.size() && r[q + 1].first == r[q].first) {
          r[q + 1].second += r[q].second;
          continue;
        }
        a_.indices.push_back(r[q].first);
        a_.data.push_back(r[q].second);
      }
      a_.indptr.push_back((int64_t)a_.indices.size());
    }
  }
  py::object get_interactions() const {
    py::module_ sp = py::module_::import("scipy.sparse");
    py::array_t<double> d(a_.data.size());
    py::array_t<int32_t> ix(a_.indices.size());
    py::array_t<int64_t> ip(a_.indptr.size());
    std::copy(a_.data.begin(), a_.data.end(), d.mutable_data());
    std::copy(a_.indices.begin(), a_.indices.end(), ix.mutable_data());
    std::copy(a_.indptr.begin(), a_.indptr.end(), ip.mutable_data());
    return sp.attr("csr_matrix")(py::make_tuple(d, ix, ip), "shape"_a = py::make_tuple(n_ + 1, n_ + 1));
  }
  double energy(const std::vector<int>& s) const { return aug_energy(a_, s); }
  oj_graph* device() const {
    if (!dev_) {
      auto d = std::make_shared<DeviceGraph>();
      check(oj_graph_create_csr(ctx(), (int32_t)n_, a_.indptr.data(), a_.indices.data(), a_.data.data(), &d->h),
            "oj_graph_create_csr");
      dev_ = d;
    }
    return dev_->h;
  }
  AugCSR a_;
  mutable std::shared_ptr<DeviceGraph> dev_;
};

// graph::Sparse (include/openjij/graph/sparse.hpp:32-250): couplings in a hash
// map keyed by (min(i,j), max(i,j)), the field of i under (i, i), and for every
// site the list of its neighbours (itself when it has a field).  A list holds
// at most num_edges sites; a site whose list is full gains no new neighbour
// (the coupling is stored but not seen by the dynamics), as in the reference's
// release build.  The dynamics read the augmented matrix built from the lists
// (utility/eigen.hpp:163-193): M[i][j] = J(i,j) for every listed neighbour
// j != i, M[i][n] = M[n][i] = h(i) when i lists itself, M[n][n] = 1.
struct Sparse : Graph {
  Sparse(size_t n, size_t num_edges) : Graph(n), num_edges_(std::min(n, num_edges)), adj_(n) {}
  explicit Sparse(size_t n) : Sparse(n, n) {}
  struct KeyHash {
    size_t operator()(const std::pair<size_t, size_t>& k) const {
      return std::hash<uint64_t>()(((uint64_t)k.first << 32) ^ (uint64_t)k.second);
    }
  };
  void check_index(size_t i) const {
    if (i >= n_) throw std::out_of_range("index " + std::to_string(i) + " out of range");
  }
  void link(size_t a, size_t b) {
    auto& l = adj_[a];
    if (std::find(l.begin(), l.end(), b) != l.end() || l.size() >= num_edges_) return;
    l.push_back(b);
    link(b, a);
  }
  double& J(size_t i, size_t j) {
    check_index(i);
    check_index(j);
    link(i, j);
    dev_.reset();
    return J_[{std::min(i, j), std::max(i, j)}];
  }
  double J(size_t i, size_t j) const {
    check_index(i);
    check_index(j);
    auto it = J_.find({std::min(i, j), std::max(i, j)});
    if (it == J_.end()) throw std::out_of_range("no interaction between " + std::to_string(i) + " and " + std::to_string(j));
    return it->second;
  }
  double& h(size_t i) { return J(i, i); }
  double h(size_t i) const { return J(i, i); }
  const std::vector<size_t>& adj_nodes(size_t i) const {
    check_index(i);
    return adj_[i];
  }
  size_t get_num_edges() const { return num_edges_; }
  AugCSR aug() const {
    std::vector<std::vector<std::pair<int32_t, double>>> rows(n_ + 1);
    for (size_t i = 0; i < n_; ++i)
      for (size_t j : adj_[i]) {
        if (j != i) {
          rows[i].emplace_back((int32_t)j, J(i, j));
        } else {
          rows[i].emplace_back((int32_t)n_, h(i));
          rows[n_].emplace_back((int32_t)i, h(i));
        }
      }
    rows[n_].emplace_back((int32_t)n_, 1.0);
    AugCSR a;
    a.n = n_;
    a.indptr.push_back(0);
    for (auto& r : rows) {
      std::sort(r.begin(), r.end());
      for (size_t q = 0; q < r.size(); ++q) {
        if (q + 1 < r.size() && r[q + 1].first == r[q].first) {  // setFromTriplets sums duplicates
          r[q + 1].second += r[q].second;
          continue;
        }
        a.indices.push_back(r[q].first);
        a.data.push_back(r[q].second);
      }
      a.indptr.push_back((int64_t)a.indices.size());
    }
    return a;
  }
  py::object get_interactions() const {
    const AugCSR a = aug();
    py::module_ sp = py::module_::import("scipy.sparse");
    py::array_t<double> d(a.data.size());
    py::array_t<int32_t> ix(a.indices.size());
    py::array_t<int64_t> ip(a.indptr.size());
    std::copy(a.data.begin(), a.data.end(), d.mutable_data());
    std::copy(a.indices.begin(), a.indices.end(), ix.mutable_data());
    std::copy(a.indptr.begin(), a.indptr.end(), ip.mutable_data());
    return sp.attr("csr_matrix")(py::make_tuple(d, ix, ip), "shape"_a = py::make_tuple(n_ + 1, n_ + 1));
  }
  double energy(const std::vector<int>& s) const { return aug_energy(aug(), s); }
  oj_graph* device() const {
    if (!dev_) {
      const AugCSR a = aug();
      auto d = std::make_shared<DeviceGraph>();
      check(oj_graph_create_csr(ctx(), (int32_t)n_, a.indptr.data(), a.indices.data(), a.data.data(), &d->h),
            "oj_graph_create_csr");
      dev_ = d;
    }
    return dev_->h;
  }
  size_t num_edges_;
  std::vector<std::vector<size_t>> adj_;
  std::unordered_map<std::pair<size_t, size_t>, double, KeyHash> J_;
  mutable std::shared_ptr<DeviceGraph> dev_;
};

// graph::Square (include/openjij/graph/square.hpp:33-387): a rows x cols grid,
// site (r, c) = cols * r + c; built with the open-boundary bonds and a field
// per site, all set to init_val; a bond given by direction wraps around the
// edges (row -1 is row rows-1 and so on).
enum class Dir { PLUS_R, MINUS_R, PLUS_C, MINUS_C };

struct Square : Sparse {
  Square(size_t rows, size_t cols, double init_val)
      : Sparse(checked(rows, cols) * cols, 4 + 1), rows_(rows), cols_(cols) {
    for (size_t r = 0; r < rows; ++r)
      for (size_t c = 0; c < cols; ++c) {
        const size_t i = to_ind((int64_t)r, (int64_t)c);
        if (r > 0) Sparse::J(i, to_ind((int64_t)r - 1, (int64_t)c)) = init_val;
        if (c > 0) Sparse::J(i, to_ind((int64_t)r, (int64_t)c - 1)) = init_val;
        if (r + 1 < rows) Sparse::J(i, to_ind((int64_t)r + 1, (int64_t)c)) = init_val;
        if (c + 1 < cols) Sparse::J(i, to_ind((int64_t)r, (int64_t)c + 1)) = init_val;
        Sparse::J(i, i) = init_val;
      }
  }
  static size_t checked(size_t rows, size_t cols) {
    if (rows < 1 || cols < 1) throw std::invalid_argument("num_row and num_column must be at least 1");
    return rows;
  }
  size_t to_ind(int64_t r, int64_t c) const {
    if (!(-1 <= r && r <= (int64_t)rows_)) throw std::runtime_error("invalid value r=" + std::to_string(r) + " inserted in Square");
    if (!(-1 <= c && c <= (int64_t)cols_)) throw std::runtime_error("invalid value c=" + std::to_string(c) + " inserted in Square");
    return cols_ * (size_t)((r + (int64_t)rows_) % (int64_t)rows_) + (size_t)((c + (int64_t)cols_) % (int64_t)cols_);
  }
  std::pair<size_t, size_t> to_rc(size_t ind) const {
    if (ind >= n_) throw std::runtime_error("invalid value index=" + std::to_string(ind) + " inserted in Square");
    return {ind / cols_, ind % cols_};
  }
  size_t neighbour(size_t r, size_t c, Dir d) const {
    if (r >= rows_ || c >= cols_) throw std::out_of_range("(r, c) out of range");
    const int64_t R = (int64_t)r, C = (int64_t)c;
    switch (d) {
      case Dir::MINUS_R: return to_ind(R - 1, C);
      case Dir::MINUS_C: return to_ind(R, C - 1);
      case Dir::PLUS_R: return to_ind(R + 1, C);
      default: return to_ind(R, C + 1);
    }
  }
  size_t rows_, cols_;
};

// graph::Chimera (include/openjij/graph/chimera.hpp:36-513): rows x cols unit
// cells of 8 sites, site (r, c, i) = 8 cols r + 8 c + i.  Sites 0-3 of a cell
// couple to 4-7 of the same cell (IN_*) and to the same i in the cells above
// and below (R directions); sites 4-7 to the same i left and right (C
// directions).  Built with every bond and field set to init_val, open edges;
// a bond given by direction wraps around.
enum class ChimeraDir { PLUS_R, MINUS_R, PLUS_C, MINUS_C, IN_0or4, IN_1or5, IN_2or6, IN_3or7 };

struct Chimera : Sparse {
  static constexpr size_t kCell = 8;
  Chimera(size_t rows, size_t cols, double init_val)
      : Sparse(Square::checked(rows, cols) * cols * kCell, 6 + 1), rows_(rows), cols_(cols) {
    for (size_t r = 0; r < rows; ++r)
      for (size_t c = 0; c < cols; ++c)
        for (size_t i = 0; i < kCell; ++i) {
          const int64_t R = (int64_t)r, C = (int64_t)c, I = (int64_t)i;
          const size_t x = to_ind(R, C, I);
          if (r > 0 && i < 4) Sparse::J(x, to_ind(R - 1, C, I)) = init_val;
          if (c > 0 && i >= 4) Sparse::J(x, to_ind(R, C - 1, I)) = init_val;
          if (r + 1 < rows && i < 4) Sparse::J(x, to_ind(R + 1, C, I)) = init_val;
          if (c + 1 < cols && i >= 4) Sparse::J(x, to_ind(R, C + 1, I)) = init_val;
          for (int64_t k = 0; k < 4; ++k) Sparse::J(x, to_ind(R, C, (i < 4 ? 4 : 0) + k)) = init_val;
          Sparse::J(x, x) = init_val;
        }
  }
  size_t to_ind(int64_t r, int64_t c, int64_t i) const {
    if (!(-1 <= r && r <= (int64_t)rows_)) throw std::runtime_error("invalid value r=" + std::to_string(r) + " inserted in Chimera");
    if (!(-1 <= c && c <= (int64_t)cols_)) throw std::runtime_error("invalid value c=" + std::to_string(c) + " inserted in Chimera");
    if (!(0 <= i && i < (int64_t)kCell)) throw std::runtime_error("invalid value i=" + std::to_string(i) + " inserted in Chimera");
    return cols_ * kCell * (size_t)((r + (int64_t)rows_) % (int64_t)rows_) +
           kCell * (size_t)((c + (int64_t)cols_) % (int64_t)cols_) + (size_t)i;
  }
  std::tuple<size_t, size_t, size_t> to_rci(size_t ind) const {
    if (ind >= n_) throw std::runtime_error("invalid value index=" + std::to_string(ind) + " inserted in Chimera");
    return std::make_tuple(ind / (cols_ * kCell), (ind % (cols_ * kCell)) / kCell, ind % kCell);
  }
  size_t neighbour(size_t r, size_t c, size_t i, ChimeraDir d) const {
    if (r >= rows_ || c >= cols_ || i >= kCell) throw std::out_of_range("(r, c, i) out of range");
    const int64_t R = (int64_t)r, C = (int64_t)c, I = (int64_t)i;
    const int64_t other = i < 4 ? 4 : 0;
    switch (d) {
      case ChimeraDir::MINUS_R:
      case ChimeraDir::PLUS_R:
        if (i >= 4) throw std::invalid_argument("R directions couple sites 0-3 of a cell");
        return to_ind(d == ChimeraDir::PLUS_R ? R + 1 : R - 1, C, I);
      case ChimeraDir::MINUS_C:
      case ChimeraDir::PLUS_C:
        if (i < 4) throw std::invalid_argument("C directions couple sites 4-7 of a cell");
        return to_ind(R, d == ChimeraDir::PLUS_C ? C + 1 : C - 1, I);
      case ChimeraDir::IN_0or4: return to_ind(R, C, other + 0);
      case ChimeraDir::IN_1or5: return to_ind(R, C, other + 1);
      case ChimeraDir::IN_2or6: return to_ind(R, C, other + 2);
      default: return to_ind(R, C, other + 3);
    }
  }
  size_t rows_, cols_;
};

// Single-flip energy changes of the configurations spins[n][K] and the smallest
// coupling magnitude above thr (oj_graph_flip_stats): what the automatic beta
// range of SASampler reads (sa_sampler.py:876-965).
template <class G>
py::tuple flip_stats(const G& g, py::array_t<int8_t, py::array::c_style | py::array::forcecast> s, double thr) {
  if (s.ndim() != 2 || (size_t)s.shape(0) != g.n_) throw std::invalid_argument("spins must have shape (n, K)");
  const size_t K = (size_t)s.shape(1);
  py::array_t<double> quad({g.n_, K}), lin({g.n_, K});
  double amin = 0.0;
  oj_graph* dg = g.device();
  oj_status rc;
  {
    py::gil_scoped_release release;
    rc = oj_graph_flip_stats(ctx(), dg, (int32_t)K, s.data(), thr, quad.mutable_data(), lin.mutable_data(), &amin);
  }
  check(rc, "flip_stats");
  return py::make_tuple(quad, lin, amin);
}

// ---------------------------------------------------------------------------
// schedules (include/openjij/utility/schedule_list.hpp)
// ---------------------------------------------------------------------------

struct ClassicalParam {
  double beta = 0;
};
struct TransverseParam {
  double beta = 0, s = 0;
};
struct ClassicalSchedule {
  ClassicalParam updater_parameter;
  size_t one_mc_step = 0;
};
struct TransverseSchedule {
  TransverseParam updater_parameter;
  size_t one_mc_step = 0;
};

// schedule_list.hpp:165-181
std::vector<ClassicalSchedule> make_classical_schedule_list(double beta_min, double beta_max, size_t one_mc_step,
                                                            size_t num_call_updater) {
  double r_beta = std::pow(beta_max / beta_min, 1.0 / static_cast<double>(num_call_updater - 1));
  double beta = beta_min;
  std::vector<ClassicalSchedule> out(num_call_updater);
  for (auto& s : out) {
    s.one_mc_step = one_mc_step;
    s.updater_parameter.beta = beta;
    beta *= r_beta;
  }
  return out;
}

// schedule_list.hpp:193-207
std::vector<TransverseSchedule> make_transverse_field_schedule_list(double beta, size_t one_mc_step,
                                                                    size_t num_call_updater) {
  double ds = 1.0 / static_cast<double>(num_call_updater - 1);
  double s = 0;
  std::vector<TransverseSchedule> out(num_call_updater);
  for (auto& e : out) {
    e.one_mc_step = one_mc_step;
    e.updater_parameter.beta = beta;
    e.updater_parameter.s = s;
    s += ds;
  }
  return out;
}

std::vector<ClassicalSchedule> classical_from_list(const py::list& lst) {
  std::vector<ClassicalSchedule> out;
  for (auto item : lst) {
    if (py::isinstance<ClassicalSchedule>(item)) {
      out.push_back(item.cast<ClassicalSchedule>());
      continue;
    }
    auto t = item.cast<py::sequence>();
    if (t.size() != 2) throw std::invalid_argument("schedule is list of (beta, one_mc_step)");
    ClassicalSchedule s;
    s.updater_parameter.beta = t[0].cast<double>();
    s.one_mc_step = t[1].cast<size_t>();
    out.push_back(s);
  }
  return out;
}

std::vector<TransverseSchedule> transverse_from_list(const py::list& lst) {
  std::vector<TransverseSchedule> out;
  for (auto item : lst) {
    if (py::isinstance<TransverseSchedule>(item)) {
      out.push_back(item.cast<TransverseSchedule>());
      continue;
    }
    auto t = item.cast<py::sequence>();
    if (t.size() != 2) throw std::invalid_argument("schedule is list of ((beta, s), one_mc_step)");
    auto bs = t[0].cast<py::sequence>();
    TransverseSchedule s;
    s.updater_parameter.beta = bs[0].cast<double>();
    s.updater_parameter.s = bs[1].cast<double>();
    s.one_mc_step = t[1].cast<size_t>();
    out.push_back(s);
  }
  return out;
}

// ---------------------------------------------------------------------------
// systems
// ---------------------------------------------------------------------------

template <class G>
std::shared_ptr<G> snapshot(const G& g) {
  return std::make_shared<G>(g);
}

// Page-locked storage for the systems' spins (oj_host_alloc, ordinary memory
// where page-locking is unavailable): a run's copies in and out are then
// single DMA transfers instead of the driver's staged copies of pageable memory.
template <class T>
struct HostPinned {
  using value_type = T;
  HostPinned() = default;
  template <class U>
  HostPinned(const HostPinned<U>&) {}
  T* allocate(size_t k) {
    void* p = oj_host_alloc(k * sizeof(T));
    if (!p) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t) { oj_host_free(p); }
  // new elements are left uninitialised (every user writes them all)
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
  template <class U>
  bool operator==(const HostPinned<U>&) const { return true; }
  template <class U>
  bool operator!=(const HostPinned<U>&) const { return false; }
};
using SpinBuf = std::vector<int8_t, HostPinned<int8_t>>;

// An int8 numpy array whose last axis is contiguous (what the sampler layer
// passes, broadcast views with zero strides included) is read in place;
// anything else goes through a conversion to double.
bool as_int8_array(const py::handle& obj, py::array* out) {
  if (!py::isinstance<py::array>(obj)) return false;
  py::array a = py::reinterpret_borrow<py::array>(obj);
  if (a.dtype().kind() != 'i' || a.itemsize() != 1 || a.ndim() < 1 || a.ndim() > 3) return false;
  if (a.shape(a.ndim() - 1) > 1 && a.strides(a.ndim() - 1) != 1) return false;
  *out = a;
  return true;
}

// Row r of an int8 array of 1-3 axes, rows numbered over all but the last axis.
const int8_t* int8_row(const py::array& a, size_t r) {
  const char* base = static_cast<const char*>(a.data());
  if (a.ndim() == 1) return reinterpret_cast<const int8_t*>(base);
  if (a.ndim() == 2) return reinterpret_cast<const int8_t*>(base + (ssize_t)r * a.strides(0));
  const size_t T = (size_t)a.shape(1);
  return reinterpret_cast<const int8_t*>(base + (ssize_t)(r / T) * a.strides(0) + (ssize_t)(r % T) * a.strides(1));
}

// Copies the first n spins of every row of a into out (resized to rows * n);
// throws, leaving out as it was, unless every copied value is -1 or +1 (v + 1
// is 0 or 2 exactly for those).
template <class Buf>
void copy_int8_rows(const py::array& a, size_t rows, size_t n, Buf& out) {
  unsigned bad = 0;
  for (size_t r = 0; r < rows; ++r) {
    const int8_t* src = int8_row(a, r);
    for (size_t i = 0; i < n; ++i) bad |= (uint8_t)(src[i] + 1) & 0xFDu;
  }
  if (bad) throw std::invalid_argument("spins must be -1 or +1");
  out.resize(rows * n);
  for (size_t r = 0; r < rows; ++r) {
    const int8_t* src = int8_row(a, r);
    std::copy(src, src + n, out.data() + r * n);
  }
}

// Parses 1-D (one replica) or 2-D ([R][n]) +-1 spins into out (resized).
template <class Buf>
void parse_spins(const py::handle& obj, size_t n, int* R_out, Buf& out) {
  py::array a8;
  const bool i8 = as_int8_array(obj, &a8);
  py::array_t<double> arr;
  if (!i8) {
    arr = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(obj);
    if (!arr) throw std::invalid_argument("spins must be array-like");
  }
  const py::array& shp = i8 ? a8 : static_cast<const py::array&>(arr);
  int R = 1;
  size_t len = 0;
  if (shp.ndim() == 1) {
    len = (size_t)shp.shape(0);
  } else if (shp.ndim() == 2) {
    R = (int)shp.shape(0);
    len = (size_t)shp.shape(1);
  } else {
    throw std::invalid_argument("spins must be 1-D or 2-D");
  }
  if (len != n && len != n + 1) throw std::invalid_argument("the size of the initial spins does not match the graph");
  if (i8) {
    copy_int8_rows(a8, (size_t)R, n, out);
  } else {
    Buf tmp((size_t)R * n);
    const double* p = arr.data();
    for (int r = 0; r < R; ++r)
      for (size_t i = 0; i < n; ++i) {
        const double v = p[(size_t)r * len + i];
        if (v != 1.0 && v != -1.0) throw std::invalid_argument("spins must be -1 or +1");
        tmp[(size_t)r * n + i] = (int8_t)v;
      }
    out.swap(tmp);
  }
  *R_out = R;
}

template <class G>
struct ClassicalIsing {
  ClassicalIsing(const py::object& init, const G& g) : graph(snapshot(g)), num_spins(g.size()) { reset(init); }
  void reset(const py::object& init) {
    int Rn = 1;
    parse_spins(init, num_spins, &Rn, spins);
    R = Rn;
    ecache_valid = false;
  }
  py::array_t<double> get_spin() const {
    std::vector<ssize_t> shape = R == 1 ? std::vector<ssize_t>{(ssize_t)num_spins + 1}
                                        : std::vector<ssize_t>{R, (ssize_t)num_spins + 1};
    py::array_t<double> out(shape);
    double* o = out.mutable_data();
    for (int r = 0; r < R; ++r) {
      for (size_t i = 0; i < num_spins; ++i) o[(size_t)r * (num_spins + 1) + i] = spins[(size_t)r * num_spins + i];
      o[(size_t)r * (num_spins + 1) + num_spins] = 1.0;
    }
    return out;
  }
  void set_spin(const py::object& v) { reset(v); }
  py::array_t<double> energies() const {
    py::array_t<double> out(R);
    if (num_spins == 0) {
      std::fill(out.mutable_data(), out.mutable_data() + R, 0.0);
      return out;
    }
    if (ecache_valid && ecache.size() == (size_t)R) {  // from the last run's own call
      std::copy(ecache.begin(), ecache.end(), out.mutable_data());
      return out;
    }
    oj_graph* dg = graph->device();
    const int8_t* sp = spins.data();
    double* e = out.mutable_data();
    check(oj_energy(ctx(), dg, R, sp, 0, e), "oj_energy");
    return out;
  }
  std::shared_ptr<G> graph;
  size_t num_spins;
  int R = 1;
  // energies of the current spins, written by the run call that produced them
  std::vector<double> ecache;
  bool ecache_valid = false;
  SpinBuf spins;
};

template <class G>
struct TransverseIsing {
  TransverseIsing(const py::object& trotter, const G& g, double gamma_) : graph(snapshot(g)), num_classical_spins(g.size()), gamma(gamma_) {
    reset_trotter(trotter);
  }
  TransverseIsing(const py::object& classical, const G& g, double gamma_, size_t T_)
      : graph(snapshot(g)), num_classical_spins(g.size()), gamma(gamma_) {
    if (!(T_ >= 2)) throw std::invalid_argument("trotter slices must be equal or larger than 2.");
    T = (int)T_;
    reset_classical(classical);
  }
  // [T][n] (one replica) or [R][T][n]
  void reset_trotter(const py::object& obj) {
    ecache_valid = false;
    py::array a8;
    const bool i8 = as_int8_array(obj, &a8);
    py::array_t<double> arr;
    if (!i8) {
      arr = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(obj);
      if (!arr) throw std::invalid_argument("trotter spins must be array-like");
    }
    const py::array& shp = i8 ? a8 : static_cast<const py::array&>(arr);
    const size_t n = num_classical_spins;
    int Rn = 1, Tn = 0;
    size_t len = 0;
    if (shp.ndim() == 2) {
      Tn = (int)shp.shape(0);
      len = (size_t)shp.shape(1);
    } else if (shp.ndim() == 3) {
      Rn = (int)shp.shape(0);
      Tn = (int)shp.shape(1);
      len = (size_t)shp.shape(2);
    } else {
      throw std::invalid_argument("trotter spins must be [T][n] or [R][T][n]");
    }
    if (!(Tn >= 2)) throw std::invalid_argument("trotter slices must be equal or larger than 2.");
    if (len != n && len != n + 1) throw std::invalid_argument("the size of the trotter spins does not match the graph");
    if (i8) {
      copy_int8_rows(a8, (size_t)Rn * Tn, n, spins);
    } else {
      SpinBuf tmp((size_t)Rn * Tn * n);
      const double* p = arr.data();
      for (size_t idx = 0; idx < (size_t)Rn * Tn; ++idx)
        for (size_t i = 0; i < n; ++i) {
          const double v = p[idx * len + i];
          if (v != 1.0 && v != -1.0) throw std::invalid_argument("spins must be -1 or +1");
          tmp[idx * n + i] = (int8_t)v;
        }
      spins.swap(tmp);
    }
    R = Rn;
    T = Tn;
  }
  void reset_classical(const py::object& obj) {
    ecache_valid = false;
    const size_t n = num_classical_spins;
    int Rn = 1;
    std::vector<int8_t> cl;
    parse_spins(obj, n, &Rn, cl);
    R = Rn;
    spins.assign((size_t)R * T * n, 1);
    for (int r = 0; r < R; ++r)
      for (int t = 0; t < T; ++t)
        std::copy(cl.begin() + (size_t)r * n, cl.begin() + (size_t)(r + 1) * n, spins.begin() + ((size_t)r * T + t) * n);
  }
  // 1-D: classical spins copied into every slice; 2-D: [T][n]; 3-D: [R][T][n]
  void reset(const py::object& obj) {
    auto arr = py::array::ensure(obj);
    if (!arr || arr.ndim() == 1)
      reset_classical(obj);
    else
      reset_trotter(obj);
  }
  // (n+1) x T (one replica, reference layout) or R x (n+1) x T
  py::array_t<double> get_trotter() const {
    const size_t n = num_classical_spins;
    std::vector<ssize_t> shape = R == 1 ? std::vector<ssize_t>{(ssize_t)n + 1, T}
                                        : std::vector<ssize_t>{R, (ssize_t)n + 1, T};
    py::array_t<double> out(shape);
    double* o = out.mutable_data();
    for (int r = 0; r < R; ++r)
      for (size_t i = 0; i <= n; ++i)
        for (int t = 0; t < T; ++t)
          o[((size_t)r * (n + 1) + i) * T + t] = i < n ? spins[((size_t)r * T + t) * n + i] : 1.0;
    return out;
  }
  void set_trotter(const py::object& v) {
    // accepts the reference layout (n+1) x T / R x (n+1) x T
    auto arr = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(v);
    if (!arr || (arr.ndim() != 2 && arr.ndim() != 3)) throw std::invalid_argument("trotter_spins must be 2-D or 3-D");
    py::object t = arr.ndim() == 2 ? arr.attr("T") : arr.attr("transpose")(0, 2, 1);
    reset_trotter(t);
  }
  py::array_t<double> energies() const {
    const size_t n = num_classical_spins;
    py::array_t<double> out(std::vector<ssize_t>{R, T});
    if (n == 0) {
      std::fill(out.mutable_data(), out.mutable_data() + (size_t)R * T, 0.0);
      return out;
    }
    if (ecache_valid && ecache.size() == (size_t)R * T) {  // from the last run's own call
      std::copy(ecache.begin(), ecache.end(), out.mutable_data());
      return out;
    }
    check(oj_energy(ctx(), graph->device(), R * T, spins.data(), 0, out.mutable_data()), "oj_energy");
    return out;
  }
  std::shared_ptr<G> graph;
  size_t num_classical_spins;
  double gamma;
  int R = 1, T = 0;
  // slice energies of the current spins, written by the run call that produced them
  std::vector<double> ecache;
  bool ecache_valid = false;
  SpinBuf spins;  // [R][T][n]
};

uint64_t random_seed() {
  std::random_device rd;
  return ((uint64_t)rd() << 32) ^ (uint64_t)rd();
}

uint32_t kernel_flag(const std::string& k) {
  if (k == "auto" || k.empty()) return OJ_KERNEL_AUTO;
  if (k == "colour" || k == "color") return OJ_KERNEL_COLOUR;
  if (k == "dense_plain") return OJ_KERNEL_DENSE_PLAIN;
  if (k == "bitpacked") return OJ_KERNEL_BITPACKED;
  if (k == "dense_tc") return OJ_KERNEL_DENSE_TC;
  if (k == "dense_jump") return OJ_KERNEL_DENSE_JUMP;
  throw std::invalid_argument("unknown kernel " + k);
}

std::string g_kernel = "auto";

// Algorithm<SingleSpinFlip>::run (algorithm.hpp:26-56) for R classical replicas.
template <class G>
void run_classical(ClassicalIsing<G>& sys, uint64_t seed, const std::vector<ClassicalSchedule>& sched,
                   const std::function<void(const ClassicalIsing<G>&, double)>& cb) {
  g_last_run = RunInfo();
  sys.ecache_valid = false;
  if (sys.num_spins == 0 || sched.empty()) {
    if (cb)
      for (auto& s : sched)
        for (size_t m = 0; m < s.one_mc_step; ++m) cb(sys, s.updater_parameter.beta);
    return;
  }
  oj_graph* dg = sys.graph->device();
  const uint32_t flags = kernel_flag(g_kernel);
  if (!cb) {
    std::vector<double> betas;
    std::vector<int32_t> mcs;
    for (auto& s : sched) {
      if (s.updater_parameter.beta < 0) throw std::invalid_argument("beta must be >= 0");
      betas.push_back(s.updater_parameter.beta);
      mcs.push_back((int32_t)s.one_mc_step);
    }
    oj_run_stats st;
    oj_status rc;
    {
      py::gil_scoped_release release;
      sys.ecache.resize((size_t)sys.R);
      rc = oj_sa_run(ctx(), dg, sys.R, sys.spins.data(), betas.data(), mcs.data(), (int32_t)betas.size(), seed, 0, 0,
                     flags, sys.ecache.data(), &st);
    }
    check(rc, "Algorithm_SingleSpinFlip_run");
    sys.ecache_valid = true;
    record(st);
    return;
  }
  // with a callback: one GPU call per updater call, the global sweep index
  // carried in first_sweep so the random stream equals the one-call run
  int64_t sweep = 0;
  for (auto& s : sched) {
    for (size_t m = 0; m < s.one_mc_step; ++m) {
      const double b = s.updater_parameter.beta;
      const int32_t one = 1;
      oj_run_stats st;
      oj_status rc;
      {
        py::gil_scoped_release release;
        rc = oj_sa_run(ctx(), dg, sys.R, sys.spins.data(), &b, &one, 1, seed, sweep, 0, flags, nullptr, &st);
      }
      check(rc, "Algorithm_SingleSpinFlip_run");
      record(st);
      ++sweep;
      cb(sys, b);
    }
  }
}

// Algorithm<SwendsenWang>::run (algorithm.hpp:26-56 with
// updater/swendsen_wang.hpp:43-182) for R classical replicas on a sparse graph.
template <class G>
void run_swendsen_wang(ClassicalIsing<G>& sys, uint64_t seed, const std::vector<ClassicalSchedule>& sched,
                       const std::function<void(const ClassicalIsing<G>&, double)>& cb) {
  g_last_run = RunInfo();
  sys.ecache_valid = false;
  if (sys.num_spins == 0 || sched.empty()) {
    if (cb)
      for (auto& s : sched)
        for (size_t m = 0; m < s.one_mc_step; ++m) cb(sys, s.updater_parameter.beta);
    return;
  }
  oj_graph* dg = sys.graph->device();
  if (!cb) {
    std::vector<double> betas;
    std::vector<int32_t> mcs;
    for (auto& s : sched) {
      if (s.updater_parameter.beta < 0) throw std::invalid_argument("beta must be >= 0");
      betas.push_back(s.updater_parameter.beta);
      mcs.push_back((int32_t)s.one_mc_step);
    }
    oj_run_stats st;
    oj_status rc;
    {
      py::gil_scoped_release release;
      sys.ecache.resize((size_t)sys.R);
      rc = oj_sw_run(ctx(), dg, sys.R, sys.spins.data(), betas.data(), mcs.data(), (int32_t)betas.size(), seed, 0, 0,
                     0, sys.ecache.data(), &st);
    }
    check(rc, "Algorithm_SwendsenWang_run");
    sys.ecache_valid = true;
    record(st);
    return;
  }
  int64_t sweep = 0;
  for (auto& s : sched) {
    for (size_t m = 0; m < s.one_mc_step; ++m) {
      const double b = s.updater_parameter.beta;
      const int32_t one = 1;
      oj_run_stats st;
      oj_status rc;
      {
        py::gil_scoped_release release;
        rc = oj_sw_run(ctx(), dg, sys.R, sys.spins.data(), &b, &one, 1, seed, sweep, 0, 0, nullptr, &st);
      }
      check(rc, "Algorithm_SwendsenWang_run");
      record(st);
      ++sweep;
      cb(sys, b);
    }
  }
}

template <class G>
void run_transverse(TransverseIsing<G>& sys, uint64_t seed, const std::vector<TransverseSchedule>& sched,
                    const std::function<void(const TransverseIsing<G>&, std::pair<double, double>)>& cb) {
  g_last_run = RunInfo();
  sys.ecache_valid = false;
  if (sys.num_classical_spins == 0 || sched.empty()) {
    if (cb)
      for (auto& s : sched)
        for (size_t m = 0; m < s.one_mc_step; ++m) cb(sys, {s.updater_parameter.beta, s.updater_parameter.s});
    return;
  }
  oj_graph* dg = sys.graph->device();
  if (!cb) {
    std::vector<double> betas, ss;
    std::vector<int32_t> mcs;
    for (auto& s : sched) {
      betas.push_back(s.updater_parameter.beta);
      ss.push_back(s.updater_parameter.s);
      mcs.push_back((int32_t)s.one_mc_step);
    }
    oj_run_stats st;
    oj_status rc;
    {
      py::gil_scoped_release release;
      sys.ecache.resize((size_t)sys.R * sys.T);
      rc = oj_sqa_run(ctx(), dg, sys.R, sys.T, sys.spins.data(), sys.gamma, betas.data(), ss.data(), mcs.data(),
                      (int32_t)betas.size(), seed, 0, 0, 0, sys.ecache.data(), nullptr, &st);
    }
    check(rc, "Algorithm_SingleSpinFlip_run");
    sys.ecache_valid = true;
    record(st);
    return;
  }
  int64_t sweep = 0;
  for (auto& s : sched) {
    for (size_t m = 0; m < s.one_mc_step; ++m) {
      const double b = s.updater_parameter.beta, sv = s.updater_parameter.s;
      const int32_t one = 1;
      oj_run_stats st;
      oj_status rc;
      {
        py::gil_scoped_release release;
        rc = oj_sqa_run(ctx(), dg, sys.R, sys.T, sys.spins.data(), sys.gamma, &b, &sv, &one, 1, seed, sweep, 0, 0,
                        nullptr, nullptr, &st);
      }
      check(rc, "Algorithm_SingleSpinFlip_run");
      record(st);
      ++sweep;
      cb(sys, {b, sv});
    }
  }
}

// get_solution (get_solution.hpp:39-49): spins times the dummy spin (always +1)
template <class G>
py::object solution(const ClassicalIsing<G>& sys) {
  const size_t n = sys.num_spins;
  if (sys.R == 1) return py::cast(std::vector<int>(sys.spins.begin(), sys.spins.end()));
  py::list out;
  for (int r = 0; r < sys.R; ++r)
    out.append(std::vector<int>(sys.spins.begin() + (size_t)r * n, sys.spins.begin() + (size_t)(r + 1) * n));
  return out;
}

// get_solution (get_solution.hpp:59-84): the first slice of minimum energy
template <class G>
py::object solution(const TransverseIsing<G>& sys) {
  const size_t n = sys.num_classical_spins;
  std::vector<double> e((size_t)sys.R * sys.T, 0.0);
  if (sys.ecache_valid && sys.ecache.size() == e.size())
    e = sys.ecache;
  else if (n > 0)
    check(oj_energy(ctx(), sys.graph->device(), sys.R * sys.T, sys.spins.data(), 0, e.data()), "oj_energy");
  py::list out;
  for (int r = 0; r < sys.R; ++r) {
    int best = 0;
    double m = DBL_MAX;
    for (int t = 0; t < sys.T; ++t)
      if (e[(size_t)r * sys.T + t] < m) {
        m = e[(size_t)r * sys.T + t];
        best = t;
      }
    const auto b = sys.spins.begin() + ((size_t)r * sys.T + best) * n;
    std::vector<int> v(b, b + n);
    if (sys.R == 1) return py::cast(v);
    out.append(v);
  }
  return out;
}

// The replicas' spins as an int8 array of the given shape (a copy), for the
// sampler layer: no per-spin Python objects.
template <class V>
py::array_t<int8_t> int8_view(const V& v, std::vector<ssize_t> shape) {
  py::array_t<int8_t> out(shape);
  std::copy(v.begin(), v.end(), out.mutable_data());
  return out;
}

template <class G>
void bind_graph_systems(py::module_& msys, py::module_& malg, py::module_& mres, const std::string& suffix) {
  using CI = ClassicalIsing<G>;
  using TI = TransverseIsing<G>;
  py::class_<CI>(msys, ("ClassicalIsing" + suffix).c_str(), py::module_local())
      .def(py::init<const py::object&, const G&>(), "init_spin"_a, "init_interaction"_a)
      .def("reset_spins", &CI::reset, "init_spin"_a)
      .def_property("spin", &CI::get_spin, &CI::set_spin)
      .def_property_readonly("interaction", [](const CI& s) { return s.graph->get_interactions(); })
      .def_readonly("num_spins", &CI::num_spins)
      .def_readonly("num_replicas", &CI::R)
      .def("energies", &CI::energies)
      .def("_spins_int8", [](const CI& s) { return int8_view(s.spins, {s.R, (ssize_t)s.num_spins}); });
  msys.def(
      "make_classical_ising", [](const py::object& init, const G& g) { return CI(init, g); }, "init_spin"_a,
      "init_interaction"_a);

  py::class_<TI>(msys, ("TransverseIsing" + suffix).c_str(), py::module_local())
      .def(py::init<const py::object&, const G&, double>(), "init_spin"_a, "init_interaction"_a, "gamma"_a)
      .def(py::init<const py::object&, const G&, double, size_t>(), "init_classical_spins"_a, "init_interaction"_a,
           "gamma"_a, "num_trotter_slices"_a)
      .def("reset_spins", &TI::reset, "init_trotter_spins"_a)
      .def_property("trotter_spins", &TI::get_trotter, &TI::set_trotter)
      .def_property_readonly("interaction", [](const TI& s) { return s.graph->get_interactions(); })
      .def_readonly("num_classical_spins", &TI::num_classical_spins)
      .def_readonly("num_replicas", &TI::R)
      .def_readonly("num_trotter_slices", &TI::T)
      .def_readwrite("gamma", &TI::gamma)
      .def("energies", &TI::energies)
      .def("_spins_int8", [](const TI& s) {
        return int8_view(s.spins, {s.R, s.T, (ssize_t)s.num_classical_spins});
      });
  msys.def(
      "make_transverse_ising", [](const py::object& tr, const G& g, double gamma) { return TI(tr, g, gamma); },
      "init_trotter_spins"_a, "init_interaction"_a, "gamma"_a);
  msys.def(
      "make_transverse_ising",
      [](const py::object& cl, const G& g, double gamma, size_t T) { return TI(cl, g, gamma, T); },
      "classical_spins"_a, "init_interaction"_a, "gamma"_a, "num_trotter_slices"_a);

  using CCb = std::function<void(const CI&, double)>;
  using TCb = std::function<void(const TI&, std::pair<double, double>)>;
  const char* name = "Algorithm_SingleSpinFlip_run";
  // classical: with seed / without seed; ScheduleList or list of tuples
  malg.def(
      name, [](CI& s, uint64_t seed, const py::list& sched, const CCb& cb) { run_classical(s, seed, classical_from_list(sched), cb); },
      "system"_a, "seed"_a, "schedule_list"_a, "callback"_a = nullptr);
  malg.def(
      name, [](CI& s, const py::list& sched, const CCb& cb) { run_classical(s, random_seed(), classical_from_list(sched), cb); },
      "system"_a, "schedule_list"_a, "callback"_a = nullptr);
  malg.def(
      name, [](TI& s, uint64_t seed, const py::list& sched, const TCb& cb) { run_transverse(s, seed, transverse_from_list(sched), cb); },
      "system"_a, "seed"_a, "schedule_list"_a, "callback"_a = nullptr);
  malg.def(
      name, [](TI& s, const py::list& sched, const TCb& cb) { run_transverse(s, random_seed(), transverse_from_list(sched), cb); },
      "system"_a, "schedule_list"_a, "callback"_a = nullptr);
  mres.def("get_solution", [](const CI& s) { return solution(s); }, "system"_a);
  mres.def("get_solution", [](const TI& s) { return solution(s); }, "system"_a);
  // Swendsen-Wang: sparse systems only, as the reference (openjij/main.cpp:144-154)
  if (std::is_same<G, CSRSparse>::value || std::is_same<G, Sparse>::value) {
    const char* sw = "Algorithm_SwendsenWang_run";
    malg.def(
        sw, [](CI& s, uint64_t seed, const py::list& sched, const CCb& cb) { run_swendsen_wang(s, seed, classical_from_list(sched), cb); },
        "system"_a, "seed"_a, "schedule_list"_a, "callback"_a = nullptr);
    malg.def(
        sw, [](CI& s, const py::list& sched, const CCb& cb) { run_swendsen_wang(s, random_seed(), classical_from_list(sched), cb); },
        "system"_a, "schedule_list"_a, "callback"_a = nullptr);
  }
}

}  // namespace

PYBIND11_MODULE(_cxxjij, m) {
  m.doc() = "openjij_b200 cxxjij: OpenJij's cxxjij API with the sweeps on the GPU";
  py::module_ mg = m.def_submodule("graph", "graph submodule");
  py::module_ ms = m.def_submodule("system", "system submodule");
  py::module_ ma = m.def_submodule("algorithm", "algorithm submodule");
  py::module_ mu = m.def_submodule("utility", "utility submodule");
  py::module_ mr = m.def_submodule("result", "result submodule");

  // ---- graph
  py::class_<Graph, std::shared_ptr<Graph>>(mg, "Graph", py::module_local())
      .def(py::init<size_t>(), "num_spins"_a)
      .def("gen_spin", [](const Graph& g, size_t seed) { Xorshift e((unsigned)seed); return g.gen_spin(e); }, "seed"_a)
      .def("gen_spin", [](const Graph& g) { Xorshift e(std::random_device{}()); return g.gen_spin(e); })
      .def("gen_binary", [](const Graph& g, size_t seed) { Xorshift e((unsigned)seed); return g.gen_binary(e); }, "seed"_a)
      .def("gen_binary", [](const Graph& g) { Xorshift e(std::random_device{}()); return g.gen_binary(e); })
      .def("size", &Graph::size);

  py::class_<Dense, Graph, std::shared_ptr<Dense>>(mg, "Dense", py::module_local())
      .def(py::init<size_t>(), "num_spins"_a)
      .def(py::init<const Dense&>(), "other"_a)
      .def("set_interaction_matrix", &Dense::set_interaction_matrix, "interaction"_a)
      .def("get_interactions", &Dense::get_interactions)
      .def("_flip_stats", &flip_stats<Dense>, "spins"_a, "threshold"_a)
      .def("calc_energy", [](const Dense& g, const std::vector<int>& s) { return g.energy(s); }, "spins"_a)
      .def("energy", [](const Dense& g, const std::vector<int>& s) { return g.energy(s); }, "spins"_a)
      .def("__setitem__", [](Dense& g, std::pair<size_t, size_t> k, double v) { g.set(k.first, k.second, v); }, "key"_a, "val"_a)
      .def("__getitem__", [](const Dense& g, std::pair<size_t, size_t> k) { return g.get(k.first, k.second); }, "key"_a)
      .def("__setitem__", [](Dense& g, size_t k, double v) { g.set(k, k, v); }, "key"_a, "val"_a)
      .def("__getitem__", [](const Dense& g, size_t k) { return g.get(k, k); }, "key"_a);

  py::class_<CSRSparse, Graph, std::shared_ptr<CSRSparse>>(mg, "CSRSparse", py::module_local())
      .def(py::init<const py::object&>(), "interaction"_a)
      .def(py::init<const CSRSparse&>(), "other"_a)
      .def("get_interactions", &CSRSparse::get_interactions)
      .def("_flip_stats", &flip_stats<CSRSparse>, "spins"_a, "threshold"_a)
      .def("calc_energy", [](const CSRSparse& g, const std::vector<int>& s) { return g.energy(s); }, "spins"_a)
      .def("energy", [](const CSRSparse& g, const std::vector<int>& s) { return g.energy(s); }, "spins"_a);

  py::class_<Sparse, Graph, std::shared_ptr<Sparse>>(mg, "Sparse", py::module_local())
      .def(py::init<size_t, size_t>(), "num_spins"_a, "num_edges"_a)
      .def(py::init<size_t>(), "num_spins"_a)
      .def(py::init<const Sparse&>(), "other"_a)
      .def("adj_nodes", &Sparse::adj_nodes, "ind"_a)
      .def("get_num_edges", &Sparse::get_num_edges)
      .def("get_interactions", &Sparse::get_interactions)
      .def("_flip_stats", &flip_stats<Sparse>, "spins"_a, "threshold"_a)
      .def("calc_energy", [](const Sparse& g, const std::vector<int>& s) { return g.energy(s); }, "spins"_a)
      .def("energy", [](const Sparse& g, const std::vector<int>& s) { return g.energy(s); }, "spins"_a)
      .def("__setitem__", [](Sparse& g, std::pair<size_t, size_t> k, double v) { g.J(k.first, k.second) = v; }, "key"_a, "val"_a)
      .def("__getitem__", [](const Sparse& g, std::pair<size_t, size_t> k) { return g.J(k.first, k.second); }, "key"_a)
      .def("__setitem__", [](Sparse& g, size_t k, double v) { g.h(k) = v; }, "key"_a, "val"_a)
      .def("__getitem__", [](const Sparse& g, size_t k) { return g.h(k); }, "key"_a);

  py::enum_<Dir>(mg, "Dir", py::module_local())
      .value("PLUS_R", Dir::PLUS_R)
      .value("MINUS_R", Dir::MINUS_R)
      .value("PLUS_C", Dir::PLUS_C)
      .value("MINUS_C", Dir::MINUS_C);
  using SqKey = std::tuple<size_t, size_t, Dir>;
  py::class_<Square, Sparse, std::shared_ptr<Square>>(mg, "Square", py::module_local())
      .def(py::init<size_t, size_t, double>(), "num_row"_a, "num_column"_a, "init_val"_a = 0.0)
      .def(py::init<const Square&>(), "other"_a)
      .def("to_ind", &Square::to_ind, "r"_a, "c"_a)
      .def("to_rc", &Square::to_rc, "ind"_a)
      .def("get_num_row", [](const Square& g) { return g.rows_; })
      .def("get_num_column", [](const Square& g) { return g.cols_; })
      .def("__setitem__", [](Square& g, const SqKey& k, double v) {
             const size_t r = std::get<0>(k), c = std::get<1>(k);
             const size_t j = g.neighbour(r, c, std::get<2>(k));
             g.J(g.to_ind((int64_t)r, (int64_t)c), j) = v;
           }, "key"_a, "val"_a)
      .def("__getitem__", [](const Square& g, const SqKey& k) {
             const size_t r = std::get<0>(k), c = std::get<1>(k);
             const size_t j = g.neighbour(r, c, std::get<2>(k));
             return g.J(g.to_ind((int64_t)r, (int64_t)c), j);
           }, "key"_a)
      .def("__setitem__", [](Square& g, std::pair<size_t, size_t> k, double v) {
             g.neighbour(k.first, k.second, Dir::PLUS_R);  // range check
             g.h(g.to_ind((int64_t)k.first, (int64_t)k.second)) = v;
           }, "key"_a, "val"_a)
      .def("__getitem__", [](const Square& g, std::pair<size_t, size_t> k) {
             g.neighbour(k.first, k.second, Dir::PLUS_R);
             return g.h(g.to_ind((int64_t)k.first, (int64_t)k.second));
           }, "key"_a);

  py::enum_<ChimeraDir>(mg, "ChimeraDir", py::module_local())
      .value("PLUS_R", ChimeraDir::PLUS_R)
      .value("MINUS_R", ChimeraDir::MINUS_R)
      .value("PLUS_C", ChimeraDir::PLUS_C)
      .value("MINUS_C", ChimeraDir::MINUS_C)
      .value("IN_0or4", ChimeraDir::IN_0or4)
      .value("IN_1or5", ChimeraDir::IN_1or5)
      .value("IN_2or6", ChimeraDir::IN_2or6)
      .value("IN_3or7", ChimeraDir::IN_3or7);
  using ChKey = std::tuple<size_t, size_t, size_t, ChimeraDir>;
  using ChSite = std::tuple<size_t, size_t, size_t>;
  py::class_<Chimera, Sparse, std::shared_ptr<Chimera>>(mg, "Chimera", py::module_local())
      .def(py::init<size_t, size_t, double>(), "num_row"_a, "num_column"_a, "init_val"_a = 0.0)
      .def(py::init<const Chimera&>(), "other"_a)
      .def("to_ind", &Chimera::to_ind, "r"_a, "c"_a, "i"_a)
      .def("to_rci", &Chimera::to_rci, "ind"_a)
      .def("get_num_row", [](const Chimera& g) { return g.rows_; })
      .def("get_num_column", [](const Chimera& g) { return g.cols_; })
      .def("get_num_in_chimera", [](const Chimera&) { return Chimera::kCell; })
      .def("__setitem__", [](Chimera& g, const ChKey& k, double v) {
             const size_t r = std::get<0>(k), c = std::get<1>(k), i = std::get<2>(k);
             const size_t j = g.neighbour(r, c, i, std::get<3>(k));
             g.J(g.to_ind((int64_t)r, (int64_t)c, (int64_t)i), j) = v;
           }, "key"_a, "val"_a)
      .def("__getitem__", [](const Chimera& g, const ChKey& k) {
             const size_t r = std::get<0>(k), c = std::get<1>(k), i = std::get<2>(k);
             const size_t j = g.neighbour(r, c, i, std::get<3>(k));
             return g.J(g.to_ind((int64_t)r, (int64_t)c, (int64_t)i), j);
           }, "key"_a)
      .def("__setitem__", [](Chimera& g, const ChSite& k, double v) {
             g.neighbour(std::get<0>(k), std::get<1>(k), std::get<2>(k), ChimeraDir::IN_0or4);  // range check
             g.h(g.to_ind((int64_t)std::get<0>(k), (int64_t)std::get<1>(k), (int64_t)std::get<2>(k))) = v;
           }, "key"_a, "val"_a)
      .def("__getitem__", [](const Chimera& g, const ChSite& k) {
             g.neighbour(std::get<0>(k), std::get<1>(k), std::get<2>(k), ChimeraDir::IN_0or4);
             return g.h(g.to_ind((int64_t)std::get<0>(k), (int64_t)std::get<1>(k), (int64_t)std::get<2>(k)));
           }, "key"_a);

  // ---- utility
  py::class_<ClassicalParam>(mu, "ClassicalUpdaterParameter", py::module_local())
      .def(py::init<>())
      .def(py::init([](double b) { return ClassicalParam{b}; }), "beta"_a)
      .def_readwrite("beta", &ClassicalParam::beta)
      .def("__repr__", [](const ClassicalParam& p) { return "(beta: " + std::to_string(p.beta) + ")"; });
  py::class_<TransverseParam>(mu, "TransverseFieldUpdaterParameter", py::module_local())
      .def(py::init<>())
      .def(py::init([](double b, double s) { return TransverseParam{b, s}; }), "beta"_a, "s"_a)
      .def(py::init([](std::pair<double, double> t) { return TransverseParam{t.first, t.second}; }), "obj"_a)
      .def_readwrite("beta", &TransverseParam::beta)
      .def_readwrite("s", &TransverseParam::s)
      .def("__repr__", [](const TransverseParam& p) {
        return "(beta: " + std::to_string(p.beta) + ", s: " + std::to_string(p.s) + ")";
      });
  py::class_<ClassicalSchedule>(mu, "ClassicalSchedule", py::module_local())
      .def(py::init<>())
      .def(py::init([](std::pair<ClassicalParam, size_t> o) { return ClassicalSchedule{o.first, o.second}; }), "obj"_a)
      .def_readwrite("one_mc_step", &ClassicalSchedule::one_mc_step)
      .def_readwrite("updater_parameter", &ClassicalSchedule::updater_parameter)
      .def("__repr__", [](const ClassicalSchedule& s) {
        return "((beta: " + std::to_string(s.updater_parameter.beta) + ") mcs: " + std::to_string(s.one_mc_step) + ")";
      });
  py::class_<TransverseSchedule>(mu, "TransverseFieldSchedule", py::module_local())
      .def(py::init<>())
      .def(py::init([](std::pair<TransverseParam, size_t> o) { return TransverseSchedule{o.first, o.second}; }), "obj"_a)
      .def_readwrite("one_mc_step", &TransverseSchedule::one_mc_step)
      .def_readwrite("updater_parameter", &TransverseSchedule::updater_parameter)
      .def("__repr__", [](const TransverseSchedule& s) {
        return "((beta: " + std::to_string(s.updater_parameter.beta) + ", s: " + std::to_string(s.updater_parameter.s) +
               ") mcs: " + std::to_string(s.one_mc_step) + ")";
      });
  mu.def("make_classical_schedule_list", &make_classical_schedule_list, "beta_min"_a, "beta_max"_a, "one_mc_step"_a,
         "num_call_updater"_a);
  mu.def("make_transverse_field_schedule_list", &make_transverse_field_schedule_list, "beta"_a, "one_mc_step"_a,
         "num_call_updater"_a);
  mu.def(
      "make_schedule_list",
      [](const std::vector<std::pair<double, size_t>>& tl) {
        std::vector<ClassicalSchedule> out;
        for (auto& e : tl) out.push_back(ClassicalSchedule{ClassicalParam{e.first}, e.second});
        return out;
      },
      "tuplelist"_a);
  mu.def(
      "make_schedule_list",
      [](const std::vector<std::pair<std::pair<double, double>, size_t>>& tl) {
        std::vector<TransverseSchedule> out;
        for (auto& e : tl) out.push_back(TransverseSchedule{TransverseParam{e.first.first, e.first.second}, e.second});
        return out;
      },
      "tuplelist"_a);

  // ---- systems, algorithm, result
  bind_graph_systems<Dense>(ms, ma, mr, "_Dense");
  bind_graph_systems<CSRSparse>(ms, ma, mr, "_CSRSparse");
  bind_graph_systems<Sparse>(ms, ma, mr, "_Sparse");  // Square and Chimera are Sparse graphs

  // ---- runtime controls (no reference counterpart)
  m.def(
      "set_device",
      [](int dev) {
        std::lock_guard<std::mutex> lk(g_ctx_mu);
        if (g_ctx) {
          oj_ctx_destroy(g_ctx);
          g_ctx = nullptr;
        }
        g_device = dev;
      },
      "device"_a);
  m.def("set_kernel", [](const std::string& k) {
    kernel_flag(k);
    g_kernel = k;
  }, "kernel"_a);
  m.def("last_run_info", []() {
    py::dict d;
    d["kernel"] = g_last_run.kernel;
    d["launches"] = g_last_run.launches;
    d["sweeps"] = g_last_run.sweeps;
    d["attempts"] = g_last_run.attempts;
    d["anneal_ms"] = g_last_run.anneal_ms;
    d["total_ms"] = g_last_run.total_ms;
    d["accepted"] = g_last_run.accepted;
    d["field_drift"] = g_last_run.field_drift;
    return d;
  });
  m.def("version", []() { return std::string(oj_version()); });
}
