// CPU oracle (TEST INFRASTRUCTURE ONLY) -- a C++17 restatement of the reference's
// single-threaded CPU linear-algebra path for the mguso implicit step.
//
// Only tests, the smoke check and the CPU-baseline leg of the benchmark may call this
// code; it is the checker, never the product. The product path lives in
// nguo-3d_b200/csrc and fails loudly when its CUDA library is missing.
//
// Parity status: pinned against the reference's own unit-test known answers
// (core-engine/crates/engine-core/src/linsolve.rs:856-1030, csr.rs:471-588), which the
// tests under tests/ port. The Rust reference itself cannot be compiled here (no cargo).
//
// Float rules: f32 math exactly in the reference's operation order, compiled with
// -ffp-contract=off and without -ffast-math. Templated on the real type so the same
// code gives the float restatement and the FP64 oracle.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace mo {

// ---------------------------------------------------------------------------------------
// Vec3 with glam's scalar semantics (dot = x*x' + y*y' + z*z', left to right;
// length = sqrt(dot); normalize = v * (1/length)).
// ---------------------------------------------------------------------------------------
template <class R>
struct V3 {
  R x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator-() const { return V3(-x, -y, -z); }
  V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
  V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
  V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  V3& operator*=(R s) { x *= s; y *= s; z *= s; return *this; }
  bool operator==(const V3& o) const { return x == o.x && y == o.y && z == o.z; }
  R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
  V3 cross(const V3& o) const {
    return V3(y * o.z - o.y * z, z * o.x - o.z * x, x * o.y - o.x * y);
  }
  R length_squared() const { return dot(*this); }
  R length() const { return std::sqrt(dot(*this)); }
  V3 normalize() const { return (*this) * (R(1) / length()); }
  V3 normalize_or(const V3& fb) const {
    R rcp = R(1) / length();
    if (std::isfinite(rcp) && rcp > R(0)) return (*this) * rcp;
    return fb;
  }
  V3 normalize_or_zero() const { return normalize_or(V3()); }
  V3 vmin(const V3& o) const { return V3(std::min(x, o.x), std::min(y, o.y), std::min(z, o.z)); }
  V3 vmax(const V3& o) const { return V3(std::max(x, o.x), std::max(y, o.y), std::max(z, o.z)); }
  bool finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
  template <class S>
  V3<S> cast() const { return V3<S>(S(x), S(y), S(z)); }
};
template <class R>
inline V3<R> operator*(R s, const V3<R>& v) { return v * s; }

// Rust's f32::max / f32::min ignore a NaN operand (IEEE maxNum); std::fmax does the same.
template <class R> inline R rmax(R a, R b) { return std::fmax(a, b); }
template <class R> inline R rmin(R a, R b) { return std::fmin(a, b); }
template <class R> inline R rclamp(R v, R lo, R hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------------------
// CSR (engine-core/src/csr.rs:9-14)
// ---------------------------------------------------------------------------------------
template <class R>
struct TripletT {
  uint32_t r, c;
  R v;
};

template <class R>
struct CsrT {
  size_t n = 0;
  std::vector<uint32_t> row_ptr, col_idx;
  std::vector<R> values;
  size_t nnz() const { return values.size(); }
};
using Triplet = TripletT<float>;
using Csr = CsrT<float>;

// Sort one row's (col, value) entries by column and coalesce duplicates (csr.rs:63-84).
// The reference uses an unstable sort; a stable sort is used here so duplicate cells are
// summed in push order (the Rust order of equal keys is implementation-defined, so the
// two agree up to the summation order of duplicates).
template <class R>
inline void sort_coalesce_row(std::vector<std::pair<uint32_t, R>>& flat, size_t lo, size_t hi,
                              std::vector<uint32_t>& col_idx, std::vector<R>& values) {
  std::stable_sort(flat.begin() + lo, flat.begin() + hi,
                   [](const std::pair<uint32_t, R>& a, const std::pair<uint32_t, R>& b) {
                     return a.first < b.first;
                   });
  size_t j = lo;
  while (j < hi) {
    uint32_t c = flat[j].first;
    R sum = R(0);
    while (j < hi && flat[j].first == c) {
      sum += flat[j].second;
      ++j;
    }
    col_idx.push_back(c);
    values.push_back(sum);
  }
}

// CsrMatrix::from_triplets (csr.rs:37-91): counting sort by row, per-row sort + coalesce.
template <class R>
inline CsrT<R> csr_from_triplets(size_t n, const TripletT<R>* t, size_t nt) {
  std::vector<uint32_t> starts(n + 1, 0);
  for (size_t k = 0; k < nt; ++k) starts[t[k].r + 1] += 1;
  for (size_t k = 0; k < n; ++k) starts[k + 1] += starts[k];
  std::vector<uint32_t> cursor(starts.begin(), starts.end() - 1);
  std::vector<std::pair<uint32_t, R>> flat(nt);
  for (size_t k = 0; k < nt; ++k) flat[cursor[t[k].r]++] = {t[k].c, t[k].v};
  CsrT<R> m;
  m.n = n;
  m.row_ptr.reserve(n + 1);
  m.row_ptr.push_back(0);
  for (size_t r = 0; r < n; ++r) {
    sort_coalesce_row(flat, starts[r], starts[r + 1], m.col_idx, m.values);
    m.row_ptr.push_back((uint32_t)m.col_idx.size());
  }
  return m;
}

// merge_csr (csr.rs:420-461): out = a + b, a's partial sums first.
template <class R>
inline void merge_csr(const CsrT<R>& a, const CsrT<R>& b, CsrT<R>& out) {
  size_t n = a.n;
  out.n = n;
  out.row_ptr.clear();
  out.col_idx.clear();
  out.values.clear();
  out.row_ptr.push_back(0);
  for (size_t r = 0; r < n; ++r) {
    size_t i = a.row_ptr[r], ie = a.row_ptr[r + 1];
    size_t j = b.row_ptr[r], je = b.row_ptr[r + 1];
    while (i < ie || j < je) {
      uint32_t ca = i < ie ? a.col_idx[i] : 0xffffffffu;
      uint32_t cb = j < je ? b.col_idx[j] : 0xffffffffu;
      if (ca < cb) {
        out.col_idx.push_back(ca);
        out.values.push_back(a.values[i++]);
      } else if (ca > cb) {
        out.col_idx.push_back(cb);
        out.values.push_back(b.values[j++]);
      } else {
        out.col_idx.push_back(ca);
        out.values.push_back(a.values[i] + b.values[j]);
        ++i;
        ++j;
      }
    }
    out.row_ptr.push_back((uint32_t)out.col_idx.size());
  }
}

// TripletSink (csr.rs:205-416): streaming chunked accumulator, CHUNK_MIN = 2^14 growing by
// doubling to CHUNK_MAX = 2^21, then folding; `finish` applies the Dirichlet filter.
template <class R>
struct TripletSinkT {
  static constexpr size_t CHUNK_MIN = size_t(1) << 14;
  static constexpr size_t CHUNK_MAX = size_t(1) << 21;
  size_t n = 0;
  std::vector<TripletT<R>> buf;
  size_t flush_at = CHUNK_MIN;
  size_t pushed = 0, flushes = 0;
  CsrT<R> acc, scratch, chunk;
  bool acc_empty = true;

  void begin(size_t n_) {
    n = n_;
    buf.clear();
    pushed = 0;
    flushes = 0;
    acc = CsrT<R>();
    acc.n = n;
    acc_empty = true;
  }
  void push(const TripletT<R>& t) {
    ++pushed;
    buf.push_back(t);
    if (buf.size() >= flush_at) {
      if (flush_at < CHUNK_MAX) {
        flush_at = std::min(flush_at * 2, CHUNK_MAX);
      } else {
        flush();
      }
    }
  }
  void flush() {
    if (buf.empty()) return;
    chunk = csr_from_triplets(n, buf.data(), buf.size());
    buf.clear();
    if (acc_empty) {
      std::swap(acc, chunk);
      acc_empty = false;
    } else {
      merge_csr(acc, chunk, scratch);
      std::swap(acc, scratch);
    }
    ++flushes;
  }
  // `pinned` indexed by vertex (dof / 3); empty pins nothing (csr.rs:385-415).
  CsrT<R> finish(const std::vector<uint8_t>& pinned) {
    flush();
    CsrT<R> out;
    out.n = n;
    out.row_ptr.push_back(0);
    auto pin = [&](size_t dof) { return dof / 3 < pinned.size() && pinned[dof / 3]; };
    for (size_t r = 0; r < n; ++r) {
      if (pin(r)) {
        out.col_idx.push_back((uint32_t)r);
        out.values.push_back(R(1));
      } else if (!acc_empty) {
        for (size_t k = acc.row_ptr[r]; k < acc.row_ptr[r + 1]; ++k) {
          uint32_t c = acc.col_idx[k];
          if (!pin(c)) {
            out.col_idx.push_back(c);
            out.values.push_back(acc.values[k]);
          }
        }
      }
      out.row_ptr.push_back((uint32_t)out.col_idx.size());
    }
    return out;
  }
};
using TripletSink = TripletSinkT<float>;

// CsrMatrix::spmv_cpu (csr.rs:98-111), accumulation in the value type.
template <class R>
inline void spmv_f32(const CsrT<R>& a, const R* x, R* y) {
  for (size_t r = 0; r < a.n; ++r) {
    R s = R(0);
    for (size_t k = a.row_ptr[r]; k < a.row_ptr[r + 1]; ++k) s += a.values[k] * x[a.col_idx[k]];
    y[r] = s;
  }
}

// CsrMatrix::diagonal (csr.rs:113-124).
template <class R>
inline std::vector<R> csr_diagonal(const CsrT<R>& a) {
  std::vector<R> d(a.n, R(0));
  for (size_t r = 0; r < a.n; ++r)
    for (size_t k = a.row_ptr[r]; k < a.row_ptr[r + 1]; ++k)
      if (a.col_idx[k] == r) d[r] = a.values[k];
  return d;
}

// ---------------------------------------------------------------------------------------
// linsolve.rs
// ---------------------------------------------------------------------------------------
enum class Precond { Diagonal = 0, Block = 1, Schwarz = 2, SchwarzMl = 3 };

struct LinearStats {
  uint32_t iters = 0;
  double residual = 0.0;
};

// invert3x3 (linsolve.rs:38-63); returns false when |det| < 1e-20.
inline bool invert3x3(const double m[3][3], double out[3][3]) {
  double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
               m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if (std::fabs(det) < 1e-20) return false;
  double id = 1.0 / det;
  out[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
  out[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
  out[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
  out[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
  out[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
  out[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
  out[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
  out[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
  out[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
  return true;
}

// cholesky (linsolve.rs:80-99): dense lower factor, row-major; false if not PD.
inline bool cholesky(const std::vector<double>& a, size_t m, std::vector<double>& l) {
  l.assign(m * m, 0.0);
  for (size_t i = 0; i < m; ++i) {
    for (size_t j = 0; j <= i; ++j) {
      double s = a[i * m + j];
      for (size_t k = 0; k < j; ++k) s -= l[i * m + k] * l[j * m + k];
      if (i == j) {
        if (s <= 1e-14) return false;
        l[i * m + i] = std::sqrt(s);
      } else {
        l[i * m + j] = s / l[j * m + j];
      }
    }
  }
  return true;
}

// chol_solve (linsolve.rs:102-118).
inline void chol_solve(const std::vector<double>& l, size_t m, const double* b, double* out) {
  std::vector<double> y(m, 0.0);
  for (size_t i = 0; i < m; ++i) {
    double s = b[i];
    for (size_t k = 0; k < i; ++k) s -= l[i * m + k] * y[k];
    y[i] = s / l[i * m + i];
  }
  for (size_t ii = m; ii-- > 0;) {
    double s = y[ii];
    for (size_t k = ii + 1; k < m; ++k) s -= l[k * m + ii] * out[k];
    out[ii] = s / l[ii * m + ii];
  }
}

// Greedy BFS aggregation of the block graph into disjoint domains of <= domain_size
// vertices (SchwarzTopology::build, linsolve.rs:134-173). Exposed on its own because the
// CUDA path computes the same domains on the host from the elastic block pattern.
inline std::vector<std::vector<uint32_t>> bfs_domains(const std::vector<std::vector<uint32_t>>& adj,
                                                      size_t domain_size) {
  size_t nv = adj.size();
  std::vector<uint8_t> assigned(nv, 0);
  std::vector<std::vector<uint32_t>> domains;
  for (size_t seed = 0; seed < nv; ++seed) {
    if (assigned[seed]) continue;
    std::vector<uint32_t> dom{(uint32_t)seed};
    assigned[seed] = 1;
    size_t fi = 0;
    while (dom.size() < domain_size && fi < dom.size()) {
      uint32_t v = dom[fi++];
      for (uint32_t nb : adj[v]) {
        if (!assigned[nb] && dom.size() < domain_size) {
          assigned[nb] = 1;
          dom.push_back(nb);
        }
      }
    }
    domains.push_back(std::move(dom));
  }
  return domains;
}

template <class R>
inline std::vector<std::vector<uint32_t>> vertex_adjacency(const CsrT<R>& a) {
  size_t nv = a.n / 3;
  std::vector<std::vector<uint32_t>> adj(nv);
  for (size_t row = 0; row < a.n; ++row) {
    uint32_t i = (uint32_t)(row / 3);
    for (size_t k = a.row_ptr[row]; k < a.row_ptr[row + 1]; ++k) {
      uint32_t j = a.col_idx[k] / 3;
      if (j != i) adj[i].push_back(j);
    }
  }
  for (auto& ai : adj) {
    std::sort(ai.begin(), ai.end());
    ai.erase(std::unique(ai.begin(), ai.end()), ai.end());
  }
  return adj;
}

struct SchwarzTopology {
  std::vector<std::vector<uint32_t>> domains;
  std::vector<std::vector<int64_t>> gather;  // -1 = structurally absent

  template <class R>
  static SchwarzTopology build(const CsrT<R>& a, size_t domain_size) {
    SchwarzTopology t;
    t.domains = bfs_domains(vertex_adjacency(a), domain_size);
    auto find_idx = [&](size_t row, size_t col) -> int64_t {
      for (size_t k = a.row_ptr[row]; k < a.row_ptr[row + 1]; ++k)
        if (a.col_idx[k] == col) return (int64_t)k;
      return -1;
    };
    for (auto& dom : t.domains) {
      std::vector<size_t> dofs;
      for (uint32_t v : dom)
        for (int c = 0; c < 3; ++c) dofs.push_back(3 * v + c);
      size_t m = dofs.size();
      std::vector<int64_t> g(m * m, -1);
      for (size_t p = 0; p < m; ++p)
        for (size_t q = 0; q < m; ++q) g[p * m + q] = find_idx(dofs[p], dofs[q]);
      t.gather.push_back(std::move(g));
    }
    return t;
  }

  // factorize (linsolve.rs:204-237): diagonal floor 1e-6*(tr/m) + 1e-8, then Cholesky;
  // a non-PD block falls back to sqrt of the floored diagonal.
  template <class R>
  std::vector<std::vector<double>> factorize(const CsrT<R>& a) const {
    std::vector<std::vector<double>> factors;
    factors.reserve(domains.size());
    for (size_t di = 0; di < domains.size(); ++di) {
      size_t m = 3 * domains[di].size();
      const auto& g = gather[di];
      std::vector<double> ad(m * m, 0.0);
      for (size_t e = 0; e < g.size(); ++e) ad[e] = g[e] < 0 ? 0.0 : (double)a.values[g[e]];
      double tr = 0.0;
      for (size_t k = 0; k < m; ++k) tr += ad[k * m + k];
      double floor = 1e-6 * (tr / (double)m) + 1e-8;
      for (size_t k = 0; k < m; ++k) ad[k * m + k] += floor;
      std::vector<double> l;
      if (!cholesky(ad, m, l)) {
        l.assign(m * m, 0.0);
        for (size_t p = 0; p < m; ++p) {
          double v = ad[p * m + p];
          l[p * m + p] = v > 1e-14 ? std::sqrt(v) : 1.0;
        }
      }
      factors.push_back(std::move(l));
    }
    return factors;
  }

  void apply(const std::vector<std::vector<double>>& factors, const double* r, double* z) const {
    for (size_t di = 0; di < domains.size(); ++di) {
      const auto& dom = domains[di];
      size_t m = 3 * dom.size();
      std::vector<double> rd(m), xd(m, 0.0);
      for (size_t p = 0; p < dom.size(); ++p)
        for (int c = 0; c < 3; ++c) rd[3 * p + c] = r[3 * dom[p] + c];
      chol_solve(factors[di], m, rd.data(), xd.data());
      for (size_t p = 0; p < dom.size(); ++p)
        for (int c = 0; c < 3; ++c) z[3 * dom[p] + c] = xd[3 * p + c];
    }
  }
};

// Two-level Galerkin additive Schwarz (MultilevelSchwarz, linsolve.rs:534-655):
//   z = S0 r + w C1^T S1 (C1 r)
// S0: the one-level domain solves; C1: restriction of a fine vertex to its level-0 domain
// (one coarse node per domain, three dofs), by summation; A1 = C1 A0 C1^T, the Galerkin
// coarse operator, aggregated in fine value order in the matrix's own precision
// (coarse_matrix, linsolve.rs:618-630); S1: a one-level Schwarz over A1 with the same domain
// size (its coarse domains are BFS groups of coarse nodes).
struct MultilevelSchwarz {
  SchwarzTopology l0;
  std::vector<uint32_t> agg0;  // fine vertex -> coarse node (its level-0 domain)
  size_t n_coarse = 0;
  CsrT<float> coarse_structure;        // values unused (structure only)
  std::vector<size_t> coarse_gather;   // fine value index -> coarse value index
  SchwarzTopology l1;
  double weight = 1.0;

  // build (linsolve.rs:555-608)
  template <class R>
  static MultilevelSchwarz build(const CsrT<R>& a, size_t domain, double weight) {
    MultilevelSchwarz ml;
    ml.l0 = SchwarzTopology::build(a, domain);
    const size_t nv = a.n / 3;
    ml.agg0.assign(nv, 0);
    for (size_t d = 0; d < ml.l0.domains.size(); ++d)
      for (uint32_t v : ml.l0.domains[d]) ml.agg0[v] = (uint32_t)d;
    ml.n_coarse = ml.l0.domains.size();
    auto coarse_dof = [&](size_t row) -> uint32_t { return (uint32_t)(3 * (size_t)ml.agg0[row / 3] + row % 3); };
    std::vector<TripletT<float>> trips;
    trips.reserve(a.nnz());
    for (size_t row = 0; row < a.n; ++row) {
      const uint32_t cr = coarse_dof(row);
      for (size_t k = a.row_ptr[row]; k < a.row_ptr[row + 1]; ++k)
        trips.push_back({cr, coarse_dof(a.col_idx[k]), 0.0f});
    }
    ml.coarse_structure = csr_from_triplets(3 * ml.n_coarse, trips.data(), trips.size());
    // (coarse row, coarse col) -> flat index: columns are sorted and unique per row
    const CsrT<float>& cs = ml.coarse_structure;
    ml.coarse_gather.assign(a.nnz(), 0);
    for (size_t row = 0; row < a.n; ++row) {
      const uint32_t cr = coarse_dof(row);
      const uint32_t* b = cs.col_idx.data() + cs.row_ptr[cr];
      const uint32_t* e = cs.col_idx.data() + cs.row_ptr[cr + 1];
      for (size_t k = a.row_ptr[row]; k < a.row_ptr[row + 1]; ++k) {
        const uint32_t cc = coarse_dof(a.col_idx[k]);
        ml.coarse_gather[k] = (size_t)(std::lower_bound(b, e, cc) - cs.col_idx.data());
      }
    }
    ml.l1 = SchwarzTopology::build(ml.coarse_structure, domain);
    ml.weight = weight;
    return ml;
  }

  // coarse_matrix (linsolve.rs:618-630): values summed in fine value order
  template <class R>
  CsrT<R> coarse_matrix(const CsrT<R>& a) const {
    CsrT<R> c;
    c.n = coarse_structure.n;
    c.row_ptr = coarse_structure.row_ptr;
    c.col_idx = coarse_structure.col_idx;
    c.values.assign(coarse_structure.nnz(), R(0));
    for (size_t k = 0; k < coarse_gather.size(); ++k) c.values[coarse_gather[k]] += a.values[k];
    return c;
  }

  // apply (linsolve.rs:641-666): level 0, restriction by sums in vertex order, coarse
  // smoother, weighted prolongation added to z
  void apply(const std::vector<std::vector<double>>& f0, const std::vector<std::vector<double>>& f1, const double* r,
             double* z) const {
    l0.apply(f0, r, z);
    const size_t nv = agg0.size();
    std::vector<double> rc(3 * n_coarse, 0.0), ec(3 * n_coarse, 0.0);
    for (size_t i = 0; i < nv; ++i) {
      const size_t g = agg0[i];
      rc[3 * g] += r[3 * i];
      rc[3 * g + 1] += r[3 * i + 1];
      rc[3 * g + 2] += r[3 * i + 2];
    }
    l1.apply(f1, rc.data(), ec.data());
    for (size_t i = 0; i < nv; ++i) {
      const size_t g = agg0[i];
      z[3 * i] += weight * ec[3 * g];
      z[3 * i + 1] += weight * ec[3 * g + 1];
      z[3 * i + 2] += weight * ec[3 * g + 2];
    }
  }
};

// cg_run (linsolve.rs:350-411): f64 PCG, x0 = 0, relative residual stop, pAp <= 0 break.
template <class R, class PrecondFn>
inline LinearStats cg_run(const CsrT<R>& a, const R* b, R tol, uint32_t max_iter, PrecondFn precond,
                          R* x_out) {
  size_t n = a.n;
  auto spmv = [&](const std::vector<double>& x, std::vector<double>& out) {
    for (size_t row = 0; row < n; ++row) {
      double s = 0.0;
      for (size_t k = a.row_ptr[row]; k < a.row_ptr[row + 1]; ++k)
        s += (double)a.values[k] * x[a.col_idx[k]];
      out[row] = s;
    }
  };
  auto dot = [&](const std::vector<double>& u, const std::vector<double>& v) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += u[i] * v[i];
    return s;
  };
  std::vector<double> bf(n);
  for (size_t i = 0; i < n; ++i) bf[i] = (double)b[i];
  double bnorm = std::max(std::sqrt(dot(bf, bf)), 1e-30);
  std::vector<double> x(n, 0.0), r = bf, z(n, 0.0), ap(n, 0.0);
  precond(r, z);
  std::vector<double> p = z;
  double rz = dot(r, z);
  LinearStats st;
  st.residual = std::sqrt(dot(r, r)) / bnorm;
  while (st.iters < max_iter) {
    spmv(p, ap);
    double pap = dot(p, ap);
    if (pap <= 0.0 || std::isnan(pap)) break;
    double alpha = rz / pap;
    for (size_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
    }
    st.iters += 1;
    st.residual = std::sqrt(dot(r, r)) / bnorm;
    if (st.residual <= (double)tol) break;
    precond(r, z);
    double rz_new = dot(r, z);
    double beta = rz_new / rz;
    for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rz = rz_new;
  }
  for (size_t i = 0; i < n; ++i) x_out[i] = (R)x[i];
  return st;
}

// cg_cpu_precond (linsolve.rs:272-346) with an explicit preconditioner kind.
template <class R>
inline LinearStats cg_precond(const CsrT<R>& a, const R* b, R tol, uint32_t max_iter, Precond kind_in,
                              size_t domain, R* x_out) {
  size_t n = a.n;
  bool block3 = n % 3 == 0;
  Precond kind = kind_in;
  if ((kind == Precond::Block || kind == Precond::Schwarz) && !block3) kind = Precond::Diagonal;
  std::vector<R> dg = csr_diagonal(a);
  std::vector<double> inv_diag(n);
  for (size_t i = 0; i < n; ++i) inv_diag[i] = dg[i] != R(0) ? 1.0 / (double)dg[i] : 1.0;
  std::vector<std::array<double, 9>> binv;
  if (kind == Precond::Block) {
    size_t nv = n / 3;
    binv.resize(nv);
    for (size_t i = 0; i < nv; ++i) {
      double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int r = 0; r < 3; ++r) {
        size_t row = 3 * i + r;
        for (size_t k = a.row_ptr[row]; k < a.row_ptr[row + 1]; ++k) {
          size_t c = a.col_idx[k];
          if (c >= 3 * i && c < 3 * i + 3) m[r][c - 3 * i] = (double)a.values[k];
        }
      }
      double inv[3][3];
      if (!invert3x3(m, inv)) {
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) inv[r][c] = r == c ? inv_diag[3 * i + r] : 0.0;
      }
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) binv[i][3 * r + c] = inv[r][c];
    }
  }
  SchwarzTopology topo;
  std::vector<std::vector<double>> factors;
  if (kind == Precond::Schwarz) {
    topo = SchwarzTopology::build(a, std::max<size_t>(domain, 1));
    factors = topo.factorize(a);
  }
  auto precond = [&](const std::vector<double>& r, std::vector<double>& z) {
    if (kind == Precond::Schwarz) {
      topo.apply(factors, r.data(), z.data());
    } else if (kind == Precond::Block) {
      for (size_t i = 0; i < binv.size(); ++i) {
        const auto& bi = binv[i];
        double r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
        z[3 * i] = bi[0] * r0 + bi[1] * r1 + bi[2] * r2;
        z[3 * i + 1] = bi[3] * r0 + bi[4] * r1 + bi[5] * r2;
        z[3 * i + 2] = bi[6] * r0 + bi[7] * r1 + bi[8] * r2;
      }
    } else {
      for (size_t i = 0; i < n; ++i) z[i] = r[i] * inv_diag[i];
    }
  };
  return cg_run(a, b, tol, max_iter, precond, x_out);
}

// relative_residual (linsolve.rs:445-455).
template <class R>
inline double relative_residual(const CsrT<R>& a, const R* x, const R* b) {
  std::vector<R> ax(a.n);
  spmv_f32(a, x, ax.data());
  double num = 0.0, den = 0.0;
  for (size_t i = 0; i < a.n; ++i) {
    double d = (double)b[i] - (double)ax[i];
    num += d * d;
    den += (double)b[i] * (double)b[i];
  }
  return std::sqrt(num) / std::max(std::sqrt(den), 1e-30);
}

// SchwarzMlCpu::solve (linsolve.rs:803-836): two-level Schwarz CG, stats from cg_run.
template <class R>
inline LinearStats cg_schwarz_ml(const CsrT<R>& a, const R* b, R tol, uint32_t max_iter, size_t domain,
                                 double weight, R* x_out) {
  MultilevelSchwarz ml = MultilevelSchwarz::build(a, std::max<size_t>(domain, 1), weight);
  CsrT<R> coarse = ml.coarse_matrix(a);
  auto f0 = ml.l0.factorize(a);
  auto f1 = ml.l1.factorize(coarse);
  auto precond = [&](const std::vector<double>& r, std::vector<double>& z) { ml.apply(f0, f1, r.data(), z.data()); };
  return cg_run(a, b, tol, max_iter, precond, x_out);
}

// A LinearSolver in the reference's sense (linsolve.rs:21-28): CgCpu (block Jacobi,
// stats residual recomputed by relative_residual), SchwarzCpu(domain) or
// SchwarzMlCpu(domain, weight).
struct LinearSolver {
  Precond kind = Precond::Block;
  size_t domain = 32;
  double weight = 0.7;
  LinearStats last;
  template <class R>
  void solve(const CsrT<R>& a, const R* b, R tol, uint32_t max_iter, R* x) {
    if (kind == Precond::SchwarzMl && a.n % 3 == 0) {
      last = cg_schwarz_ml(a, b, tol, max_iter, domain, weight, x);
    } else if (kind == Precond::SchwarzMl) {
      // SchwarzMlCpu on a non-3-block system: plain CG (solve_cg_cpu), iterations 0
      LinearStats s = cg_precond(a, b, tol, max_iter, Precond::Diagonal, domain, x);
      (void)s;
      last.iters = 0;
      last.residual = relative_residual(a, x, b);
    } else if (kind == Precond::Schwarz && a.n % 3 == 0) {
      last = cg_precond(a, b, tol, max_iter, Precond::Schwarz, domain, x);
    } else {
      Precond k = (a.n % 3 == 0) ? Precond::Block : Precond::Diagonal;
      LinearStats s = cg_precond(a, b, tol, max_iter, k, domain, x);
      last.iters = s.iters;
      last.residual = relative_residual(a, x, b);
    }
  }
};

}  // namespace mo
