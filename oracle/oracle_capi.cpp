// C entry points over the CPU oracle (TEST INFRASTRUCTURE ONLY), loaded with ctypes by
// tests/, the smoke check and the benchmark's CPU-baseline leg. Nothing in the product
// links this library.
#include <cstdint>
#include <cstring>
#include <vector>

#include "lbvh_oracle.hpp"
#include "mguso_oracle.hpp"

using namespace mo;

namespace {
Csr view_csr(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v) {
  Csr a;
  a.n = n;
  a.row_ptr.assign(rp, rp + n + 1);
  a.col_idx.assign(ci, ci + rp[n]);
  a.values.assign(v, v + rp[n]);
  return a;
}
}  // namespace

extern "C" {

// ---- CSR -------------------------------------------------------------------------------
void* oracle_csr_from_triplets(uint32_t n, const uint32_t* r, const uint32_t* c, const float* v, uint64_t nt) {
  std::vector<Triplet> t(nt);
  for (uint64_t k = 0; k < nt; ++k) t[k] = {r[k], c[k], v[k]};
  return new Csr(csr_from_triplets(n, t.data(), t.size()));
}

// Same input through the streaming TripletSink, with a Dirichlet mask (may be null).
void* oracle_csr_from_sink(uint32_t n, const uint32_t* r, const uint32_t* c, const float* v, uint64_t nt,
                           const uint8_t* pinned, uint32_t nverts) {
  TripletSink s;
  s.begin(n);
  for (uint64_t k = 0; k < nt; ++k) s.push({r[k], c[k], v[k]});
  std::vector<uint8_t> pin;
  if (pinned) pin.assign(pinned, pinned + nverts);
  return new Csr(s.finish(pin));
}

uint64_t oracle_csr_nnz(void* h) { return ((Csr*)h)->nnz(); }

void oracle_csr_copy(void* h, uint32_t* row_ptr, uint32_t* col_idx, float* values) {
  Csr* a = (Csr*)h;
  std::memcpy(row_ptr, a->row_ptr.data(), sizeof(uint32_t) * (a->n + 1));
  std::memcpy(col_idx, a->col_idx.data(), sizeof(uint32_t) * a->nnz());
  std::memcpy(values, a->values.data(), sizeof(float) * a->nnz());
}

void oracle_csr_free(void* h) { delete (Csr*)h; }

void oracle_spmv(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, const float* x, float* y) {
  Csr a = view_csr(n, rp, ci, v);
  spmv_f32(a, x, y);
}

// CG with kind 0 = diagonal, 1 = block Jacobi, 2 = one-level Schwarz(domain).
int oracle_cg(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, const float* b, float tol,
              uint32_t max_iter, int kind, uint32_t domain, float* x, uint32_t* iters, double* residual) {
  Csr a = view_csr(n, rp, ci, v);
  LinearStats s = cg_precond(a, b, tol, max_iter, (Precond)kind, domain, x);
  *iters = s.iters;
  *residual = s.residual;
  return 0;
}

// The reference's LinearSolver objects: kind 1 = CgCpu, 2 = SchwarzCpu(domain).
int oracle_linear_solve(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, const float* b,
                        float tol, uint32_t max_iter, int kind, uint32_t domain, float* x, uint32_t* iters,
                        double* residual) {
  Csr a = view_csr(n, rp, ci, v);
  LinearSolver s;
  s.kind = (Precond)kind;
  s.domain = domain;
  s.solve(a, b, tol, max_iter, x);
  *iters = s.last.iters;
  *residual = s.last.residual;
  return 0;
}

// Schwarz domains of a scalar CSR: domain id per vertex; returns the domain count.
uint32_t oracle_schwarz_domains(uint32_t n, const uint32_t* rp, const uint32_t* ci, uint32_t domain,
                                uint32_t* dom_of_vertex) {
  Csr a;
  a.n = n;
  a.row_ptr.assign(rp, rp + n + 1);
  a.col_idx.assign(ci, ci + rp[n]);
  a.values.assign(rp[n], 0.0f);
  auto doms = bfs_domains(vertex_adjacency(a), domain);
  for (size_t d = 0; d < doms.size(); ++d)
    for (uint32_t vtx : doms[d]) dom_of_vertex[vtx] = (uint32_t)d;
  return (uint32_t)doms.size();
}

// z = M^-1 r for the one-level Schwarz preconditioner (f64 factors, as the reference).
void oracle_schwarz_apply(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, uint32_t domain,
                          const double* r, double* z) {
  Csr a = view_csr(n, rp, ci, v);
  SchwarzTopology t = SchwarzTopology::build(a, domain);
  auto f = t.factorize(a);
  t.apply(f, r, z);
}

// The reference's SchwarzMlCpu(domain, weight) LinearSolver (two-level Schwarz CG).
int oracle_linear_solve_ml(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, const float* b,
                           float tol, uint32_t max_iter, uint32_t domain, double weight, float* x, uint32_t* iters,
                           double* residual) {
  Csr a = view_csr(n, rp, ci, v);
  LinearSolver s;
  s.kind = Precond::SchwarzMl;
  s.domain = domain;
  s.weight = weight;
  s.solve(a, b, tol, max_iter, x);
  *iters = s.last.iters;
  *residual = s.last.residual;
  return 0;
}

// z = M^-1 r for the two-level Schwarz preconditioner (SchwarzGpuBuilder::apply_cpu's
// arithmetic, linsolve.rs:767-775, in f64 throughout).
void oracle_schwarz_ml_apply(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, uint32_t domain,
                             double weight, const double* r, double* z) {
  Csr a = view_csr(n, rp, ci, v);
  MultilevelSchwarz ml = MultilevelSchwarz::build(a, domain, weight);
  Csr coarse = ml.coarse_matrix(a);
  auto f0 = ml.l0.factorize(a);
  auto f1 = ml.l1.factorize(coarse);
  ml.apply(f0, f1, r, z);
}

// The two-level plan: coarse node of every fine vertex (agg0), coarse domain of every
// coarse node, and the Galerkin coarse operator (scalar CSR, values aggregated in f32).
// Returns the coarse node count; coarse arrays are written only when the pointers are set
// and hold nnz entries (*nnz is set first).
uint32_t oracle_schwarz_ml_plan(uint32_t n, const uint32_t* rp, const uint32_t* ci, const float* v, uint32_t domain,
                                uint32_t* agg0, uint32_t* coarse_dom, uint64_t* nnz, uint32_t* c_rp, uint32_t* c_ci,
                                float* c_v) {
  Csr a = view_csr(n, rp, ci, v);
  MultilevelSchwarz ml = MultilevelSchwarz::build(a, domain, 1.0);
  std::memcpy(agg0, ml.agg0.data(), 4 * ml.agg0.size());
  for (size_t d = 0; d < ml.l1.domains.size(); ++d)
    for (uint32_t g : ml.l1.domains[d]) coarse_dom[g] = (uint32_t)d;
  Csr c = ml.coarse_matrix(a);
  *nnz = c.nnz();
  if (c_rp) std::memcpy(c_rp, c.row_ptr.data(), 4 * (c.n + 1));
  if (c_ci) std::memcpy(c_ci, c.col_idx.data(), 4 * c.nnz());
  if (c_v) std::memcpy(c_v, c.values.data(), 4 * c.nnz());
  return (uint32_t)ml.n_coarse;
}

// ---- LBVH ------------------------------------------------------------------------------
void oracle_morton(const float* pos, const uint32_t* tris, uint64_t nt, int bits, uint64_t* out) {
  if (bits == 30) {
    auto k = morton_codes<uint32_t>(pos, tris, nt, 30);
    for (uint64_t i = 0; i < nt; ++i) out[i] = k[i];
  } else {
    auto k = morton_codes<uint64_t>(pos, tris, nt, 63);
    for (uint64_t i = 0; i < nt; ++i) out[i] = k[i];
  }
}

void oracle_centroid_bounds(const float* pos, const uint32_t* tris, uint64_t nt, float* lo, float* inv) {
  centroid_bounds(pos, tris, nt, lo, inv);
}

// Stable (key, payload) sort; keys are u64 holding either width.
void oracle_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t n) {
  std::vector<uint64_t> k(keys, keys + n);
  std::vector<uint32_t> v(vals, vals + n);
  stable_sort_pairs(k, v);
  std::memcpy(keys, k.data(), 8 * n);
  std::memcpy(vals, v.data(), 4 * n);
}

void oracle_karras(const uint64_t* keys, uint64_t n, int bits, uint32_t* left, uint32_t* right) {
  if (bits == 30) {
    std::vector<uint32_t> k(n);
    for (uint64_t i = 0; i < n; ++i) k[i] = (uint32_t)keys[i];
    karras_tree<uint32_t>(k.data(), n, left, right);
  } else {
    karras_tree<uint64_t>(keys, n, left, right);
  }
}

void oracle_refit(const uint32_t* left, const uint32_t* right, const float* leaf, uint64_t n, float* node) {
  propagate_aabb(left, right, leaf, n, node);
}

// Full LBVH pipeline on the CPU: keys, permutation, tree, boxes and the pair set.
// Returns the number of pairs (written up to `cap`).
uint64_t oracle_lbvh(const float* pos, uint64_t nv, const uint32_t* tris, uint64_t nt, int bits, float dhat,
                     uint64_t* out_keys, uint32_t* out_perm, uint32_t* out_left, uint32_t* out_right,
                     float* out_node, uint32_t* out_pairs, uint64_t cap) {
  std::vector<uint64_t> keys(nt);
  oracle_morton(pos, tris, nt, bits, keys.data());
  std::vector<uint32_t> perm(nt);
  for (uint64_t i = 0; i < nt; ++i) perm[i] = (uint32_t)i;
  stable_sort_pairs(keys, perm);
  std::vector<uint32_t> left(nt > 0 ? nt - 1 : 0), right(nt > 0 ? nt - 1 : 0);
  oracle_karras(keys.data(), nt, bits, left.data(), right.data());
  std::vector<float> leaf = leaf_boxes(pos, tris, perm.data(), nt);
  std::vector<float> node(6 * (nt > 0 ? nt - 1 : 0));
  propagate_aabb(left.data(), right.data(), leaf.data(), nt, node.data());
  auto pairs = traverse_pairs(left.data(), right.data(), node.data(), leaf.data(), perm.data(), nt, pos, nv, dhat);
  if (out_keys) std::memcpy(out_keys, keys.data(), 8 * nt);
  if (out_perm) std::memcpy(out_perm, perm.data(), 4 * nt);
  if (out_left && nt > 1) std::memcpy(out_left, left.data(), 4 * (nt - 1));
  if (out_right && nt > 1) std::memcpy(out_right, right.data(), 4 * (nt - 1));
  if (out_node && nt > 1) std::memcpy(out_node, node.data(), 4 * 6 * (nt - 1));
  uint64_t np = pairs.size();
  if (out_pairs)
    for (uint64_t i = 0; i < np && i < cap; ++i) {
      out_pairs[2 * i] = pairs[i].first;
      out_pairs[2 * i + 1] = pairs[i].second;
    }
  return np;
}

}  // extern "C"
