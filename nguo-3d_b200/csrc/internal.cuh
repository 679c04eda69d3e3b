// Internal object layouts behind the opaque C-ABI handles.
#pragma once
#include <memory>
#include <vector>

#include <cuda_fp16.h>

#include "common.cuh"

namespace mg {
struct Lbvh;
}

struct mguso_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  mg::Lbvh* sort_scratch = nullptr;  // scratch for mguso_radix_sort_pairs
};

namespace mg {

// SpMV kernel variants (mguso_bsr_set_kernel).
enum SpmvVariant : int { SPMV_AUTO = 0, SPMV_TMA = 1, SPMV_DIRECT = 2, SPMV_SELL = 3 };

// Sliced-ELL copy of a BSR matrix: 32 block rows per slice, each slice padded to its
// longest row; within a slice, block k of lane l keeps its column at
// col[(base + k) * 32 + l] and entry e of its 3x3 block at val[((base + k) * 9 + e) * 32 + l],
// so every warp-wide load is one contiguous 128-byte line. Padding blocks are zero with
// the row's own column.
struct SellLayout {
  uint32_t nslices = 0;
  uint64_t total_k = 0;           // sum over slices of the padded length
  DevBuf<uint32_t> slice_base;    // nslices + 1 (in units of 32-block groups)
  DevBuf<uint32_t> col;           // 32 * total_k
  DevBuf<float> val;              // 9 * 32 * total_k
  bool ready = false;
};

// One TMA-staged tiling of a BSR matrix: tiles of <= `rows` block rows and <= `cap`
// blocks; each tile's value and column ranges are staged into shared memory by 1-D bulk
// copies (rounded out to 16-byte boundaries).
struct SpmvTiling {
  int rows = 0;     // block rows per tile (= threads per CTA)
  int stages = 0;   // pipeline depth
  uint32_t cap = 0; // max blocks per tile
  uint32_t ntiles = 0;
  uint32_t val_stage_bytes = 0, col_stage_bytes = 0;
  int grid = 0;     // persistent CTAs
  DevBuf<uint32_t> tile_row;  // ntiles + 1
  bool ok = false;  // false when some row is longer than `cap`
};

}  // namespace mg

struct mguso_bsr {
  mguso_ctx* ctx = nullptr;
  uint32_t nb = 0, nnzb = 0;
  std::vector<uint32_t> h_row_ptr, h_col;  // host copy of the pattern
  mg::DevBuf<uint32_t> row_ptr, col;
  mg::DevBuf<float> val;
  int variant = mg::SPMV_AUTO;
  int tiling_choice = 0;  // index into tilings when variant == TMA
  std::vector<std::unique_ptr<mg::SpmvTiling>> tilings;
  mg::SellLayout sell;
  std::vector<float> h_val_keep;  // host values kept for building the sliced copy lazily
  mg::DevBuf<uint32_t> status;
  mg::DevBuf<float> hx, hy;  // staging for spmv_host
};

struct mguso_schwarz {
  mguso_bsr* a = nullptr;
  uint32_t domain = 32;
  uint32_t ndom = 0;
  uint32_t max_m = 0;
  std::vector<uint32_t> inst_vert;  // optional instance vertex ranges (domains stay inside one)
  std::vector<uint32_t> h_dom_start, h_dom_verts, h_dom_of;
  mg::DevBuf<uint32_t> dom_start;  // ndom + 1 (vertex offsets)
  mg::DevBuf<uint32_t> dom_verts;  // nb
  mg::DevBuf<uint32_t> dom_of;     // nb
  mg::DevBuf<uint32_t> loc;        // nb: local index of a vertex inside its domain
  mg::DevBuf<uint64_t> fac_off;    // ndom + 1 (float offsets, 4-float aligned)
  mg::DevBuf<float> fac;           // W = L^-1 per domain, swizzled 32x32 FP32 tiles
  uint64_t fac_floats = 0;         // elements of the tile storage
  // FP16 storage instead (the step's preconditioner): W = fac_scale[d] * fac_h (the largest
  // |W| of the domain), which halves the apply's traffic and shared-memory slice
  bool half = false;
  mg::DevBuf<__half> fac_h;
  mg::DevBuf<float> fac_scale;
  mg::DevBuf<uint32_t> status;
  // Packed domains of vertices without off-diagonal blocks are block diagonal: each of their
  // vertices is factored on its own, as the reference's one-vertex domain (floor from its
  // own trace), and stores its 3x3 lower W_v (6 floats: w00 w10 w11 w20 w21 w22, in vfac at
  // 6 v); such a domain has no tiles. dom_diag[d] marks them.
  std::vector<uint8_t> h_dom_diag;
  mg::DevBuf<uint8_t> dom_diag;
  mg::DevBuf<float> vfac;
  // each domain's instance; the factorisation skips the domains of instances outside
  // `active` (their factors keep their last values; a batch step sets it per Newton iteration)
  mg::DevBuf<uint8_t> dom_inst;
  uint32_t active = 0xffffffffu;
  // Two-level Galerkin form (MultilevelSchwarz, linsolve.rs:534-666) when levels == 2: every
  // level-0 domain is a coarse node (three dofs), coarse domains are BFS groups of <= domain
  // coarse nodes over the coarse block graph, and each coarse domain's dense block of
  // A1 = C1 A C1^T is factored like a level-0 domain (FP32 W1 tiles). Level-0 isolated
  // vertices are packed only when pack_singles is set (the reference gives each its own domain).
  uint32_t levels = 1;
  float weight = 0.7f;
  bool pack_singles = true;
  uint32_t ncdom = 0, max_m1 = 0;
  std::vector<uint32_t> h_cdom_start, h_cdom_nodes;
  mg::DevBuf<uint32_t> cdom_start;  // ncdom + 1
  mg::DevBuf<uint32_t> cdom_nodes;  // ndom: coarse nodes (level-0 domains) by coarse domain
  mg::DevBuf<uint32_t> cdom_of;     // ndom: coarse domain of each coarse node
  mg::DevBuf<uint32_t> cloc;        // ndom: local index of a coarse node in its coarse domain
  mg::DevBuf<uint32_t> dom_sorted;  // nb: each level-0 domain's vertices in ascending order
  mg::DevBuf<uint64_t> cfac_off;    // ncdom + 1
  mg::DevBuf<float> cfac;           // W1 tiles
  mg::DevBuf<float> ec;             // 3 * ndom: the coarse correction of the last apply
};

namespace mg {

// ---- BSR -------------------------------------------------------------------------------
int bsr_build_host_from_csr(const mguso_csr* a, uint32_t& nb, std::vector<uint32_t>& row_ptr,
                            std::vector<uint32_t>& col, std::vector<float>& val);
int bsr_upload(mguso_bsr* m, uint32_t nb, const std::vector<uint32_t>& row_ptr, const std::vector<uint32_t>& col,
               const float* val_host);
int bsr_prepare_tilings(mguso_bsr* m);
// y = A x; optional fused dot(x, y) partial reduction into `dot` (see Reduce).
struct DotSink;
int bsr_spmv(mguso_bsr* m, const float* x, float* y, cudaStream_t s, const DotSink* dot);
int bsr_autotune(mguso_bsr* m, float* best_us);
int bsr_build_sell(mguso_bsr* m);

// ---- Schwarz ---------------------------------------------------------------------------
int schwarz_build(mguso_schwarz* s);
int schwarz_factor(mguso_schwarz* s, cudaStream_t st);
int schwarz_apply(mguso_schwarz* s, const float* r, float* z, cudaStream_t st, const DotSink* dot);

// ---- deterministic grid reductions ----------------------------------------------------
// Kernels that produce a dot product write one partial per CTA into `partials`; the last
// CTA to finish (counted through `counter`) sums the partials in index order and runs the
// `finish` step, so results do not depend on CTA scheduling.
enum DotFinish : int {
  FIN_STORE = 0,   // out = sum
  FIN_PAP = 1,     // pap = sum; alpha = rz / pap; breakdown when pap <= 0 or NaN
  FIN_RR = 2,      // residual = sqrt(sum)/bnorm; ++iters; done when residual <= tol or iters == max
  FIN_RZ = 3,      // beta = sum / rz; rz = sum
  FIN_RZ0 = 4,     // rz = sum (setup)
  FIN_BNORM = 5,   // bnorm = max(sqrt(sum), 1e-30)
  FIN_RR0 = 6,     // residual = sqrt(sum) / bnorm (setup)
};

struct PcgScalars {
  double rz, pap, alpha, beta, bnorm, residual, tol, out;
  uint32_t iters, max_iter, done, status;
  uint32_t counter;
  uint32_t pad[3];
};

struct DotSink {
  PcgScalars* sc;     // device
  void* partials;     // device, >= max grid entries (double or float per `mixed`)
  int finish;
  bool mixed;         // accumulate in FP64
};

constexpr int MAX_PARTIALS = 4096;

// Persistent PCG: instances per launch and each instance's result.
constexpr int PCG_MAX_INST = 8;
// Fused (two-kernel) PCG: device-resident per-instance state and control words.
struct FusedInst {
  double rz, alpha, beta, bnorm, residual;
  uint32_t iters, done, upd, status;
};
struct FusedCtl {
  uint32_t counter[2];
  uint32_t all_done;
  uint32_t rounds;  // graph bodies of FUSED_CHECK iterations run (device-driven loop)
};

struct PcgInstResult {
  double residual;
  uint32_t iters, status, done, pad;
};

// Device vectors, scalars and the cached CUDA graph of one PCG operator.
struct PcgWork {
  uint32_t n = 0;
  DevBuf<float> b, x, r, z, p, ap, p2;  // p2: second direction buffer (persistent PCG)
  DevBuf<PcgScalars> sc;
  DevBuf<double> partials;
  PcgScalars* h_sc = nullptr;  // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_key = 0;
  bool graph_mixed = false;
  int reserve(uint32_t n);
  void drop_graph();
  PcgWork() = default;
  PcgWork(const PcgWork&) = delete;
  PcgWork& operator=(const PcgWork&) = delete;
  ~PcgWork();
};

}  // namespace mg

struct mguso_linear_solver {
  mguso_ctx* ctx = nullptr;
  int precond = MGUSO_PRECOND_SCHWARZ;
  uint32_t domain = 32;
  int precision = MGUSO_PRECISION_MIXED;
  uint32_t levels = 1;  // 2: two-level Schwarz (SchwarzMlCpu)
  float weight = 0.7f;
  // cached pattern (rebuild BSR/domains only when the scalar sparsity changes)
  std::vector<uint32_t> csr_row_ptr, csr_col;
  std::unique_ptr<mguso_bsr> bsr;
  std::unique_ptr<mguso_schwarz> schwarz;
  mg::DevBuf<float> bjinv;  // 9 per vertex (block Jacobi)
  mg::PcgWork work;
  uint64_t generation = 0;         // bumped whenever the pattern is rebuilt
  std::vector<uint32_t> map_val;   // scalar CSR entry -> BSR value slot
  std::vector<float> h_val;
};

namespace mg {
int pcg_solve(mguso_linear_solver* s, float tol, uint32_t max_iter, mguso_lin_stats* st);
int blockjacobi_factor(mguso_bsr* a, float* inv, cudaStream_t s);
}  // namespace mg
