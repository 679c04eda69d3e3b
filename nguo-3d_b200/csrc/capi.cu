// extern "C" entry points declared in include/mguso_cuda.h (linear-algebra half).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "lbvh.cuh"

namespace mg {
static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const std::string& get_error() { return g_err; }
}  // namespace mg

using namespace mg;

extern "C" {

int mguso_version(void) { return 100; }

size_t mguso_last_error(char* buf, size_t len) {
  const std::string& e = get_error();
  if (buf && len) {
    size_t n = std::min(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = 0;
  }
  return e.size();
}

int mguso_ctx_create(int device, mguso_ctx** out) {
  MG_CHECK_ARG(out, "out is null");
  int count = 0;
  MG_CUDA(cudaGetDeviceCount(&count));
  MG_CHECK_ARG(device >= 0 && device < count, "device index out of range");
  MG_CUDA(cudaSetDevice(device));
  auto* c = new mguso_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    set_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    return MGUSO_ERR_CUDA;
  }
  *out = c;
  return MGUSO_OK;
}

int mguso_ctx_destroy(mguso_ctx* ctx) {
  if (!ctx) return MGUSO_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx->sort_scratch;
  delete ctx;
  return MGUSO_OK;
}

void* mguso_ctx_stream(mguso_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

// ---- BSR -------------------------------------------------------------------------------
int mguso_bsr_create(mguso_ctx* ctx, uint32_t nb, const uint32_t* row_ptr, const uint32_t* col, const float* val,
                     mguso_bsr** out) {
  MG_CHECK_ARG(ctx && out && row_ptr, "null argument");
  uint32_t nnzb = row_ptr[nb];
  MG_CHECK_ARG(nnzb == 0 || (col && val), "null col/val");
  for (uint32_t r = 0; r < nb; ++r) {
    MG_CHECK_ARG(row_ptr[r] <= row_ptr[r + 1], "row_ptr not monotone");
    for (uint32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
      MG_CHECK_ARG(col[k] < nb, "block column out of range");
      MG_CHECK_ARG(k == row_ptr[r] || col[k] > col[k - 1], "block columns must be sorted and unique per row");
    }
  }
  MG_CUDA(cudaSetDevice(ctx->device));
  auto m = std::make_unique<mguso_bsr>();
  m->ctx = ctx;
  std::vector<uint32_t> rp(row_ptr, row_ptr + nb + 1), cl(col, col + nnzb);
  MG_TRY(bsr_upload(m.get(), nb, rp, cl, val));
  *out = m.release();
  return MGUSO_OK;
}

int mguso_bsr_create_from_csr(mguso_ctx* ctx, const mguso_csr* a, mguso_bsr** out) {
  MG_CHECK_ARG(ctx && a && out, "null argument");
  uint32_t nb = 0;
  std::vector<uint32_t> rp, cl;
  std::vector<float> val;
  MG_TRY(bsr_build_host_from_csr(a, nb, rp, cl, val));
  MG_CUDA(cudaSetDevice(ctx->device));
  auto m = std::make_unique<mguso_bsr>();
  m->ctx = ctx;
  MG_TRY(bsr_upload(m.get(), nb, rp, cl, val.data()));
  *out = m.release();
  return MGUSO_OK;
}

int mguso_bsr_destroy(mguso_bsr* a) {
  delete a;
  return MGUSO_OK;
}

int mguso_bsr_info(const mguso_bsr* a, uint32_t* nb, uint32_t* nnzb) {
  MG_CHECK_ARG(a, "null bsr");
  if (nb) *nb = a->nb;
  if (nnzb) *nnzb = a->nnzb;
  return MGUSO_OK;
}

int mguso_bsr_spmv(mguso_bsr* a, const float* x, float* y, void* stream) {
  MG_CHECK_ARG(a && (a->nb == 0 || (x && y)), "null argument");
  return bsr_spmv(a, x, y, (cudaStream_t)stream, nullptr);
}

int mguso_bsr_spmv_host(mguso_bsr* a, const float* x, float* y) {
  MG_CHECK_ARG(a && x && y, "null argument");
  cudaStream_t s = a->ctx->stream;
  size_t n = 3 * (size_t)a->nb;
  MG_TRY(a->hx.reserve(n));
  MG_TRY(a->hy.reserve(n));
  MG_CUDA(cudaMemcpyAsync(a->hx.p, x, n * 4, cudaMemcpyHostToDevice, s));
  MG_TRY(bsr_spmv(a, a->hx.p, a->hy.p, s, nullptr));
  MG_CUDA(cudaMemcpyAsync(y, a->hy.p, n * 4, cudaMemcpyDeviceToHost, s));
  MG_CUDA(cudaStreamSynchronize(s));
  uint32_t st = 0;
  MG_CUDA(cudaMemcpy(&st, a->status.p, 4, cudaMemcpyDeviceToHost));
  if (st & ST_WAIT_TIMEOUT) {
    set_error("SpMV: a bounded wait on a bulk copy timed out");
    return MGUSO_ERR_TIMEOUT;
  }
  return MGUSO_OK;
}

int mguso_bsr_set_kernel(mguso_bsr* a, int variant, int* active) {
  MG_CHECK_ARG(a && variant >= 0 && variant <= 3, "bad variant");
  if (variant == SPMV_SELL) MG_TRY(bsr_build_sell(a));
  a->variant = variant;
  if (active) *active = (variant == SPMV_AUTO) ? (a->tiling_choice >= 0 ? SPMV_TMA : SPMV_DIRECT) : variant;
  return MGUSO_OK;
}

int mguso_bsr_kernel(const mguso_bsr* a, int* variant, int* tile_rows, int* stages) {
  MG_CHECK_ARG(a && variant, "bad argument");
  *variant = a->variant;
  const bool tma = a->variant == SPMV_TMA && a->tiling_choice >= 0 && a->tiling_choice < (int)a->tilings.size();
  if (tile_rows) *tile_rows = tma ? a->tilings[a->tiling_choice]->rows : 0;
  if (stages) *stages = tma ? a->tilings[a->tiling_choice]->stages : 0;
  return MGUSO_OK;
}

int mguso_bsr_autotune(mguso_bsr* a, float* best_us) {
  MG_CHECK_ARG(a, "null bsr");
  return bsr_autotune(a, best_us);
}

// ---- Schwarz ---------------------------------------------------------------------------
int mguso_schwarz_create(mguso_bsr* a, uint32_t domain, mguso_schwarz** out) {
  MG_CHECK_ARG(a && out, "null argument");
  MG_CHECK_ARG(domain >= 1 && domain <= 32, "Schwarz domain size must be in [1, 32] vertices");
  auto s = std::make_unique<mguso_schwarz>();
  s->a = a;
  s->domain = domain;
  MG_TRY(schwarz_build(s.get()));
  *out = s.release();
  return MGUSO_OK;
}

int mguso_schwarz_create_ml(mguso_bsr* a, uint32_t domain, float weight, mguso_schwarz** out) {
  MG_CHECK_ARG(a && out, "null argument");
  MG_CHECK_ARG(domain >= 1 && domain <= 32, "Schwarz domain size must be in [1, 32] vertices");
  MG_CHECK_ARG(std::isfinite(weight) && weight >= 0.f, "coarse weight must be finite and >= 0");
  auto s = std::make_unique<mguso_schwarz>();
  s->a = a;
  s->domain = domain;
  s->levels = 2;
  s->weight = weight;
  s->pack_singles = false;
  MG_TRY(schwarz_build(s.get()));
  *out = s.release();
  return MGUSO_OK;
}

int mguso_schwarz_coarse_domains(const mguso_schwarz* s, uint32_t* coarse_dom_of_domain) {
  MG_CHECK_ARG(s && coarse_dom_of_domain, "null argument");
  MG_CHECK_ARG(s->levels == 2, "not a two-level Schwarz preconditioner");
  for (uint32_t d = 0; d < s->ncdom; ++d)
    for (uint32_t k = s->h_cdom_start[d]; k < s->h_cdom_start[d + 1]; ++k) coarse_dom_of_domain[s->h_cdom_nodes[k]] = d;
  return MGUSO_OK;
}

int mguso_schwarz_destroy(mguso_schwarz* s) {
  delete s;
  return MGUSO_OK;
}

int mguso_schwarz_info(const mguso_schwarz* s, uint32_t* ndomains, uint64_t* factor_bytes) {
  MG_CHECK_ARG(s, "null schwarz");
  if (ndomains) *ndomains = s->ndom;
  if (factor_bytes) *factor_bytes = (s->half ? 2 : 4) * s->fac_floats;
  return MGUSO_OK;
}

int mguso_schwarz_factor(mguso_schwarz* s, void* stream) {
  MG_CHECK_ARG(s, "null schwarz");
  return schwarz_factor(s, (cudaStream_t)stream);
}

int mguso_schwarz_apply(mguso_schwarz* s, const float* r, float* z, void* stream) {
  MG_CHECK_ARG(s && r && z, "null argument");
  return schwarz_apply(s, r, z, (cudaStream_t)stream, nullptr);
}

int mguso_schwarz_domains(const mguso_schwarz* s, uint32_t* dom_of_vertex) {
  MG_CHECK_ARG(s && dom_of_vertex, "null argument");
  std::memcpy(dom_of_vertex, s->h_dom_of.data(), 4 * s->h_dom_of.size());
  return MGUSO_OK;
}

// ---- LinearSolver ----------------------------------------------------------------------
int mguso_linear_solver_create(mguso_ctx* ctx, int precond, uint32_t domain, int precision,
                               mguso_linear_solver** out) {
  MG_CHECK_ARG(ctx && out, "null argument");
  MG_CHECK_ARG(precond == MGUSO_PRECOND_BLOCK_JACOBI || precond == MGUSO_PRECOND_SCHWARZ, "unknown preconditioner");
  MG_CHECK_ARG(precision == MGUSO_PRECISION_FP32 || precision == MGUSO_PRECISION_MIXED, "unknown precision");
  MG_CHECK_ARG(precond != MGUSO_PRECOND_SCHWARZ || (domain >= 1 && domain <= 32),
               "Schwarz domain size must be in [1, 32] vertices");
  auto* s = new mguso_linear_solver();
  s->ctx = ctx;
  s->precond = precond;
  s->domain = domain;
  s->precision = precision;
  *out = s;
  return MGUSO_OK;
}

int mguso_linear_solver_create_ml(mguso_ctx* ctx, uint32_t domain, float weight, int precision,
                                  mguso_linear_solver** out) {
  MG_CHECK_ARG(std::isfinite(weight) && weight >= 0.f, "coarse weight must be finite and >= 0");
  MG_TRY(mguso_linear_solver_create(ctx, MGUSO_PRECOND_SCHWARZ, domain, precision, out));
  (*out)->levels = 2;
  (*out)->weight = weight;
  return MGUSO_OK;
}

int mguso_linear_solver_destroy(mguso_linear_solver* s) {
  if (!s) return MGUSO_OK;
  delete s;
  return MGUSO_OK;
}

int mguso_linear_solve(mguso_linear_solver* s, const mguso_csr* a, const float* b, float tol, uint32_t max_iter,
                       float* x, mguso_lin_stats* stats) {
  MG_CHECK_ARG(s && a && b && x, "null argument");
  MG_CHECK_ARG(a->n % 3 == 0, "CSR order must be a multiple of 3");
  MG_CUDA(cudaSetDevice(s->ctx->device));
  cudaStream_t st = s->ctx->stream;
  uint32_t nnz = a->row_ptr[a->n];
  bool same = s->bsr && s->csr_row_ptr.size() == (size_t)a->n + 1 &&
              std::equal(s->csr_row_ptr.begin(), s->csr_row_ptr.end(), a->row_ptr) &&
              s->csr_col.size() == nnz && std::equal(s->csr_col.begin(), s->csr_col.end(), a->col_idx);
  if (!same) {
    uint32_t nb = 0;
    std::vector<uint32_t> rp, cl;
    std::vector<float> val;
    MG_TRY(bsr_build_host_from_csr(a, nb, rp, cl, val));
    s->bsr = std::make_unique<mguso_bsr>();
    s->bsr->ctx = s->ctx;
    MG_TRY(bsr_upload(s->bsr.get(), nb, rp, cl, val.data()));
    // scalar entry -> BSR value slot, so a re-solve on the same pattern scatters values only
    s->map_val.resize(nnz);
    for (uint32_t row = 0; row < a->n; ++row) {
      uint32_t v = row / 3;
      for (uint32_t k = a->row_ptr[row]; k < a->row_ptr[row + 1]; ++k) {
        uint32_t cb = a->col_idx[k] / 3;
        uint32_t j = (uint32_t)(std::lower_bound(cl.begin() + rp[v], cl.begin() + rp[v + 1], cb) - cl.begin());
        s->map_val[k] = 9 * j + 3 * (row % 3) + a->col_idx[k] % 3;
      }
    }
    s->csr_row_ptr.assign(a->row_ptr, a->row_ptr + a->n + 1);
    s->csr_col.assign(a->col_idx, a->col_idx + nnz);
    s->generation++;
    if (s->precond == MGUSO_PRECOND_SCHWARZ) {
      s->schwarz = std::make_unique<mguso_schwarz>();
      s->schwarz->a = s->bsr.get();
      s->schwarz->domain = s->domain;
      s->schwarz->levels = s->levels;
      s->schwarz->weight = s->weight;
      s->schwarz->pack_singles = s->levels != 2;  // two levels: every domain a coarse node, as the reference
      MG_TRY(schwarz_build(s->schwarz.get()));
    }
  } else {
    s->h_val.assign((size_t)9 * s->bsr->nnzb, 0.0f);
    for (uint32_t k = 0; k < nnz; ++k) s->h_val[s->map_val[k]] += a->values[k];
    MG_CUDA(cudaMemcpyAsync(s->bsr->val.p, s->h_val.data(), 4 * s->h_val.size(), cudaMemcpyHostToDevice, st));
  }
  uint32_t n = a->n;
  MG_TRY(s->work.reserve(n));
  MG_CUDA(cudaMemcpyAsync(s->work.b.p, b, 4 * (size_t)n, cudaMemcpyHostToDevice, st));
  if (s->precond == MGUSO_PRECOND_SCHWARZ) {
    MG_TRY(schwarz_factor(s->schwarz.get(), st));
  } else {
    MG_TRY(s->bjinv.reserve((size_t)9 * s->bsr->nb));
    MG_TRY(blockjacobi_factor(s->bsr.get(), s->bjinv.p, st));
  }
  mguso_lin_stats local{};
  MG_TRY(pcg_solve(s, tol, max_iter, &local));
  MG_CUDA(cudaMemcpyAsync(x, s->work.x.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  if (stats) *stats = local;
  return MGUSO_OK;
}

}  // extern "C"
