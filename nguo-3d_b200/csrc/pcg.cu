// Preconditioned conjugate gradient on the device (linsolve.rs:350-411).
//
// Same iteration as the reference's cg_run: x0 = 0, r = b, z = M^-1 r, p = z; per
// iteration Ap = A p, alpha = rz / pAp (break on pAp <= 0 or NaN), x += alpha p,
// r -= alpha Ap, stop when ||r||/||b|| <= tol, else z = M^-1 r, beta = rz'/rz,
// p = z + beta p. Vectors are FP32; dot products and norms are FP64 (MIXED) or FP32.
//
// Every dot product is fused into the kernel producing its operand and reduced
// deterministically (per-CTA partials summed in index order by the last CTA), which also
// computes alpha/beta/residual on the device. Kernels after convergence exit at entry, so
// the host launches CHECK iterations (captured once as a CUDA graph) between reads of the
// done flag.
#include <algorithm>
#include <cstring>

#include "reduce.cuh"

namespace mg {

template <class Acc>
__global__ void k_pcg_init(const float* __restrict__ b, float* __restrict__ x, float* __restrict__ r, uint32_t n,
                           DotSink d) {
  Acc acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float bi = b[i];
    x[i] = 0.f;
    r[i] = bi;
    acc += (Acc)bi * (Acc)bi;
  }
  grid_dot_commit<Acc>(d, acc);
}

template <class Acc>
__global__ void k_copy_dot(const float* __restrict__ z, float* __restrict__ p, const float* __restrict__ r,
                           uint32_t n, DotSink d) {
  Acc acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    p[i] = z[i];
    float ri = r[i];
    acc += (Acc)ri * (Acc)ri;
  }
  grid_dot_commit<Acc>(d, acc);
}

// x += alpha p; r -= alpha Ap; partial r.r
template <class Acc>
__global__ void k_pcg_update(float* __restrict__ x, float* __restrict__ r, const float* __restrict__ p,
                             const float* __restrict__ ap, uint32_t n, DotSink d) {
  if (d.sc->done) return;
  const float alpha = (float)d.sc->alpha;
  Acc acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fmaf(alpha, p[i], x[i]);
    float ri = fmaf(-alpha, ap[i], r[i]);
    r[i] = ri;
    acc += (Acc)ri * (Acc)ri;
  }
  grid_dot_commit<Acc>(d, acc);
}

// p = z + beta p
__global__ void k_pcg_pupdate(float* __restrict__ p, const float* __restrict__ z, uint32_t n, PcgScalars* sc) {
  if (sc->done) return;
  const float beta = (float)sc->beta;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = fmaf(beta, p[i], z[i]);
}

// z = Binv r (block Jacobi) with partial r.z
template <class Acc>
__global__ void k_bj_apply(const float* __restrict__ inv, const float* __restrict__ r, float* __restrict__ z,
                           uint32_t nb, DotSink d, int with_dot) {
  if (with_dot && d.sc->done) return;
  Acc acc = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nb; v += gridDim.x * blockDim.x) {
    const float* m = inv + 9 * (size_t)v;
    float r0 = r[3 * v], r1 = r[3 * v + 1], r2 = r[3 * v + 2];
    float z0 = m[0] * r0 + m[1] * r1 + m[2] * r2;
    float z1 = m[3] * r0 + m[4] * r1 + m[5] * r2;
    float z2 = m[6] * r0 + m[7] * r1 + m[8] * r2;
    z[3 * v] = z0;
    z[3 * v + 1] = z1;
    z[3 * v + 2] = z2;
    acc += (Acc)r0 * (Acc)z0 + (Acc)r1 * (Acc)z1 + (Acc)r2 * (Acc)z2;
  }
  if (with_dot) grid_dot_commit<Acc>(d, acc);
}

static int vec_grid(uint32_t n, int threads, int sms) {
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, threads), (uint64_t)sms * 8));
}

static int precond_apply(mguso_linear_solver* s, const float* r, float* z, cudaStream_t st, const DotSink* d) {
  if (s->precond == MGUSO_PRECOND_SCHWARZ) return schwarz_apply(s->schwarz.get(), r, z, st, d);
  uint32_t nb = s->bsr->nb;
  int grid = vec_grid(nb, 256, s->ctx->sm_count);
  DotSink dd = d ? *d : DotSink{};
  if (d && d->mixed)
    k_bj_apply<double><<<grid, 256, 0, st>>>(s->bjinv.p, r, z, nb, dd, d ? 1 : 0);
  else
    k_bj_apply<float><<<grid, 256, 0, st>>>(s->bjinv.p, r, z, nb, dd, d ? 1 : 0);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int pcg_solve(mguso_linear_solver* s, float tol, uint32_t max_iter, mguso_lin_stats* out) {
  cudaStream_t st = s->ctx->stream;
  mguso_bsr* a = s->bsr.get();
  const uint32_t n = 3 * a->nb;
  const bool mixed = s->precision == MGUSO_PRECISION_MIXED;
  const int sms = s->ctx->sm_count;
  if (!s->h_sc) MG_CUDA(cudaMallocHost((void**)&s->h_sc, sizeof(PcgScalars)));
  MG_TRY(s->sc.reserve(1));
  MG_TRY(s->partials.reserve(MAX_PARTIALS));
  MG_TRY(s->x.reserve(n));
  MG_TRY(s->r.reserve(n));
  MG_TRY(s->z.reserve(n));
  MG_TRY(s->p.reserve(n));
  MG_TRY(s->ap.reserve(n));
  PcgScalars h{};
  h.tol = tol;
  h.max_iter = max_iter;
  MG_CUDA(cudaMemcpyAsync(s->sc.p, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  auto sink = [&](int fin) { return DotSink{s->sc.p, s->partials.p, fin, mixed}; };
  const int vg = vec_grid(n, 256, sms);

  DotSink d0 = sink(FIN_BNORM);
  if (mixed)
    k_pcg_init<double><<<vg, 256, 0, st>>>(s->b.p, s->x.p, s->r.p, n, d0);
  else
    k_pcg_init<float><<<vg, 256, 0, st>>>(s->b.p, s->x.p, s->r.p, n, d0);
  MG_CUDA(cudaGetLastError());
  DotSink d1 = sink(FIN_RZ0);
  MG_TRY(precond_apply(s, s->r.p, s->z.p, st, &d1));
  DotSink d2 = sink(FIN_RR0);
  if (mixed)
    k_copy_dot<double><<<vg, 256, 0, st>>>(s->z.p, s->p.p, s->r.p, n, d2);
  else
    k_copy_dot<float><<<vg, 256, 0, st>>>(s->z.p, s->p.p, s->r.p, n, d2);
  MG_CUDA(cudaGetLastError());

  const uint32_t CHECK = 16;
  DotSink dp = sink(FIN_PAP), dr = sink(FIN_RR), dz = sink(FIN_RZ);
  auto one_iter = [&]() -> int {
    MG_TRY(bsr_spmv(a, s->p.p, s->ap.p, st, &dp));
    if (mixed)
      k_pcg_update<double><<<vg, 256, 0, st>>>(s->x.p, s->r.p, s->p.p, s->ap.p, n, dr);
    else
      k_pcg_update<float><<<vg, 256, 0, st>>>(s->x.p, s->r.p, s->p.p, s->ap.p, n, dr);
    MG_CUDA(cudaGetLastError());
    MG_TRY(precond_apply(s, s->r.p, s->z.p, st, &dz));
    k_pcg_pupdate<<<vg, 256, 0, st>>>(s->p.p, s->z.p, n, s->sc.p);
    MG_CUDA(cudaGetLastError());
    return MGUSO_OK;
  };
  // Capture CHECK iterations once as a graph; replay until the done flag is set.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = max_iter > CHECK;
  if (use_graph) {
    MG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = MGUSO_OK;
    for (uint32_t i = 0; i < CHECK && rc == MGUSO_OK; ++i) rc = one_iter();
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc != MGUSO_OK) return rc;
    MG_CUDA(e);
    MG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  }
  uint32_t launched = 0;
  int rc = MGUSO_OK;
  while (launched < max_iter) {
    if (use_graph && max_iter - launched >= CHECK) {
      cudaError_t e = cudaGraphLaunch(exec, st);
      if (e != cudaSuccess) {
        set_error(std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
        rc = MGUSO_ERR_CUDA;
        break;
      }
      launched += CHECK;
    } else {
      uint32_t k = std::min<uint32_t>(CHECK, max_iter - launched);
      for (uint32_t i = 0; i < k && rc == MGUSO_OK; ++i) rc = one_iter();
      if (rc != MGUSO_OK) break;
      launched += k;
    }
    cudaError_t e = cudaMemcpyAsync(s->h_sc, s->sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      set_error(std::string("pcg sync: ") + cudaGetErrorString(e));
      rc = MGUSO_ERR_CUDA;
      break;
    }
    if (s->h_sc->done) break;
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (rc != MGUSO_OK) return rc;
  MG_CUDA(cudaMemcpyAsync(s->h_sc, s->sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  if (out) {
    out->iters = s->h_sc->iters;
    out->residual = s->h_sc->residual;
    out->status = (s->h_sc->residual <= tol) ? MGUSO_OK : MGUSO_ERR_PCG_CAP;
    if (s->h_sc->status & ST_PCG_BREAKDOWN) out->status = MGUSO_OK;
  }
  return MGUSO_OK;
}

}  // namespace mg
