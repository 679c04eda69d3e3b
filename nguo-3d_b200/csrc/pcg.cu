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
// the host replays a CUDA graph of CHECK iterations between reads of the done flag; the
// graph is captured once per operator and kept until its buffers change.
#include <algorithm>
#include <cstring>

#include "pcg.cuh"
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

int vec_grid(uint32_t n, int threads, int sms) {
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n, threads), (uint64_t)sms * 8));
}

int bj_apply(const float* inv, const float* r, float* z, uint32_t nb, int sms, cudaStream_t st, const DotSink* d) {
  int grid = vec_grid(nb, 256, sms);
  DotSink dd = d ? *d : DotSink{};
  if (d && d->mixed)
    k_bj_apply<double><<<grid, 256, 0, st>>>(inv, r, z, nb, dd, d ? 1 : 0);
  else
    k_bj_apply<float><<<grid, 256, 0, st>>>(inv, r, z, nb, dd, d ? 1 : 0);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// One x/r update with its fused r.r into PcgScalars::out (used to time the kernel alone;
// the scalar block must not be marked done).
int pcg_vector_update(PcgWork& w, bool mixed, int sms, cudaStream_t st) {
  DotSink d{w.sc.p, w.partials.p, FIN_STORE, mixed};
  const int vg = vec_grid(w.n, 256, sms);
  if (mixed)
    k_pcg_update<double><<<vg, 256, 0, st>>>(w.x.p, w.r.p, w.p.p, w.ap.p, w.n, d);
  else
    k_pcg_update<float><<<vg, 256, 0, st>>>(w.x.p, w.r.p, w.p.p, w.ap.p, w.n, d);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int PcgWork::reserve(uint32_t n_) {
  n = n_;
  if (!h_sc) MG_CUDA(cudaMallocHost((void**)&h_sc, sizeof(PcgScalars)));
  size_t before = (size_t)b.p + (size_t)x.p + (size_t)r.p + (size_t)z.p + (size_t)p.p + (size_t)ap.p;
  MG_TRY(sc.reserve(1));
  MG_TRY(partials.reserve(MAX_PARTIALS));
  MG_TRY(b.reserve(n));
  MG_TRY(x.reserve(n));
  MG_TRY(r.reserve(n));
  // z and the directions have room for 4 floats per vertex (the fused PCG's padded layout)
  MG_TRY(z.reserve(4 * ((size_t)n / 3 + 1)));
  MG_TRY(p.reserve(4 * ((size_t)n / 3 + 1)));
  MG_TRY(ap.reserve(n));
  size_t after = (size_t)b.p + (size_t)x.p + (size_t)r.p + (size_t)z.p + (size_t)p.p + (size_t)ap.p;
  if (before != after) drop_graph();
  return MGUSO_OK;
}

void PcgWork::drop_graph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
}

PcgWork::~PcgWork() {
  drop_graph();
  if (h_sc) cudaFreeHost(h_sc);
}

int pcg_run(const PcgOps& ops, PcgWork& w, float tol, uint32_t max_iter, mguso_lin_stats* out) {
  cudaStream_t st = ops.stream;
  const uint32_t n = w.n;
  const bool mixed = ops.mixed;
  const int sms = ops.sms;
  PcgScalars h{};
  h.tol = tol;
  h.max_iter = max_iter;
  MG_CUDA(cudaMemcpyAsync(w.sc.p, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  auto sink = [&](int fin) { return DotSink{w.sc.p, w.partials.p, fin, mixed}; };
  const int vg = vec_grid(n, 256, sms);

  DotSink d0 = sink(FIN_BNORM);
  if (mixed)
    k_pcg_init<double><<<vg, 256, 0, st>>>(w.b.p, w.x.p, w.r.p, n, d0);
  else
    k_pcg_init<float><<<vg, 256, 0, st>>>(w.b.p, w.x.p, w.r.p, n, d0);
  MG_CUDA(cudaGetLastError());
  DotSink d1 = sink(FIN_RZ0);
  MG_TRY(ops.precond(w.r.p, w.z.p, st, &d1));
  DotSink d2 = sink(FIN_RR0);
  if (mixed)
    k_copy_dot<double><<<vg, 256, 0, st>>>(w.z.p, w.p.p, w.r.p, n, d2);
  else
    k_copy_dot<float><<<vg, 256, 0, st>>>(w.z.p, w.p.p, w.r.p, n, d2);
  MG_CUDA(cudaGetLastError());

  const uint32_t CHECK = 16;
  DotSink dp = sink(FIN_PAP), dr = sink(FIN_RR), dz = sink(FIN_RZ);
  auto one_iter = [&]() -> int {
    MG_TRY(ops.spmv(w.p.p, w.ap.p, st, &dp));
    if (mixed)
      k_pcg_update<double><<<vg, 256, 0, st>>>(w.x.p, w.r.p, w.p.p, w.ap.p, n, dr);
    else
      k_pcg_update<float><<<vg, 256, 0, st>>>(w.x.p, w.r.p, w.p.p, w.ap.p, n, dr);
    MG_CUDA(cudaGetLastError());
    MG_TRY(ops.precond(w.r.p, w.z.p, st, &dz));
    k_pcg_pupdate<<<vg, 256, 0, st>>>(w.p.p, w.z.p, n, w.sc.p);
    MG_CUDA(cudaGetLastError());
    return MGUSO_OK;
  };
  bool use_graph = max_iter >= CHECK && ops.graphable;
  if (use_graph && (!w.exec || w.graph_key != ops.key || w.graph_mixed != mixed)) {
    w.drop_graph();
    MG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = MGUSO_OK;
    for (uint32_t i = 0; i < CHECK && rc == MGUSO_OK; ++i) rc = one_iter();
    cudaError_t e = cudaStreamEndCapture(st, &w.graph);
    if (rc != MGUSO_OK) {
      if (w.graph) cudaGraphDestroy(w.graph);
      w.graph = nullptr;
      return rc;
    }
    MG_CUDA(e);
    MG_CUDA(cudaGraphInstantiate(&w.exec, w.graph, 0));
    w.graph_key = ops.key;
    w.graph_mixed = mixed;
  }
  uint32_t launched = 0;
  while (launched < max_iter) {
    if (use_graph && max_iter - launched >= CHECK) {
      MG_CUDA(cudaGraphLaunch(w.exec, st));
      launched += CHECK;
    } else {
      uint32_t k = std::min<uint32_t>(CHECK, max_iter - launched);
      for (uint32_t i = 0; i < k; ++i) MG_TRY(one_iter());
      launched += k;
    }
    MG_CUDA(cudaMemcpyAsync(w.h_sc, w.sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    if (w.h_sc->done) break;
  }
  MG_CUDA(cudaMemcpyAsync(w.h_sc, w.sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  if (out) {
    out->iters = w.h_sc->iters;
    out->residual = w.h_sc->residual;
    out->status = (w.h_sc->residual <= tol || (w.h_sc->status & ST_PCG_BREAKDOWN)) ? MGUSO_OK : MGUSO_ERR_PCG_CAP;
  }
  return MGUSO_OK;
}

// The LinearSolver entry point's system: the solver's own BSR and preconditioner.
int pcg_solve(mguso_linear_solver* s, float tol, uint32_t max_iter, mguso_lin_stats* out) {
  mguso_bsr* a = s->bsr.get();
  MG_TRY(s->work.reserve(3 * a->nb));
  PcgOps ops;
  ops.stream = s->ctx->stream;
  ops.mixed = s->precision == MGUSO_PRECISION_MIXED;
  ops.sms = s->ctx->sm_count;
  ops.key = (uint64_t)(uintptr_t)a ^ ((uint64_t)a->val.p << 1) ^ ((uint64_t)s->precond << 60) ^ s->generation;
  ops.spmv = [a](const float* p, float* ap, cudaStream_t st, const DotSink* d) { return bsr_spmv(a, p, ap, st, d); };
  if (s->precond == MGUSO_PRECOND_SCHWARZ) {
    mguso_schwarz* sw = s->schwarz.get();
    ops.precond = [sw](const float* r, float* z, cudaStream_t st, const DotSink* d) {
      return schwarz_apply(sw, r, z, st, d);
    };
  } else {
    const float* inv = s->bjinv.p;
    uint32_t nb = a->nb;
    int sms = ops.sms;
    ops.precond = [inv, nb, sms](const float* r, float* z, cudaStream_t st, const DotSink* d) {
      return bj_apply(inv, r, z, nb, sms, st, d);
    };
  }
  return pcg_run(ops, s->work, tol, max_iter, out);
}

}  // namespace mg
