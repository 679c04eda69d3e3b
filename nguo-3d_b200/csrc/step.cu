// Newton driver of one implicit step on the GPU (ImplicitSolver::step, implicit.rs:1951-2191).
//
// Per Newton iteration: LBVHs over the iterate, active stencils, assembly (elastic gather,
// colliders, contact), the preconditioner factorisation, the device PCG, the uniform
// max_dx rescale, the CCD step fraction, x += t dx and the termination tests. The host
// reads back only the scalars the control flow needs (stencil count, CCD fractions,
// step length).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <chrono>

#include "elements.cuh"
#include "reduce.cuh"
#include "scene.cuh"

namespace mg {

__global__ void k_predict(const float* __restrict__ x0, const float* __restrict__ v, const float* __restrict__ im,
                          uint32_t nv, float h, float gx, float gy, float gz, float* __restrict__ xt) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  float g[3] = {gx, gy, gz};
  for (int c = 0; c < 3; ++c) {
    float p = x0[3 * i + c];
    xt[3 * i + c] = im[i] > 0.f ? p + v[3 * i + c] * h + g[c] * (h * h) : p;
  }
}

__global__ void k_scale_copy(const float* __restrict__ in, float s, uint32_t n, float* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = s == 1.f ? in[i] : in[i] * s;
}

// x += t dx, red[0] = max |t dx_i| (float bits)
__global__ void k_advance(float* __restrict__ x, const float* __restrict__ dx, float t, uint32_t nv,
                          unsigned int* __restrict__ red) {
  float m = 0.f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    float d0 = dx[3 * i] * t, d1 = dx[3 * i + 1] * t, d2 = dx[3 * i + 2] * t;
    x[3 * i] += d0;
    x[3 * i + 1] += d1;
    x[3 * i + 2] += d2;
    m = fmaxf(m, sqrtf(d0 * d0 + d1 * d1 + d2 * d2));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(red, __float_as_uint(m));
}

// floor projection, finiteness, velocity update and commit (implicit.rs:2032-2070);
// red[1] counts non-finite components (computed before the commit pass).
__global__ void k_check_finite(float* __restrict__ x, const float* __restrict__ im, uint32_t nv, float floor_y,
                               unsigned int* __restrict__ red) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  if (im[i] > 0.f && isfinite(floor_y) && x[3 * i + 1] < floor_y) x[3 * i + 1] = floor_y;
  bool f = isfinite(x[3 * i]) && isfinite(x[3 * i + 1]) && isfinite(x[3 * i + 2]);
  if (!f) atomicAdd(red + 1, 1u);
}

__global__ void k_commit(float* __restrict__ x, const float* __restrict__ x0, float* __restrict__ v,
                         const float* __restrict__ im, uint32_t nv, float inv_h, const unsigned int* __restrict__ red) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  bool finite = red[1] == 0u;
  for (int c = 0; c < 3; ++c) {
    if (finite) {
      v[3 * i + c] = im[i] > 0.f ? (x[3 * i + c] - x0[3 * i + c]) * inv_h : 0.f;
    } else {
      v[3 * i + c] = 0.f;
      x[3 * i + c] = x0[3 * i + c];
    }
  }
}

// count_active_contacts / penetration_free for analytic colliders (implicit.rs:2213-2268)
__global__ void k_collider_metrics(const float* __restrict__ x, const float* __restrict__ im, uint32_t nv,
                                   const float* __restrict__ cols, uint32_t ncol, float dhat,
                                   unsigned int* __restrict__ red) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv || !(im[i] > 0.f)) return;
  V3<float> xi = ld3<float>(x, i);
  float tol = -1.0e-3f * fmaxf(dhat, 1.0e-6f);
  bool contact = false, pen = false;
  for (uint32_t c = 0; c < ncol; ++c) {
    const float* cc = cols + 8 * c;
    V3<float> a(cc[1], cc[2], cc[3]);
    float d;
    if (cc[0] == 0.f) {
      d = (xi - a).dot(V3<float>(cc[4], cc[5], cc[6]));
    } else {
      float l = (xi - a).length();
      d = l < 1e-9f ? -cc[7] : l - cc[7];
    }
    if (d < dhat) contact = true;
    if (d < tol) pen = true;
  }
  if (contact) atomicAdd(red + 2, 1u);
  if (pen) atomicAdd(red + 3, 1u);
}

__global__ void k_max_norm(const float* __restrict__ dx, uint32_t nv, unsigned int* __restrict__ out);
int schwarz_factor_with(mguso_schwarz* s, const uint32_t* c_rp, const uint32_t* c_col, const float* c_val,
                        cudaStream_t st);

static int linear_solve(Scene& s, mguso_lin_stats* ls) {
  cudaStream_t st = s.st;
  if (s.schwarz) {
    MG_TRY(schwarz_factor_with(s.schwarz.get(), s.c_row_ptr.p, s.c_col.p, s.c_val.p, st));
  } else {
    MG_TRY(blockjacobi_factor(s.A.get(), s.bjinv.p, st));
  }
  if (s.p.pcg_mode == 0) {
    const uint32_t rows[2] = {0, s.nv};
    PcgInstResult r{};
    int rc = pcg_persistent(s, rows, 1, &r);
    if (rc == MGUSO_OK) {
      ls->iters = r.iters;
      ls->residual = r.residual;
      ls->status = (r.residual <= s.p.cg_tol || (r.status & ST_PCG_BREAKDOWN)) ? MGUSO_OK : MGUSO_ERR_PCG_CAP;
      return MGUSO_OK;
    }
    if (rc != MGUSO_ERR_UNSUPPORTED) return rc;
  }
  PcgOps ops;
  ops.stream = st;
  ops.mixed = s.mixed;
  ops.sms = s.ctx->sm_count;
  ops.key = (uint64_t)(uintptr_t)&s ^ ((uint64_t)(uintptr_t)s.c_col.p << 3) ^ ((uint64_t)(uintptr_t)s.c_val.p << 7);
  Scene* sp = &s;
  ops.spmv = [sp](const float* p, float* ap, cudaStream_t stream, const DotSink* d) {
    return system_spmv(*sp, p, ap, stream, d);
  };
  if (s.schwarz) {
    mguso_schwarz* sw = s.schwarz.get();
    ops.precond = [sw](const float* r, float* z, cudaStream_t stream, const DotSink* d) {
      return schwarz_apply(sw, r, z, stream, d);
    };
  } else {
    const float* inv = s.bjinv.p;
    uint32_t nb = s.nv;
    int sms = ops.sms;
    ops.precond = [inv, nb, sms](const float* r, float* z, cudaStream_t stream, const DotSink* d) {
      return bj_apply(inv, r, z, nb, sms, stream, d);
    };
  }
  return pcg_run(ops, s.work, s.p.cg_tol, s.p.cg_max_iter, ls);
}

int scene_step(Scene& s, mguso_step_stats* out) {
  cudaStream_t st = s.st;
  const uint32_t nv = s.nv, n3 = 3 * nv;
  const float h = s.p.dt;
  mguso_step_stats stats{};
  stats.t_min = 1.0;
  MG_CUDA(cudaMemcpyAsync(s.x0.p, s.x.p, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
  k_predict<<<ceil_div(nv, 256), 256, 0, st>>>(s.x0.p, s.v.p, s.inv_mass.p, nv, h, s.p.gravity[0], s.p.gravity[1],
                                               s.p.gravity[2], s.xt.p);
  MG_CUDA(cudaGetLastError());
  const uint32_t cap = std::max<uint32_t>(s.p.newton_iters, 1);
  bool final_step = false;
  uint32_t taken = 0;
  const int sms = s.ctx->sm_count;
  const bool contacts = s.p.self_collision != 0;
  // MGUSO_TRACE=1 prints one line per Newton iteration to stderr (diagnostics only)
  static const bool trace = std::getenv("MGUSO_TRACE") != nullptr;
  // with MGUSO_TRACE=2 the stream is drained at each phase boundary and the host time of
  // the phases is printed too (stencils, assembly, linear solve, CCD + advance), in ms
  static const bool trace_phases = trace && std::getenv("MGUSO_TRACE")[0] == '2';
  double ph[5] = {0, 0, 0, 0, 0};
  auto mark = [&]() -> double {
    if (!trace_phases) return 0.0;
    cudaStreamSynchronize(st);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  for (uint32_t it = 0; it < cap; ++it) {
    ++taken;
    uint32_t nst = 0;
    ph[0] = mark();
    if (contacts) {
      MG_TRY(build_bvhs(s, s.x.p));
      MG_TRY(collect_stencils(s, &nst));
    }
    ph[1] = mark();
    stats.stencils = std::max(stats.stencils, nst);
    MG_TRY(assemble_elastic(s));
    MG_TRY(assemble_colliders(s));
    MG_TRY(assemble_contacts(s, nst));
    MG_TRY(finish_rhs(s));
    ph[2] = mark();
    mguso_lin_stats ls{};
    MG_TRY(linear_solve(s, &ls));
    ph[3] = mark();
    stats.max_reresid = std::max(stats.max_reresid, ls.residual);
    stats.max_cg_iters = std::max(stats.max_cg_iters, ls.iters);
    // uniform max_dx rescale (implicit.rs:1996-2004); INFINITY leaves dx unchanged
    float rescale = 1.f;
    if (std::isfinite(s.p.max_dx)) {
      unsigned int zero = 0;
      MG_CUDA(cudaMemcpyAsync(s.red.p + 8, &zero, 4, cudaMemcpyHostToDevice, st));
      k_max_norm<<<std::min<uint32_t>(ceil_div(nv, 256), sms * 4), 256, 0, st>>>(s.work.x.p, nv, s.red.p + 8);
      unsigned int mb = 0;
      MG_CUDA(cudaMemcpyAsync(&mb, s.red.p + 8, 4, cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaStreamSynchronize(st));
      float max_norm = u2f_host(mb);
      if (max_norm > 0.f) rescale = std::min(s.p.max_dx / max_norm, 1.0f);
    }
    k_scale_copy<<<ceil_div(n3, 256), 256, 0, st>>>(s.work.x.p, rescale < 1.f ? rescale : 1.f, n3, s.dx.p);
    MG_CUDA(cudaGetLastError());
    float t = 1.f;
    uint32_t caps = 0;
    MG_TRY(ccd_step(s, &t, &caps));
    stats.ccd_cap_hits += caps;
    stats.t_min = std::min(stats.t_min, (double)t);
    unsigned int zero = 0;
    MG_CUDA(cudaMemcpyAsync(s.red.p + 9, &zero, 4, cudaMemcpyHostToDevice, st));
    k_advance<<<std::min<uint32_t>(ceil_div(nv, 256), sms * 4), 256, 0, st>>>(s.x.p, s.dx.p, t, nv, s.red.p + 9);
    unsigned int msb = 0;
    MG_CUDA(cudaMemcpyAsync(&msb, s.red.p + 9, 4, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    float max_step = u2f_host(msb);
    if (trace)
      std::fprintf(stderr, "[mguso] newton %u stencils %u cg %u res %.3e lin_status %d t %.4f max_step %.3e\n", it,
                   nst, ls.iters, ls.residual, ls.status, t, max_step);
    if (trace_phases) {
      ph[4] = mark();
      std::fprintf(stderr, "[mguso]   ms: stencils %.3f assembly %.3f solve %.3f ccd+advance %.3f\n", ph[1] - ph[0],
                   ph[2] - ph[1], ph[3] - ph[2], ph[4] - ph[3]);
    }
    if (max_step < 1.0e-7f) break;
    if (s.p.newton_tol > 0.f && max_step < s.p.newton_tol) break;
    if (final_step) break;
    if (s.p.target_toi > 0.f && t >= s.p.target_toi && taken > s.p.min_newton_steps) final_step = true;
  }
  unsigned int zeros[4] = {0, 0, 0, 0};
  MG_CUDA(cudaMemcpyAsync(s.red.p + 10, zeros, 16, cudaMemcpyHostToDevice, st));
  k_check_finite<<<ceil_div(nv, 256), 256, 0, st>>>(s.x.p, s.inv_mass.p, nv, s.p.floor_y, s.red.p + 10);
  k_commit<<<ceil_div(nv, 256), 256, 0, st>>>(s.x.p, s.x0.p, s.v.p, s.inv_mass.p, nv, 1.0f / h, s.red.p + 10);
  if (s.n_col)
    k_collider_metrics<<<ceil_div(nv, 256), 256, 0, st>>>(s.x.p, s.inv_mass.p, nv, s.colliders.p, s.n_col,
                                                          s.p.contact_dhat, s.red.p + 10);
  MG_CUDA(cudaGetLastError());
  unsigned int m[4];
  MG_CUDA(cudaMemcpyAsync(m, s.red.p + 10, 16, cudaMemcpyDeviceToHost, st));
  uint32_t dev_status = 0;
  MG_CUDA(cudaMemcpyAsync(&dev_status, s.status.p, 4, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  s.time += (double)h;
  stats.newton_iters = taken;
  stats.all_finite = m[1] == 0 ? 1 : 0;
  stats.num_contacts = m[2];
  stats.penetration_free = (m[1] == 0 && m[3] == 0) ? 1 : 0;
  stats.status = m[1] ? MGUSO_ERR_NONFINITE : MGUSO_OK;
  if (dev_status & ST_STACK_OVERFLOW) stats.status = MGUSO_ERR_BVH_STACK;
  if (dev_status & ST_WAIT_TIMEOUT) stats.status = MGUSO_ERR_TIMEOUT;
  if (stats.ccd_cap_hits && stats.status == MGUSO_OK) stats.status = MGUSO_OK;  // reported, not fatal (reference)
  MG_CUDA(cudaMemsetAsync(s.status.p, 0, 4, st));
  s.history.push_back(stats);
  if (out) *out = stats;
  return MGUSO_OK;
}

}  // namespace mg
