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

// dx = s_k * x on instance k's rows; with red given, s_k = min(max_dx / |x|_max, 1) from
// instance k's largest vertex norm red[RED_STRIDE k] (float bits; 0 leaves x alone), the
// uniform max_dx rescale of implicit.rs:1996-2004 decided on the device
__global__ void k_scale_copy(const float* __restrict__ in, const unsigned int* __restrict__ red, float max_dx,
                             const uint8_t* __restrict__ vinst, uint32_t n, float* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 1.f;
  if (red) {
    const float m = __uint_as_float(red[RED_STRIDE * vinst[i / 3]]);
    if (m > 0.f) s = fminf(max_dx / m, 1.0f);
  }
  out[i] = s == 1.f ? in[i] : in[i] * s;
}

// x += t_k dx on instance k's vertices, t the CCD's device array of step fractions (0 for
// inactive instances); red[RED_STRIDE k + 9] = max |t dx_i| (float bits)
__global__ void k_advance(float* __restrict__ x, const float* __restrict__ dx, const float* __restrict__ t,
                          const uint8_t* __restrict__ vinst, uint32_t nv, unsigned int* __restrict__ red) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const uint32_t k = vinst[i];
    const float tk = t[k];
    if (tk == 0.f) continue;
    float d0 = dx[3 * i] * tk, d1 = dx[3 * i + 1] * tk, d2 = dx[3 * i + 2] * tk;
    x[3 * i] += d0;
    x[3 * i + 1] += d1;
    x[3 * i + 2] += d2;
    const float m = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
    if (m > 0.f) atomicMax(red + RED_STRIDE * k + 9, __float_as_uint(m));
  }
}

// floor projection, finiteness, velocity update and commit (implicit.rs:2032-2070), per
// instance: red[RED_STRIDE k + 11] counts instance k's non-finite vertices (computed before
// the commit pass), + 12 its collider contacts, + 13 its collider penetrations.
__global__ void k_check_finite(float* __restrict__ x, const float* __restrict__ im, const uint8_t* __restrict__ vinst,
                               uint32_t nv, float floor_y, unsigned int* __restrict__ red) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  if (im[i] > 0.f && isfinite(floor_y) && x[3 * i + 1] < floor_y) x[3 * i + 1] = floor_y;
  bool f = isfinite(x[3 * i]) && isfinite(x[3 * i + 1]) && isfinite(x[3 * i + 2]);
  if (!f) atomicAdd(red + RED_STRIDE * vinst[i] + 11, 1u);
}

__global__ void k_commit(float* __restrict__ x, const float* __restrict__ x0, float* __restrict__ v,
                         const float* __restrict__ im, const uint8_t* __restrict__ vinst, uint32_t nv, float inv_h,
                         const unsigned int* __restrict__ red) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  bool finite = red[RED_STRIDE * vinst[i] + 11] == 0u;
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
__global__ void k_collider_metrics(const float* __restrict__ x, const float* __restrict__ im,
                                   const uint8_t* __restrict__ vinst, uint32_t nv, const float* __restrict__ cols,
                                   uint32_t ncol, float dhat, unsigned int* __restrict__ red) {
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
  unsigned int* r = red + RED_STRIDE * vinst[i];
  if (contact) atomicAdd(r + 12, 1u);
  if (pen) atomicAdd(r + 13, 1u);
}

__global__ void k_max_norm(const float* __restrict__ dx, const uint8_t* __restrict__ vinst, uint32_t nv,
                           unsigned int* __restrict__ out);
int schwarz_factor_with(mguso_schwarz* s, const uint32_t* c_rp, const uint32_t* c_col, const float* c_val,
                        cudaStream_t st);

static void fused_stats(const Scene& s, const PcgInstResult* r, mguso_lin_stats* ls) {
  for (uint32_t k = 0; k < s.ninst; ++k) {
    ls[k].iters = r[k].iters;
    ls[k].residual = r[k].residual;
    ls[k].status = (r[k].residual <= s.p.cg_tol || (r[k].status & ST_PCG_BREAKDOWN)) ? MGUSO_OK : MGUSO_ERR_PCG_CAP;
  }
}

// Factorises the preconditioner and solves every instance in `active` (the others get
// dx = 0); ls[k] = instance k's PCG statistics. With `deferred` given, the fused PCG leaves
// its statistics to be read after the caller's next stream synchronisation
// (pcg_fused_results) and sets *deferred; ls is then not written.
static int linear_solve(Scene& s, uint32_t active, mguso_lin_stats* ls, bool* deferred = nullptr) {
  cudaStream_t st = s.st;
  if (s.schwarz) {
    // only the instances still iterating need their domains factored
    s.schwarz->active = active;
    const int rc = schwarz_factor_with(s.schwarz.get(), s.c_row_ptr.p, s.c_col.p, s.c_val.p, st);
    s.schwarz->active = 0xffffffffu;
    MG_TRY(rc);
  } else {
    MG_TRY(blockjacobi_factor(s.A.get(), s.bjinv.p, st));
  }
  const bool two_level = s.schwarz && s.schwarz->levels == 2;
  if (!two_level && (s.p.pcg_mode == 0 || s.p.pcg_mode == 2 || s.ninst > 1)) {
    PcgInstResult r[PCG_MAX_INST] = {};
    if (s.p.pcg_mode != 2) MG_TRY(pcg_fused_select(s));
    const bool defer = deferred && s.p.pcg_mode != 2;
    int rc = s.p.pcg_mode == 2 ? pcg_persistent(s, s.inst_vert.data(), s.ninst, active, r)
                               : pcg_fused(s, s.inst_vert.data(), s.ninst, active, defer ? nullptr : r);
    if (rc == MGUSO_OK) {
      if (defer)
        *deferred = true;
      else
        fused_stats(s, r, ls);
      return MGUSO_OK;
    }
    if (rc != MGUSO_ERR_UNSUPPORTED) return rc;
    if (s.ninst > 1) {
      set_error("batched step: the persistent PCG cannot run on this device");
      return MGUSO_ERR_UNSUPPORTED;
    }
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

// One implicit step of every instance; out[k] = instance k's statistics. Each instance runs
// its own Newton loop (termination, CCD step fraction, iteration count); the instances that
// are still iterating share the launches of an iteration.
int scene_step(Scene& s, mguso_step_stats* out) {
  cudaStream_t st = s.st;
  const uint32_t nv = s.nv, n3 = 3 * nv, K = s.ninst;
  const float h = s.p.dt;
  mguso_step_stats stats[PCG_MAX_INST] = {};
  for (uint32_t k = 0; k < K; ++k) stats[k].t_min = 1.0;
  MG_CUDA(cudaMemcpyAsync(s.x0.p, s.x.p, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
  k_predict<<<ceil_div(nv, 256), 256, 0, st>>>(s.x0.p, s.v.p, s.inv_mass.p, nv, h, s.p.gravity[0], s.p.gravity[1],
                                               s.p.gravity[2], s.xt.p);
  MG_CUDA(cudaGetLastError());
  const uint32_t cap = std::max<uint32_t>(s.p.newton_iters, 1);
  bool final_step[PCG_MAX_INST] = {};
  uint32_t active = (K >= 32) ? ~0u : ((1u << K) - 1u);
  const int sms = s.ctx->sm_count;
  const bool contacts = s.p.self_collision != 0;
  // MGUSO_TRACE=1 prints one line per Newton iteration to stderr (diagnostics only); with
  // MGUSO_TRACE=2 the stream is drained at each phase boundary and the host time of the
  // phases is printed too (stencils, assembly, linear solve, CCD + advance), in ms
  static const bool trace = std::getenv("MGUSO_TRACE") != nullptr;
  static const bool trace_phases = trace && std::getenv("MGUSO_TRACE")[0] == '2';
  double ph[5] = {0, 0, 0, 0, 0};
  auto mark = [&]() -> double {
    if (!trace_phases) return 0.0;
    cudaStreamSynchronize(st);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  std::vector<unsigned int> hred(RED_STRIDE * K);
  // the instances each Newton iteration works on; every exit restores "all"
  struct ActiveGuard {
    Scene& s;
    ~ActiveGuard() { s.iter_active = 0xffffffffu; }
  } active_guard{s};
  for (uint32_t it = 0; it < cap && active; ++it) {
    s.iter_active = active;
    for (uint32_t k = 0; k < K; ++k)
      if ((active >> k) & 1u) stats[k].newton_iters++;
    uint32_t nst = 0;
    ph[0] = mark();
    if (contacts) {
      // the first iterate's tree shapes serve the step's later iterations (boxes refitted)
      MG_TRY(build_bvhs(s, s.x.p, it > 0));
      MG_TRY(collect_stencils(s, &nst));
    }
    ph[1] = mark();
    MG_TRY(assemble_elastic(s));
    MG_TRY(assemble_colliders(s));
    MG_TRY(assemble_contacts(s, nst));
    MG_TRY(finish_rhs(s));
    ph[2] = mark();
    mguso_lin_stats ls[PCG_MAX_INST] = {};
    bool deferred = false;
    MG_TRY(linear_solve(s, active, ls, &deferred));
    ph[3] = mark();
    // uniform max_dx rescale per instance (implicit.rs:1996-2004); INFINITY leaves dx alone
    const bool cap_dx = std::isfinite(s.p.max_dx);
    if (cap_dx) {
      MG_CUDA(cudaMemsetAsync(s.red.p, 0, 4 * RED_STRIDE * K, st));
      k_max_norm<<<std::min<uint32_t>(ceil_div(nv, 256), sms * 4), 256, 0, st>>>(s.work.x.p, s.vinst.p, nv, s.red.p);
    }
    k_scale_copy<<<ceil_div(n3, 256), 256, 0, st>>>(s.work.x.p, cap_dx ? s.red.p : nullptr, s.p.max_dx, s.vinst.p, n3,
                                                    s.dx.p);
    MG_CUDA(cudaGetLastError());
    MG_TRY(ccd_step(s, active));
    std::vector<unsigned int> hccd;
    if (trace_phases) {  // the self-contact traversals' leaf and root-solve counts
      hccd.resize(RED_STRIDE * K);
      MG_CUDA(cudaMemcpyAsync(hccd.data(), s.red.p, 4 * hccd.size(), cudaMemcpyDeviceToHost, st));
    }
    MG_CUDA(cudaMemsetAsync(s.red.p, 0, 4 * RED_STRIDE * K, st));
    k_advance<<<std::min<uint32_t>(ceil_div(nv, 256), sms * 4), 256, 0, st>>>(s.x.p, s.dx.p, ccd_t(s), s.vinst.p, nv,
                                                                             s.red.p);
    MG_CUDA(cudaMemcpyAsync(hred.data(), s.red.p, 4 * hred.size(), cudaMemcpyDeviceToHost, st));
    // the iteration's one wait: its step lengths, with the CCD's and the PCG's results
    float t[PCG_MAX_INST];
    uint32_t caps[PCG_MAX_INST];
    MG_TRY(ccd_results(s, t, caps));
    for (uint32_t k = 0; k < K; ++k) {
      if (!((active >> k) & 1u)) continue;
      stats[k].ccd_cap_hits += caps[k];
      stats[k].t_min = std::min(stats[k].t_min, (double)t[k]);
    }
    if (deferred) {  // the stream has passed the PCG's result copy
      PcgInstResult r[PCG_MAX_INST] = {};
      MG_TRY(pcg_fused_results(s, K, r));
      fused_stats(s, r, ls);
    }
    for (uint32_t k = 0; k < K; ++k) {
      if (!((active >> k) & 1u)) continue;
      stats[k].stencils = std::max(stats[k].stencils, nst);
      stats[k].max_reresid = std::max(stats[k].max_reresid, ls[k].residual);
      stats[k].max_cg_iters = std::max(stats[k].max_cg_iters, ls[k].iters);
    }
    for (uint32_t k = 0; k < K; ++k) {
      if (!((active >> k) & 1u)) continue;
      const float max_step = u2f_host(hred[RED_STRIDE * k + 9]);
      if (trace)
        std::fprintf(stderr, "[mguso] inst %u newton %u stencils %u cg %u res %.3e lin_status %d t %.4f max_step %.3e\n",
                     k, it, nst, ls[k].iters, ls[k].residual, ls[k].status, t[k], max_step);
      bool stop = max_step < 1.0e-7f || (s.p.newton_tol > 0.f && max_step < s.p.newton_tol) || final_step[k];
      if (!stop && s.p.target_toi > 0.f && t[k] >= s.p.target_toi && stats[k].newton_iters > s.p.min_newton_steps)
        final_step[k] = true;
      if (stop) active &= ~(1u << k);
    }
    if (trace_phases) {
      ph[4] = mark();
      std::fprintf(stderr, "[mguso]   ms: stencils %.3f assembly %.3f solve %.3f ccd+advance %.3f\n", ph[1] - ph[0],
                   ph[2] - ph[1], ph[3] - ph[2], ph[4] - ph[3]);
      unsigned long long c[5] = {0, 0, 0, 0, 0};
      for (uint32_t k = 0; k < K; ++k) {
        for (int q = 0; q < 4; ++q) c[q] += hccd[RED_STRIDE * k + 5 + q];
        c[4] += caps[k];
      }
      std::fprintf(stderr,
                   "[mguso]   ccd: launches %u vt leaves %llu solves %llu ee leaves %llu solves %llu caps %llu\n",
                   ccd_launches(s), c[0], c[1], c[2], c[3], c[4]);
    }
  }
  s.iter_active = 0xffffffffu;
  MG_CUDA(cudaMemsetAsync(s.red.p, 0, 4 * RED_STRIDE * K, st));
  k_check_finite<<<ceil_div(nv, 256), 256, 0, st>>>(s.x.p, s.inv_mass.p, s.vinst.p, nv, s.p.floor_y, s.red.p);
  k_commit<<<ceil_div(nv, 256), 256, 0, st>>>(s.x.p, s.x0.p, s.v.p, s.inv_mass.p, s.vinst.p, nv, 1.0f / h, s.red.p);
  if (s.n_col)
    k_collider_metrics<<<ceil_div(nv, 256), 256, 0, st>>>(s.x.p, s.inv_mass.p, s.vinst.p, nv, s.colliders.p, s.n_col,
                                                          s.p.contact_dhat, s.red.p);
  MG_CUDA(cudaGetLastError());
  // the self-intersection scan of penetration_free (implicit.rs:2250-2258), with self
  // collision on, at the committed positions (over the triangle trees built in this step)
  if (contacts) MG_TRY(self_intersections(s, true));
  MG_CUDA(cudaMemcpyAsync(hred.data(), s.red.p, 4 * hred.size(), cudaMemcpyDeviceToHost, st));
  uint32_t dev_status = 0;
  MG_CUDA(cudaMemcpyAsync(&dev_status, s.status.p, 4, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  s.time += (double)h;
  for (uint32_t k = 0; k < K; ++k) {
    const unsigned int* m = hred.data() + RED_STRIDE * k;
    mguso_step_stats& o = stats[k];
    o.all_finite = m[11] == 0 ? 1 : 0;
    o.num_contacts = m[12];
    o.penetration_free = (m[11] == 0 && m[13] == 0 && m[14] == 0) ? 1 : 0;
    o.status = m[11] ? MGUSO_ERR_NONFINITE : MGUSO_OK;
    if (dev_status & ST_STACK_OVERFLOW) o.status = MGUSO_ERR_BVH_STACK;
    if (dev_status & ST_WAIT_TIMEOUT) o.status = MGUSO_ERR_TIMEOUT;
    // CCD cap hits are reported, not fatal (reference)
    s.history.push_back(o);
    if (out) out[k] = o;
  }
  MG_CUDA(cudaMemsetAsync(s.status.p, 0, 4, st));
  // the collider move described this step only (implicit.rs:2065-2070)
  s.kin_dx_set = false;
  return MGUSO_OK;
}

}  // namespace mg
