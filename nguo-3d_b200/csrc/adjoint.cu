// Adjoint of the implicit step: gradients of a loss on the final positions of an N-step drape
// with respect to sewing-pattern parameters, as a forward/backward pair.
//
// Parameters theta (npanel = 2, nseam = 2 gives 8): per-panel membrane stiffness factors,
// per-panel rest-length scales along the warp (pattern v) and the weft (pattern u), and
// per-seam stitch stiffness factors, in that order:
//   [stiff_0 .. stiff_{P-1}, warp_0, weft_0, ..., warp_{P-1}, weft_{P-1}, seam_0 .. seam_{S-1}].
// A shell face of panel p rests at its pattern triangle scaled by (weft_p, warp_p) along
// (u, v); its (shell_mu, shell_lambda) are multiplied by stiff_p; a stitch of seam q has its
// stiffness multiplied by seam_q.
//
// Each step is an equilibrium g(x_{n+1}; x_n, v_n, theta) = M/h^2 (x_{n+1} - x~) + grad Phi = 0
// with x~ = x_n + h v_n + h^2 g_ext and v_{n+1} = (x_{n+1} - x_n) / h. Backwards through a
// step, with the adjoints (a_x, a_v) of (x_{n+1}, v_{n+1}):
//   H w = a_x + a_v / h                      (H: the exact Hessian of the step at the
//                                             converged x_{n+1}, symmetric and possibly
//                                             indefinite, solved by preconditioned MINRES
//                                             with the step's own preconditioner factored
//                                             from its projected matrix)
//   dL/dtheta -= w . dg/dtheta
//   a_x(n) = M/h^2 w - a_v / h,   a_v(n) = M/h w.
// dg/dtheta: stiffness and seam factors scale their elements' forces linearly (exact, from
// the assembled element gradients); the rest-length scales use an FP64 central difference
// of each face's force in its scale, inside the kernel. States are checkpointed every
// `checkpoint_every` steps in the forward pass; the backward pass recomputes each segment
// from its checkpoint.
//
// H is the Jacobian of the step's gradient, not the step's PSD-projected Newton matrix:
// shells keep their negative eigenvalues, stitches and springs their compressive terms,
// hinges and barriers their second-derivative terms (FP64 central differences of the
// FP64 angle and gap gradients). A contact stencil's stiffness is the Rayleigh stiffness
// the step computed; its dependence on the gap (the mass part, proportional to 1/d^2)
// enters H, its dependence on the elastic blocks (a third derivative) does not. Friction
// is not differentiated (frictionless scenes only), and neither are analytic colliders'
// stiffnesses or the CCD line search: the result is the implicit-function derivative at
// converged steps.
//
// No counterpart in the reference (it has no differentiation).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "elements.cuh"
#include "scene.cuh"

namespace mg {
int bj_apply(const float* inv, const float* r, float* z, uint32_t nb, int sms, cudaStream_t st, const DotSink* d);
int schwarz_factor_with(mguso_schwarz* s, const uint32_t* c_rp, const uint32_t* c_col, const float* c_val,
                        cudaStream_t st);
__global__ void k_predict(const float* __restrict__ x0, const float* __restrict__ v, const float* __restrict__ im,
                          uint32_t nv, float h, float gx, float gy, float gz, float* __restrict__ xt);
}  // namespace mg

using namespace mg;

struct mguso_adjoint {
  mguso_ctx* ctx = nullptr;
  // the base description and its arrays
  mguso_scene_desc base{};
  std::vector<float> pos, vel, im, sw, skl0, cols;
  std::vector<uint32_t> tris, shf, sidx;
  std::vector<uint8_t> mask;
  std::vector<float> uv;  // 6 per shell face
  std::vector<uint8_t> panel, seam;
  uint32_t npanel = 0, nseam = 0;
  // the forward pass
  std::vector<double> theta;
  std::vector<float> rest, stiff, skl;
  std::unique_ptr<mguso_scene> scene;
  uint32_t nsteps = 0, every = 1;
  std::vector<std::unique_ptr<DevBuf<float>>> ck_x, ck_v;
  DevBuf<double> ax, av, c_shell, c_stitch;
  std::vector<std::unique_ptr<DevBuf<float>>> seg_x, seg_v;
  DevBuf<float> d_uv, d_scale, d_stiff;
  DevBuf<uint8_t> d_panel;
  // MINRES work vectors
  DevBuf<double> mr[9], dots;
  DevBuf<float> mf[2];
};

namespace {

// rest shape of one face from its pattern triangle scaled by (su, sv) along (u, v):
// inverse (column-major) and area, as the scene's shells store them
template <class R>
__host__ __device__ inline void pattern_rest(const float* uv6, R su, R sv, R dm[4], R* area) {
  const R xx = su * (R)(uv6[2] - uv6[0]), xy = sv * (R)(uv6[3] - uv6[1]);
  const R yx = su * (R)(uv6[4] - uv6[0]), yy = sv * (R)(uv6[5] - uv6[1]);
  const R det = xx * yy - yx * xy;
  const R inv = R(1) / det;
  dm[0] = yy * inv;
  dm[1] = -xy * inv;
  dm[2] = -yx * inv;
  dm[3] = xx * inv;
  *area = R(0.5) * (det < R(0) ? -det : det);
}

// per shell face: [0] w.g / stiffness (d/d stiff), [1] d(w.g)/d weft, [2] d(w.g)/d warp
__global__ void k_adj_shell(uint32_t n, const uint32_t* __restrict__ sv, const float* __restrict__ mu,
                            const float* __restrict__ lam, const float* __restrict__ stiff,
                            const float* __restrict__ uv, const uint8_t* __restrict__ panel,
                            const float* __restrict__ scale /* 2 per panel: weft, warp */, const float* __restrict__ x,
                            const float* __restrict__ w, const float* __restrict__ ge, double* __restrict__ out) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const uint32_t v[3] = {sv[3 * e], sv[3 * e + 1], sv[3 * e + 2]};
  V3<double> p[3], wv[3];
  double wg = 0;
  for (int a = 0; a < 3; ++a) {
    p[a] = ld3<double>(x, v[a]);
    wv[a] = ld3<double>(w, v[a]);
    for (int c = 0; c < 3; ++c) wg += (double)w[3 * v[a] + c] * (double)ge[9 * (size_t)e + 3 * a + c];
  }
  out[3 * (size_t)e] = wg / (double)stiff[e];
  const double su = scale[2 * panel[e]], svv = scale[2 * panel[e] + 1];
  auto wdotg = [&](double a, double b) {
    double dm[4], area;
    pattern_rest<double>(uv + 6 * (size_t)e, a, b, dm, &area);
    M2<double> D{dm[0], dm[1], dm[2], dm[3]};
    V3<double> g[3];
    shell_grad<double>(p, D, area, (double)mu[e], (double)lam[e], g);
    return wv[0].dot(g[0]) + wv[1].dot(g[1]) + wv[2].dot(g[2]);
  };
  const double du = 1e-5 * su, dv = 1e-5 * svv;
  out[3 * (size_t)e + 1] = (wdotg(su + du, svv) - wdotg(su - du, svv)) / (2 * du);
  out[3 * (size_t)e + 2] = (wdotg(su, svv + dv) - wdotg(su, svv - dv)) / (2 * dv);
}

// per stitch: w.g / stiffness
__global__ void k_adj_stitch(uint32_t n, const uint32_t* __restrict__ sidx, const float* __restrict__ skl,
                             const float* __restrict__ w, const float* __restrict__ ge, double* __restrict__ out) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double wg = 0;
  for (int q = 0; q < 6; ++q)
    for (int c = 0; c < 3; ++c) wg += (double)w[3 * sidx[6 * e + q] + c] * (double)ge[18 * (size_t)e + 3 * q + c];
  out[e] = wg / (double)skl[3 * e];
}

// a_x <- M/h^2 w - a_v/h, a_v <- M/h w
__global__ void k_adj_state(const float* __restrict__ w, const float* __restrict__ im, uint32_t n3, double h,
                            double* __restrict__ ax, double* __restrict__ av) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  const float iv = im[i / 3];
  if (!(iv > 0.f)) {
    ax[i] = 0.0;
    av[i] = 0.0;
    return;
  }
  const double m = 1.0 / (double)iv, wi = (double)w[i];
  const double avo = av[i];
  ax[i] = m / (h * h) * wi - avo / h;
  av[i] = m / h * wi;
}

// ---- preconditioned MINRES for the symmetric, possibly indefinite, exact Hessian --------
// Paige & Saunders (1975), "Solution of sparse indefinite systems of linear equations": the
// Lanczos process on M^-1 H with Givens rotations of its tridiagonal matrix, x updated along
// the directions w. M is the SPD preconditioner factored from the step's projected matrix.

constexpr int DOT_BLOCKS = 256;

__global__ void k_dot_partial(const double* __restrict__ a, const double* __restrict__ b, uint32_t n,
                              double* __restrict__ part) {
  __shared__ double sh[256];
  double acc = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += a[i] * b[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_dot_final(double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[DOT_BLOCKS];
  sh[threadIdx.x] = part[threadIdx.x];
  __syncthreads();
  for (int o = DOT_BLOCKS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// v = y / beta (and its FP32 copy)
__global__ void k_mr_scale(const double* __restrict__ y, double inv_beta, uint32_t n, double* __restrict__ v,
                           float* __restrict__ vf) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double t = y[i] * inv_beta;
  v[i] = t;
  vf[i] = (float)t;
}

// y = H v - c r1  (H v arrives in FP32)
__global__ void k_mr_lanczos1(const double* __restrict__ hv, const double* __restrict__ r1, double c, uint32_t n,
                              double* __restrict__ y) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = hv[i] - c * r1[i];
}

// y = (Ps + C) x with the stored FP32 blocks and FP64 vectors and sums, one thread per block
// row: the Lanczos vectors keep their precision through the product (rounding them to FP32
// around it limits MINRES to ~1e-7 and the adjoint to ~1e-3 on stiff drapes)
__global__ void k_spmv64(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col,
                         const float* __restrict__ val, const uint32_t* __restrict__ crp,
                         const uint32_t* __restrict__ ccol, const float* __restrict__ cval, uint32_t nb,
                         const double* __restrict__ x, double* __restrict__ y) {
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nb) return;
  double y0 = 0, y1 = 0, y2 = 0;
  auto block = [&](const float* m, uint32_t c) {
    const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
    y0 += (double)m[0] * x0 + (double)m[1] * x1 + (double)m[2] * x2;
    y1 += (double)m[3] * x0 + (double)m[4] * x1 + (double)m[5] * x2;
    y2 += (double)m[6] * x0 + (double)m[7] * x1 + (double)m[8] * x2;
  };
  for (uint32_t k = rp[row]; k < rp[row + 1]; ++k) block(val + 9 * (size_t)k, col[k]);
  for (uint32_t k = crp[row]; k < crp[row + 1]; ++k) block(cval + 9 * (size_t)k, ccol[k]);
  y[3 * row] = y0;
  y[3 * row + 1] = y1;
  y[3 * row + 2] = y2;
}

// y -= c r2, then its FP32 copy for the preconditioner
__global__ void k_mr_lanczos2(const double* __restrict__ r2, double c, uint32_t n, double* __restrict__ y,
                              float* __restrict__ yf) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double t = y[i] - c * r2[i];
  y[i] = t;
  yf[i] = (float)t;
}

__global__ void k_mr_widen(const float* __restrict__ zf, uint32_t n, double* __restrict__ z) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = (double)zf[i];
}

// out = (v - e pe - dl pd) / g; x += phi out
__global__ void k_mr_update(const double* __restrict__ v, const double* __restrict__ pe, const double* __restrict__ pd,
                            double e, double dl, double inv_g, double phi, uint32_t n, double* __restrict__ out,
                            double* __restrict__ x) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double w = (v[i] - e * pe[i] - dl * pd[i]) * inv_g;
  out[i] = w;
  x[i] += phi * w;
}

// b = a_x + a_v / h in FP64 (0 on pinned rows)
__global__ void k_adj_rhs64(const double* __restrict__ ax, const double* __restrict__ av,
                            const uint8_t* __restrict__ pinned, uint32_t n3, double inv_h, double* __restrict__ b) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  b[i] = pinned[i / 3] ? 0.0 : ax[i] + av[i] * inv_h;
}

__global__ void k_narrow(const double* __restrict__ x, uint32_t n, float* __restrict__ xf) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) xf[i] = (float)x[i];
}

// Solves H x = b (b in a->mr[0]; x to xf) with the scene's assembled matrix as H and the
// factored preconditioner; relative (preconditioned) residual tol.
int minres(mguso_adjoint* a, Scene& s, double tol, uint32_t max_iter, float* xf, mguso_lin_stats* ls) {
  cudaStream_t st = s.st;
  const uint32_t n = 3 * s.nv;
  const unsigned g = ceil_div(n, 256);
  MG_CHECK_ARG(a->mr[8].cap >= n && a->mf[1].cap >= n && a->dots.cap >= DOT_BLOCKS + 2, "minres: work vectors");
  double* r1 = a->mr[0].p;  // holds b on entry
  double* r2 = a->mr[1].p;
  double* y = a->mr[2].p;
  double* v = a->mr[3].p;
  double* w = a->mr[4].p;
  double* w1 = a->mr[5].p;
  double* w2 = a->mr[6].p;
  double* x = a->mr[7].p;
  double* hv = a->mr[8].p;
  float* vf = a->mf[0].p;
  float* tf = a->mf[1].p;
  auto precond = [&](const float* r, float* z) -> int {
    if (s.schwarz) return schwarz_apply(s.schwarz.get(), r, z, st, nullptr);
    return bj_apply(s.bjinv.p, r, z, s.nv, s.ctx->sm_count, st, nullptr);
  };
  auto dot = [&](const double* p, const double* q, double* out) -> int {
    k_dot_partial<<<DOT_BLOCKS, 256, 0, st>>>(p, q, n, a->dots.p);
    k_dot_final<<<1, DOT_BLOCKS, 0, st>>>(a->dots.p, a->dots.p + DOT_BLOCKS);
    MG_CUDA(cudaMemcpyAsync(out, a->dots.p + DOT_BLOCKS, 8, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    return MGUSO_OK;
  };
  MG_CUDA(cudaMemsetAsync(x, 0, 8 * (size_t)n, st));
  MG_CUDA(cudaMemsetAsync(w, 0, 8 * (size_t)n, st));
  MG_CUDA(cudaMemsetAsync(w2, 0, 8 * (size_t)n, st));
  MG_CUDA(cudaMemcpyAsync(r2, r1, 8 * (size_t)n, cudaMemcpyDeviceToDevice, st));
  k_narrow<<<g, 256, 0, st>>>(r1, n, tf);
  MG_TRY(precond(tf, vf));
  k_mr_widen<<<g, 256, 0, st>>>(vf, n, y);
  double beta1 = 0;
  MG_TRY(dot(r1, y, &beta1));
  ls->iters = 0;
  ls->residual = 0;
  ls->status = MGUSO_OK;
  if (!(beta1 > 0)) {
    MG_CUDA(cudaMemsetAsync(xf, 0, 4 * (size_t)n, st));
    return MGUSO_OK;
  }
  beta1 = std::sqrt(beta1);
  double oldb = 0, beta = beta1, dbar = 0, epsln = 0, phibar = beta1, cs = -1, sn = 0;
  uint32_t it = 0;
  for (; it < max_iter && phibar > tol * beta1; ++it) {
    k_mr_scale<<<g, 256, 0, st>>>(y, 1.0 / beta, n, v, vf);
    k_spmv64<<<ceil_div(s.nv, 128), 128, 0, st>>>(s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.c_row_ptr.p,
                                                   s.c_col.p ? s.c_col.p : s.c_row_ptr.p, s.c_val.p, s.nv, v, hv);
    k_mr_lanczos1<<<g, 256, 0, st>>>(hv, r1, it > 0 ? beta / oldb : 0.0, n, y);
    double alfa = 0;
    MG_TRY(dot(v, y, &alfa));
    k_mr_lanczos2<<<g, 256, 0, st>>>(r2, alfa / beta, n, y, tf);
    // r1 <- r2, r2 <- y, y <- M^-1 r2 (into the old r1's storage)
    std::swap(r1, r2);
    std::swap(r2, y);
    MG_TRY(precond(tf, vf));
    k_mr_widen<<<g, 256, 0, st>>>(vf, n, y);
    oldb = beta;
    double bb = 0;
    MG_TRY(dot(r2, y, &bb));
    if (!(bb >= 0) || !std::isfinite(bb)) {
      set_error("adjoint: the preconditioner is not positive definite");
      ls->status = MGUSO_ERR_PCG_CAP;
      break;
    }
    beta = std::sqrt(bb);
    const double oldeps = epsln;
    const double delta = cs * dbar + sn * alfa;
    const double gbar = sn * dbar - cs * alfa;
    epsln = sn * beta;
    dbar = -cs * beta;
    const double gamma = std::max(std::hypot(gbar, beta), 1e-300);
    cs = gbar / gamma;
    sn = beta / gamma;
    const double phi = cs * phibar;
    phibar = sn * phibar;
    // (w1, w2, w) <- (w2, w, (v - oldeps w2 - delta w) / gamma), the new w in w1's storage
    k_mr_update<<<g, 256, 0, st>>>(v, w2, w, oldeps, delta, 1.0 / gamma, phi, n, w1, x);
    double* const wn = w1;
    w1 = w2;
    w2 = w;
    w = wn;
    if (!(beta > 0)) {
      ++it;
      break;
    }
  }
  MG_CUDA(cudaGetLastError());
  k_narrow<<<g, 256, 0, st>>>(x, n, xf);
  ls->iters = it;
  ls->residual = phibar / beta1;
  if (ls->status == MGUSO_OK && phibar > tol * beta1) ls->status = MGUSO_ERR_PCG_CAP;
  return MGUSO_OK;
}

int apply_theta(mguso_adjoint* a, const double* theta) {
  const uint32_t P = a->npanel, S = a->nseam, nsh = a->base.nshell;
  a->theta.assign(theta, theta + 3 * P + S);
  for (size_t i = 0; i < a->theta.size(); ++i)
    MG_CHECK_ARG(std::isfinite(a->theta[i]) && a->theta[i] > 0, "adjoint: parameters must be finite and > 0");
  a->rest.resize(5 * (size_t)nsh);
  a->stiff.resize(nsh);
  for (uint32_t f = 0; f < nsh; ++f) {
    const uint32_t p = a->panel[f];
    const float su = (float)theta[P + 2 * p + 1], sv = (float)theta[P + 2 * p];
    float dm[4], area;
    pattern_rest<float>(a->uv.data() + 6 * (size_t)f, su, sv, dm, &area);
    std::memcpy(&a->rest[5 * (size_t)f], dm, 16);
    a->rest[5 * (size_t)f + 4] = area;
    a->stiff[f] = (float)theta[p];
  }
  a->skl = a->skl0;
  for (uint32_t i = 0; i < a->base.nstitch; ++i) a->skl[3 * (size_t)i] *= (float)theta[3 * P + a->seam[i]];
  return MGUSO_OK;
}

}  // namespace

extern "C" {

int mguso_adjoint_create(mguso_ctx* ctx, const mguso_scene_desc* d, const mguso_adjoint_spec* spec,
                         mguso_adjoint** out) {
  MG_CHECK_ARG(ctx && d && spec && out, "null argument");
  MG_CHECK_ARG(spec->npanel >= 1 && spec->npanel <= 255 && spec->nseam <= 255, "adjoint: panel/seam counts");
  MG_CHECK_ARG(d->nshell > 0 && spec->shell_uv && spec->shell_panel, "adjoint: pattern data required");
  MG_CHECK_ARG(d->nstitch == 0 || spec->stitch_seam, "adjoint: stitch seams required");
  MG_CHECK_ARG(d->positions && d->inv_mass && d->shell_faces, "adjoint: null arrays");
  MG_CHECK_ARG(!(d->params.friction > 0), "adjoint: friction is not differentiated (set friction = 0)");
  MG_CHECK_ARG(!(d->params.membrane_warp > 0 || d->params.membrane_weft > 0 || d->params.membrane_shear > 0),
               "adjoint: the Baraff-Witkin membrane is not differentiated (set its stiffnesses to 0)");
  auto a = std::make_unique<mguso_adjoint>();
  a->ctx = ctx;
  a->base = *d;
  const uint32_t nv = d->nv;
  a->pos.assign(d->positions, d->positions + 3 * (size_t)nv);
  if (d->velocities)
    a->vel.assign(d->velocities, d->velocities + 3 * (size_t)nv);
  else
    a->vel.assign(3 * (size_t)nv, 0.f);
  a->im.assign(d->inv_mass, d->inv_mass + nv);
  if (d->nt) a->tris.assign(d->tris, d->tris + 3 * (size_t)d->nt);
  if (d->static_mask) a->mask.assign(d->static_mask, d->static_mask + nv);
  a->shf.assign(d->shell_faces, d->shell_faces + 3 * (size_t)d->nshell);
  if (d->nstitch) {
    a->sidx.assign(d->stitch_idx, d->stitch_idx + 6 * (size_t)d->nstitch);
    a->sw.assign(d->stitch_w, d->stitch_w + 6 * (size_t)d->nstitch);
    a->skl0.assign(d->stitch_kl, d->stitch_kl + 3 * (size_t)d->nstitch);
    a->seam.assign(spec->stitch_seam, spec->stitch_seam + d->nstitch);
    for (uint8_t q : a->seam) MG_CHECK_ARG(q < spec->nseam, "adjoint: seam index out of range");
    for (uint32_t i = 0; i < d->nstitch; ++i)
      MG_CHECK_ARG(a->skl0[3 * (size_t)i] > 0, "adjoint: stitches need a positive base stiffness");
  }
  if (d->ncollider) a->cols.assign(d->colliders, d->colliders + 8 * (size_t)d->ncollider);
  a->uv.assign(spec->shell_uv, spec->shell_uv + 6 * (size_t)d->nshell);
  a->panel.assign(spec->shell_panel, spec->shell_panel + d->nshell);
  for (uint8_t p : a->panel) MG_CHECK_ARG(p < spec->npanel, "adjoint: panel index out of range");
  a->npanel = spec->npanel;
  a->nseam = spec->nseam;
  *out = a.release();
  return MGUSO_OK;
}

int mguso_adjoint_destroy(mguso_adjoint* a) {
  delete a;
  return MGUSO_OK;
}

int mguso_adjoint_forward(mguso_adjoint* a, const double* theta, uint32_t nsteps, uint32_t checkpoint_every,
                          float* x_out, mguso_step_stats* stats) {
  MG_CHECK_ARG(a && theta && x_out && nsteps > 0 && checkpoint_every > 0, "bad argument");
  MG_CUDA(cudaSetDevice(a->ctx->device));
  MG_TRY(apply_theta(a, theta));
  mguso_scene_desc d = a->base;
  d.positions = a->pos.data();
  d.velocities = a->vel.data();
  d.inv_mass = a->im.data();
  d.tris = a->tris.empty() ? nullptr : a->tris.data();
  d.static_mask = a->mask.empty() ? nullptr : a->mask.data();
  d.shell_faces = a->shf.data();
  d.stitch_idx = a->sidx.empty() ? nullptr : a->sidx.data();
  d.stitch_w = a->sw.empty() ? nullptr : a->sw.data();
  d.stitch_kl = a->skl.empty() ? nullptr : a->skl.data();
  d.colliders = a->cols.empty() ? nullptr : a->cols.data();
  d.shell_rest = a->rest.data();
  d.shell_stiff = a->stiff.data();
  a->scene.reset();
  auto sc = std::make_unique<mguso_scene>();
  sc->s.ctx = a->ctx;
  // FP32 preconditioner tiles: the backward MINRES solves run to 1e-10 and converge faster
  // with them, and the forward then follows the drape's FP32-factor trajectory
  sc->s.fp16_factor = false;
  MG_TRY(scene_build(sc->s, &d, {0, d.nv}));
  a->scene = std::move(sc);
  Scene& s = a->scene->s;
  MG_CHECK_ARG(s.n_shell == d.nshell, "adjoint: every shell face must be kept");
  a->nsteps = nsteps;
  a->every = checkpoint_every;
  const size_t n3 = 3 * (size_t)s.nv;
  const uint32_t nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  a->ck_x.clear();
  a->ck_v.clear();
  for (uint32_t c = 0; c < nck; ++c) {
    a->ck_x.push_back(std::make_unique<DevBuf<float>>());
    a->ck_v.push_back(std::make_unique<DevBuf<float>>());
    MG_TRY(a->ck_x.back()->reserve(n3));
    MG_TRY(a->ck_v.back()->reserve(n3));
  }
  for (uint32_t n = 0; n < nsteps; ++n) {
    if (n % checkpoint_every == 0) {
      const uint32_t c = n / checkpoint_every;
      MG_CUDA(cudaMemcpyAsync(a->ck_x[c]->p, s.x.p, 4 * n3, cudaMemcpyDeviceToDevice, s.st));
      MG_CUDA(cudaMemcpyAsync(a->ck_v[c]->p, s.v.p, 4 * n3, cudaMemcpyDeviceToDevice, s.st));
    }
    mguso_step_stats st{};
    MG_TRY(scene_step(s, &st));
    if (stats) stats[n] = st;
  }
  MG_CUDA(cudaMemcpyAsync(x_out, s.x.p, 4 * n3, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  return MGUSO_OK;
}

int mguso_adjoint_states(mguso_adjoint* a, float* x_all, float* v_all) {
  MG_CHECK_ARG(a && x_all && v_all && a->scene, "bad argument (forward first)");
  MG_CUDA(cudaSetDevice(a->ctx->device));
  Scene& s = a->scene->s;
  cudaStream_t st = s.st;
  const size_t n3 = 3 * (size_t)s.nv;
  for (uint32_t c = 0; c < (uint32_t)a->ck_x.size(); ++c) {
    const uint32_t n0 = c * a->every, n1 = std::min(a->nsteps, n0 + a->every);
    MG_CUDA(cudaMemcpyAsync(s.x.p, a->ck_x[c]->p, 4 * n3, cudaMemcpyDeviceToDevice, st));
    MG_CUDA(cudaMemcpyAsync(s.v.p, a->ck_v[c]->p, 4 * n3, cudaMemcpyDeviceToDevice, st));
    for (uint32_t n = n0; n <= n1; ++n) {
      MG_CUDA(cudaMemcpyAsync(x_all + n * n3, s.x.p, 4 * n3, cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaMemcpyAsync(v_all + n * n3, s.v.p, 4 * n3, cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaStreamSynchronize(st));
      if (n < n1) {
        mguso_step_stats stt{};
        MG_TRY(scene_step(s, &stt));
      }
    }
  }
  return MGUSO_OK;
}

int mguso_adjoint_backward(mguso_adjoint* a, const float* dl_dx, double* dl_dtheta) {
  MG_CHECK_ARG(a && dl_dx && dl_dtheta && a->scene, "bad argument (forward first)");
  MG_CUDA(cudaSetDevice(a->ctx->device));
  Scene& s = a->scene->s;
  cudaStream_t st = s.st;
  const uint32_t nv = s.nv, n3 = 3 * nv, P = a->npanel, S = a->nseam;
  const double h = s.p.dt;
  const size_t np = 3 * P + S;
  std::vector<double> grad(np, 0.0);
  // adjoint state, parameter partials
  MG_TRY(a->ax.reserve(n3));
  MG_TRY(a->av.reserve(n3));
  MG_TRY(a->c_shell.reserve(3 * (size_t)std::max<uint32_t>(s.n_shell, 1)));
  MG_TRY(a->c_stitch.reserve(std::max<uint32_t>(s.n_stitch, 1)));
  for (auto& b : a->mr) MG_TRY(b.reserve(n3));  // the right-hand side is written into mr[0]
  for (auto& b : a->mf) MG_TRY(b.reserve(n3));
  MG_TRY(a->dots.reserve(DOT_BLOCKS + 2));
  {
    std::vector<double> h_ax(dl_dx, dl_dx + n3);
    MG_CUDA(cudaMemcpyAsync(a->ax.p, h_ax.data(), 8 * (size_t)n3, cudaMemcpyHostToDevice, st));
    MG_CUDA(cudaMemsetAsync(a->av.p, 0, 8 * (size_t)n3, st));
    MG_CUDA(cudaStreamSynchronize(st));
  }
  std::vector<float> scale(2 * P);
  for (uint32_t p = 0; p < P; ++p) {
    scale[2 * p] = (float)a->theta[P + 2 * p + 1];      // weft: pattern u
    scale[2 * p + 1] = (float)a->theta[P + 2 * p];      // warp: pattern v
  }
  MG_TRY(a->d_scale.upload(scale.data(), scale.size(), st));
  MG_TRY(a->d_uv.upload(a->uv.data(), a->uv.size(), st));
  MG_TRY(a->d_panel.upload(a->panel.data(), a->panel.size(), st));
  MG_TRY(a->d_stiff.upload(a->stiff.data(), a->stiff.size(), st));
  std::vector<double> h_cs(3 * (size_t)s.n_shell), h_ct(s.n_stitch);
  // the adjoint systems are solved to a relative (preconditioned) residual of 1e-10
  const double tol = 1e-10;
  const uint32_t max_iter = std::max<uint32_t>(s.p.cg_max_iter, 4000);
  int rc = MGUSO_OK;
  const char* tr = getenv("MGUSO_TRACE");
  const bool trace = tr && tr[0] != '0';
  const uint32_t nseg = (uint32_t)a->ck_x.size();
  for (int c = (int)nseg - 1; c >= 0 && rc == MGUSO_OK; --c) {
    const uint32_t n0 = c * a->every, n1 = std::min(a->nsteps, n0 + a->every);
    // recompute the segment's states x_n0 .. x_n1
    while (a->seg_x.size() < a->every + 1) {
      a->seg_x.push_back(std::make_unique<DevBuf<float>>());
      a->seg_v.push_back(std::make_unique<DevBuf<float>>());
    }
    for (uint32_t i = 0; i <= n1 - n0; ++i) {
      MG_TRY(a->seg_x[i]->reserve(n3));
      MG_TRY(a->seg_v[i]->reserve(n3));
    }
    MG_CUDA(cudaMemcpyAsync(s.x.p, a->ck_x[c]->p, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
    MG_CUDA(cudaMemcpyAsync(s.v.p, a->ck_v[c]->p, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
    for (uint32_t n = n0; n <= n1; ++n) {
      MG_CUDA(cudaMemcpyAsync(a->seg_x[n - n0]->p, s.x.p, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
      MG_CUDA(cudaMemcpyAsync(a->seg_v[n - n0]->p, s.v.p, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
      if (n < n1) {
        mguso_step_stats stt{};
        MG_TRY(scene_step(s, &stt));
      }
    }
    for (int n = (int)n1 - 1; n >= (int)n0 && rc == MGUSO_OK; --n) {
      const float* xn = a->seg_x[n - n0]->p;
      const float* vn = a->seg_v[n - n0]->p;
      const float* xn1 = a->seg_x[n - n0 + 1]->p;
      // the Newton system at the converged x_{n+1} of step n
      MG_CUDA(cudaMemcpyAsync(s.x.p, xn1, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
      MG_CUDA(cudaMemcpyAsync(s.x0.p, xn, 4 * (size_t)n3, cudaMemcpyDeviceToDevice, st));
      k_predict<<<ceil_div(nv, 256), 256, 0, st>>>(xn, vn, s.inv_mass.p, nv, s.p.dt, s.p.gravity[0], s.p.gravity[1],
                                                   s.p.gravity[2], s.xt.p);
      uint32_t nst = 0;
      if (s.p.self_collision) {
        MG_TRY(build_bvhs(s, s.x.p));
        MG_TRY(collect_stencils(s, &nst));
      }
      // the step's projected matrix: the contact stiffnesses as the step computed them, and
      // the (SPD) preconditioner
      s.hess_mode = 0;
      MG_TRY(assemble_elastic(s));
      MG_TRY(assemble_colliders(s));
      MG_TRY(contact_stiffness(s, nst));
      MG_TRY(assemble_contacts(s, nst));
      if (s.schwarz)
        MG_TRY(schwarz_factor_with(s.schwarz.get(), s.c_row_ptr.p, s.c_col.p, s.c_val.p, st));
      else
        MG_TRY(blockjacobi_factor(s.A.get(), s.bjinv.p, st));
      // the exact Hessian at x_{n+1}
      s.hess_mode = 2;
      rc = assemble_elastic(s);
      if (rc == MGUSO_OK) rc = assemble_colliders(s);
      if (rc == MGUSO_OK) rc = assemble_contacts(s, nst);
      s.hess_mode = 0;
      if (rc != MGUSO_OK) break;
      // H w = a_x + a_v / h
      k_adj_rhs64<<<ceil_div(n3, 256), 256, 0, st>>>(a->ax.p, a->av.p, s.pinned.p, n3, 1.0 / h, a->mr[0].p);
      mguso_lin_stats ls{};
      rc = minres(a, s, tol, max_iter, s.work.x.p, &ls);
      if (rc == MGUSO_OK && ls.status != MGUSO_OK) {
        set_error("adjoint: MINRES did not converge at step " + std::to_string(n) + " (relative residual " +
                  std::to_string(ls.residual) + " after " + std::to_string(ls.iters) + " iterations)");
        rc = MGUSO_ERR_PCG_CAP;
      }
      if (rc != MGUSO_OK) break;
      const float* wv = s.work.x.p;
      // parameter partials
      if (s.n_shell)
        k_adj_shell<<<ceil_div(s.n_shell, 128), 128, 0, st>>>(s.n_shell, s.shell_v.p, s.shell_mu.p, s.shell_lam.p,
                                                            a->d_stiff.p, a->d_uv.p, a->d_panel.p, a->d_scale.p, s.x.p,
                                                            wv, s.gentries.p + 3 * s.gb_shell, a->c_shell.p);
      if (s.n_stitch)
        k_adj_stitch<<<ceil_div(s.n_stitch, 128), 128, 0, st>>>(s.n_stitch, s.stitch_idx.p, s.stitch_kl.p, wv,
                                                              s.gentries.p + 3 * s.gb_stitch, a->c_stitch.p);
      k_adj_state<<<ceil_div(n3, 256), 256, 0, st>>>(wv, s.inv_mass.p, n3, h, a->ax.p, a->av.p);
      MG_CUDA(cudaGetLastError());
      if (trace) {
        std::vector<float> hw(n3);
        std::vector<double> hx(n3);
        MG_CUDA(cudaMemcpyAsync(hw.data(), wv, 4 * (size_t)n3, cudaMemcpyDeviceToHost, st));
        MG_CUDA(cudaMemcpyAsync(hx.data(), a->ax.p, 8 * (size_t)n3, cudaMemcpyDeviceToHost, st));
        MG_CUDA(cudaStreamSynchronize(st));
        double mw = 0, mx = 0;
        for (uint32_t i = 0; i < n3; ++i) {
          mw = std::max(mw, (double)std::fabs(hw[i]));
          mx = std::max(mx, std::fabs(hx[i]));
        }
        fprintf(stderr, "[mguso adjoint] step %d stencils %u minres %u res %.3e status %d |w| %.3e |a_x| %.3e\n", n, nst,
                ls.iters, ls.residual, ls.status, mw, mx);
      }
      if (s.n_shell)
        MG_CUDA(cudaMemcpyAsync(h_cs.data(), a->c_shell.p, 8 * h_cs.size(), cudaMemcpyDeviceToHost, st));
      if (s.n_stitch)
        MG_CUDA(cudaMemcpyAsync(h_ct.data(), a->c_stitch.p, 8 * h_ct.size(), cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaStreamSynchronize(st));
      for (uint32_t f = 0; f < s.n_shell; ++f) {
        const uint32_t p = a->panel[f];
        grad[p] -= h_cs[3 * (size_t)f];
        grad[P + 2 * p + 1] -= h_cs[3 * (size_t)f + 1];  // weft
        grad[P + 2 * p] -= h_cs[3 * (size_t)f + 2];      // warp
      }
      for (uint32_t i = 0; i < s.n_stitch; ++i) grad[3 * P + a->seam[i]] -= h_ct[i];
    }
  }
  MG_TRY(rc);
  std::memcpy(dl_dtheta, grad.data(), 8 * np);
  return MGUSO_OK;
}

}  // extern "C"
