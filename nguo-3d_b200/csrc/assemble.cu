// Hessian and gradient assembly of the implicit step on the GPU
// (ImplicitSolver::assemble, implicit.rs:2280-3155).
//
// 1. Element kernels (one thread per element) write local 3x3 blocks and gradient entries
//    into contribution buffers at push-order positions: inertia (:2394-2405), stitches
//    (:2456-2485), stretch springs (:2488-2530), StVK shells (:2608-2652), hinges
//    (:2699-2740). Elements whose vertices are all pinned are constant and computed once.
// 2. A gather kernel sums each slot's contributions in push order (no atomics), into the
//    system pattern Ps or the pinned pattern Pp, and each vertex's gradient entries.
// 3. Analytic colliders (:2954-3021) read the gathered diagonal block for the Rayleigh
//    stiffness and add their block and gradient after everything elastic.
// 4. Self contact (:3026-3103): per stencil, the Rayleigh stiffness from the gathered
//    blocks, the barrier, friction, 16 (+16) blocks and 4 (+4) gradient entries; the
//    entries are sorted by (row, col) keeping stencil order and added in that order onto
//    Ps, or collected into the contact matrix C when the block lies outside Ps.
// This file is compiled without FMA contraction so FP32 products round as the
// reference's scalar f32 code does.
#include <algorithm>

#include "elements.cuh"
#include "reduce.cuh"
#include "scene.cuh"

namespace mg {

__device__ __forceinline__ void put_block(float* dst, const float* h, int ld, int r0, int c0, float scale) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) dst[3 * r + c] = scale * h[(r0 + r) * ld + c0 + c];
}

// ---- inertia ---------------------------------------------------------------------------
__global__ void k_inertia(const uint32_t* __restrict__ free_verts, uint32_t n_free, const float* __restrict__ im,
                          const float* __restrict__ x, const float* __restrict__ xt, float inv_h2,
                          float* __restrict__ cb, float* __restrict__ ge) {
  uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_free) return;
  uint32_t i = free_verts[f];
  float m = (1.0f / im[i]) * inv_h2;
  float* b = cb + 9 * (size_t)f;
#pragma unroll
  for (int k = 0; k < 9; ++k) b[k] = (k % 4 == 0) ? m : 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) ge[3 * (size_t)f + c] = m * (x[3 * i + c] - xt[3 * i + c]);
}

// ---- stitches (stitch.rs:57-107 at the stitch's stiffness) ------------------------------
__global__ void k_stitch(const uint32_t* __restrict__ act, uint32_t n, const uint32_t* __restrict__ sidx,
                         const float* __restrict__ sw, const float* __restrict__ skl, const float* __restrict__ x,
                         float* __restrict__ cb, float* __restrict__ ge, int exact) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t e = act[k];
  const uint32_t* ix = sidx + 6 * (size_t)e;
  float w[6], swt[6];
  for (int q = 0; q < 6; ++q) {
    w[q] = sw[6 * (size_t)e + q];
    swt[q] = q < 3 ? w[q] : -w[q];
  }
  float stiff = skl[3 * e], l0 = skl[3 * e + 1], lcap = skl[3 * e + 2];
  V3<float> t;
  for (int q = 0; q < 6; ++q) t += ld3<float>(x, ix[q]) * swt[q];
  float tn = t.length();
  float* blk = cb + 9 * 36 * (size_t)e;
  float* g = ge + 18 * (size_t)e;
  if (tn < 1e-12f || l0 <= 0.f) {
    for (int q = 0; q < 36 * 9; ++q) blk[q] = 0.f;
    for (int q = 0; q < 18; ++q) g[q] = 0.f;
    return;
  }
  float l = fminf(tn, lcap);
  V3<float> nn = t / l;
  V3<float> dedt = nn * (l / l0 - 1.0f);
  for (int q = 0; q < 6; ++q) {
    V3<float> gq = dedt * swt[q];
    g[3 * q] = stiff * gq.x;
    g[3 * q + 1] = stiff * gq.y;
    g[3 * q + 2] = stiff * gq.z;
  }
  float r = (l - l0) / l;
  float c0 = fmaxf(1.0f - r, 0.f) / l0;
  float c1 = fmaxf(r / l0, 0.f);
  if (exact) {
    // the Jacobian of the gradient: no clamp below rest length; past the cap the gradient
    // is linear in t
    c1 = r / l0;
    if (tn > lcap) c0 = 0.f;
  }
  for (int a = 0; a < 6; ++a) {
    V3<float> ga = nn * swt[a];
    for (int b = 0; b < 6; ++b) {
      V3<float> gb = nn * swt[b];
      float iden = c1 * swt[a] * swt[b];
      float* o = blk + 9 * (6 * a + b);
      for (int rr = 0; rr < 3; ++rr)
        for (int cc = 0; cc < 3; ++cc) {
          float v = c0 * ga[rr] * gb[cc];
          if (rr == cc) v += iden;
          o[3 * rr + cc] = stiff * v;
        }
    }
  }
}

// ---- stretch springs (spring_block, implicit.rs:3240-3263) --------------------------------
// With the edge strain limit on (slk > 0), each spring's blocks and gradient also carry the
// one-sided limit spring on the same edge (strain_block, strain_limit.rs:31-63; pushed after
// the stretch spring, implicit.rs:2508-2530): rest length slr[e] * rest, stiffness slk,
// zero while the edge is no longer than that. Its Hessian is the clamped spring block, which
// is already exact while it acts.
__global__ void k_spring(const uint32_t* __restrict__ act, uint32_t n, const uint32_t* __restrict__ sv,
                         const float* __restrict__ rest, float k, const float* __restrict__ x, float* __restrict__ cb,
                         float* __restrict__ ge, int exact, const float* __restrict__ slr, float slk) {
  uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  uint32_t e = act[q];
  uint32_t a = sv[2 * e], b = sv[2 * e + 1];
  V3<float> d = ld3<float>(x, a) - ld3<float>(x, b);
  float l = d.length();
  float h[9];
  V3<float> ga;
  if (l < 1e-9f) {
    for (int i = 0; i < 9; ++i) h[i] = (i % 4 == 0) ? k : 0.f;
  } else {
    V3<float> nrm = d / l;
    float ct = exact ? 1.0f - rest[e] / l : fmaxf(1.0f - rest[e] / l, 0.f);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        float nnt = nrm[i] * nrm[j];
        h[3 * i + j] = k * (nnt + ct * ((i == j ? 1.f : 0.f) - nnt));
      }
    ga = nrm * (k * (l - rest[e]));
  }
  if (slk > 0.f && slr[e] > 0.f) {
    const float r = rest[e] * slr[e];
    if (l > r) {  // spring_block at rest length r (l >= 1e-9 here unless r < 0)
      if (l < 1e-9f) {
        for (int i = 0; i < 9; ++i) h[i] += (i % 4 == 0) ? slk : 0.f;
      } else {
        V3<float> nrm = d / l;
        const float ct = fmaxf(1.0f - r / l, 0.f);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            float nnt = nrm[i] * nrm[j];
            h[3 * i + j] += slk * (nnt + ct * ((i == j ? 1.f : 0.f) - nnt));
          }
        ga += nrm * (slk * (l - r));
      }
    }
  }
  float* blk = cb + 36 * (size_t)e;
  for (int i = 0; i < 9; ++i) {
    blk[i] = h[i];
    blk[9 + i] = h[i];
    blk[18 + i] = -h[i];
    blk[27 + i] = -h[i];
  }
  float* g = ge + 6 * (size_t)e;
  g[0] = ga.x; g[1] = ga.y; g[2] = ga.z;
  g[3] = -ga.x; g[4] = -ga.y; g[5] = -ga.z;
}

// ---- Baraff-Witkin membrane (implicit.rs:2532-2596) ---------------------------------------
// One element's 9 blocks (each the sum of its warp, weft and shear terms) and 3 gradient
// entries, in FP32 as the reference.
__global__ void __launch_bounds__(128) k_membrane(const uint32_t* __restrict__ act, uint32_t n,
                                                  const uint32_t* __restrict__ mv, const float* __restrict__ dm,
                                                  const float* __restrict__ area, float kw, float kf, float ks,
                                                  const float* __restrict__ x, float* __restrict__ cb,
                                                  float* __restrict__ ge) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint32_t e = act[q];
  const V3<float> p[3] = {ld3<float>(x, mv[3 * e]), ld3<float>(x, mv[3 * e + 1]), ld3<float>(x, mv[3 * e + 2])};
  const float d4[4] = {dm[4 * e], dm[4 * e + 1], dm[4 * e + 2], dm[4 * e + 3]};
  V3<float> g[3];
  float h[9][9];
  membrane_grad_hess<float>(p, d4, area[e], kw, kf, ks, g, h);
  float* blk = cb + 81 * (size_t)e;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) blk[9 * (3 * a + b) + 3 * r + c] = h[3 * a + r][3 * b + c];
  float* gg = ge + 9 * (size_t)e;
  for (int a = 0; a < 3; ++a) {
    gg[3 * a] = g[a].x;
    gg[3 * a + 1] = g[a].y;
    gg[3 * a + 2] = g[a].z;
  }
}

// ---- StVK shells ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_shell(const uint32_t* __restrict__ act, uint32_t n,
                                               const uint32_t* __restrict__ sv, const float* __restrict__ dm,
                                               const float* __restrict__ area, const float* __restrict__ mu,
                                               const float* __restrict__ lam, float eps, const float* __restrict__ x,
                                               float* __restrict__ cb, float* __restrict__ ge, int exact,
                                               const uint8_t* __restrict__ vinst, uint32_t active) {
  uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  uint32_t e = act[q];
  if (!((active >> vinst[sv[3 * e]]) & 1u)) return;  // an instance the batch no longer iterates
  V3<float> p[3] = {ld3<float>(x, sv[3 * e]), ld3<float>(x, sv[3 * e + 1]), ld3<float>(x, sv[3 * e + 2])};
  M2<float> D{dm[4 * e], dm[4 * e + 1], dm[4 * e + 2], dm[4 * e + 3]};
  V3<float> g[3];
  float h[81];
  shell_grad_hess<float>(p, D, area[e], mu[e], lam[e], eps, g, h, !exact);
  if (exact) {
    // the exact Hessian in FP64 (its eigenvalue quotients cancel in FP32 when the two
    // singular values are close)
    V3<double> pd[3] = {p[0].cast<double>(), p[1].cast<double>(), p[2].cast<double>()};
    M2<double> Dd{D.xx, D.xy, D.yx, D.yy};
    V3<double> gd[3];
    double hd[81];
    shell_grad_hess<double>(pd, Dd, (double)area[e], (double)mu[e], (double)lam[e], (double)eps, gd, hd, false);
    for (int k = 0; k < 81; ++k) h[k] = (float)hd[k];
  }
  float* blk = cb + 81 * (size_t)e;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) put_block(blk + 9 * (3 * a + b), h, 9, 3 * a, 3 * b, 1.0f);
  float* gg = ge + 9 * (size_t)e;
  for (int a = 0; a < 3; ++a) {
    gg[3 * a] = g[a].x;
    gg[3 * a + 1] = g[a].y;
    gg[3 * a + 2] = g[a].z;
  }
}

// ---- hinges ----------------------------------------------------------------------------------
__global__ void k_hinge(const uint32_t* __restrict__ act, uint32_t n, const uint32_t* __restrict__ hv,
                        const float* __restrict__ rest, float kb, const float* __restrict__ x, float* __restrict__ cb,
                        float* __restrict__ ge, int exact, const uint8_t* __restrict__ vinst, uint32_t active) {
  uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  uint32_t e = act[q];
  if (!((active >> vinst[hv[4 * e]]) & 1u)) return;  // an instance the batch no longer iterates
  V3<float> p[4];
  for (int a = 0; a < 4; ++a) p[a] = ld3<float>(x, hv[4 * e + a]);
  float theta = dihedral_angle<float>(p);
  V3<float> g[4];
  dihedral_grad<float>(p, g);
  float kwt = kb * 1.0f;  // hinge weight w = 1 (bending.rs:150-156)
  float gval = theta - rest[e];
  // the hinge's 12 gradient entries and 144 block entries are 16-byte aligned runs (48 e and
  // 576 e bytes): stored as float4, a quarter of the store instructions of scalar stores
  float gv[12];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) gv[3 * a + c] = kwt * gval * g[a][c];
  float4* gg4 = reinterpret_cast<float4*>(ge + 12 * (size_t)e);
#pragma unroll
  for (int i = 0; i < 3; ++i) gg4[i] = make_float4(gv[4 * i], gv[4 * i + 1], gv[4 * i + 2], gv[4 * i + 3]);
  float* blk = cb + 144 * (size_t)e;
  if (exact) {
    // k (grad theta grad theta^T + (theta - theta0) hess theta), hess theta from FP64
    // central differences of the angle's gradient
    V3<double> pd[4], gd[4];
    for (int a = 0; a < 4; ++a) pd[a] = ld3<double>(x, hv[4 * e + a]);
    dihedral_grad<double>(pd, gd);
    const double gv = dihedral_angle<double>(pd) - (double)rest[e];
    const double eps = 1e-6 * fmax((pd[2] - pd[1]).length(), 1e-3);
    double H[144];
    for (int i = 0; i < 12; ++i)
      for (int j = 0; j < 12; ++j) H[12 * i + j] = gd[i / 3][i % 3] * gd[j / 3][j % 3];
    for (int i = 0; i < 12; ++i) {
      V3<double> q[4] = {pd[0], pd[1], pd[2], pd[3]}, gp[4], gm[4];
      q[i / 3][i % 3] = pd[i / 3][i % 3] + eps;
      dihedral_grad<double>(q, gp);
      q[i / 3][i % 3] = pd[i / 3][i % 3] - eps;
      dihedral_grad<double>(q, gm);
      for (int j = 0; j < 12; ++j) {
        const double hij = 0.5 * gv * (gp[j / 3][j % 3] - gm[j / 3][j % 3]) / (2 * eps);
        H[12 * i + j] += hij;
        H[12 * j + i] += hij;
      }
    }
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) blk[9 * (4 * a + b) + 3 * r + c] = (float)(kwt * H[12 * (3 * a + r) + 3 * b + c]);
    return;
  }
  float4* blk4 = reinterpret_cast<float4*>(blk);
#pragma unroll
  for (int i = 0; i < 36; ++i) {
    float v4[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int f = 4 * i + u, ab = f / 9, rc = f - 9 * ab;  // block (a, b), entry (r, c)
      const int a = ab >> 2, b = ab & 3, r = rc / 3, c = rc - 3 * r;
      v4[u] = kwt * g[a][r] * g[b][c];
    }
    blk4[i] = make_float4(v4[0], v4[1], v4[2], v4[3]);
  }
}

// ---- gathers ---------------------------------------------------------------------------------
__global__ void k_gather_blocks(const uint32_t* __restrict__ slot_ptr, const uint32_t* __restrict__ slot_list,
                                const float* __restrict__ cb, uint32_t nslots, uint32_t nnz_s,
                                float* __restrict__ vals, float* __restrict__ valp,
                                const uint8_t* __restrict__ slot_inst, uint32_t active) {
  uint32_t sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= nslots || !((active >> slot_inst[sl]) & 1u)) return;
  float acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.f;
  for (uint32_t j = slot_ptr[sl]; j < slot_ptr[sl + 1]; ++j) {
    const float* c = cb + 9 * (size_t)slot_list[j];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] += c[k];
  }
  float* out = sl < nnz_s ? vals + 9 * (size_t)sl : valp + 9 * (size_t)(sl - nnz_s);
#pragma unroll
  for (int k = 0; k < 9; ++k) out[k] = acc[k];
}

__global__ void k_gather_grad(const uint32_t* __restrict__ gv_ptr, const uint32_t* __restrict__ gv_list,
                              const float* __restrict__ ge, uint32_t nv, float* __restrict__ grad,
                              const uint8_t* __restrict__ vinst, uint32_t active) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv || !((active >> vinst[v]) & 1u)) return;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  for (uint32_t j = gv_ptr[v]; j < gv_ptr[v + 1]; ++j) {
    const float* g = ge + 3 * (size_t)gv_list[j];
    a0 += g[0];
    a1 += g[1];
    a2 += g[2];
  }
  grad[3 * v] = a0;
  grad[3 * v + 1] = a1;
  grad[3 * v + 2] = a2;
}

__global__ void k_pinned_identity(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                                  const uint8_t* __restrict__ pinned, uint32_t nv, float* __restrict__ vals) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv || !pinned[v]) return;
  for (uint32_t k = row_ptr[v]; k < row_ptr[v + 1]; ++k)
    if (col[k] == v)
      for (int q = 0; q < 9; ++q) vals[9 * (size_t)k + q] = (q % 4 == 0) ? 1.f : 0.f;
}

int assemble_elastic(Scene& s) {
  cudaStream_t st = s.st;
  const float h = s.p.dt, inv_h2 = 1.0f / (h * h);
  auto grid = [](uint32_t n) { return std::max<uint32_t>(ceil_div(n, 128), 1u); };
  float* cb = s.cblocks.p;
  float* ge = s.gentries.p;
  const int exact_all = s.hess_mode == 2;
  const int ex_shell = exact_all && (s.exact_terms & EXACT_SHELLS), ex_stitch = exact_all && (s.exact_terms & EXACT_STITCHES);
  const int ex_hinge = exact_all && (s.exact_terms & EXACT_HINGES), ex_spring = exact_all && (s.exact_terms & EXACT_SPRINGS);
  if (s.n_free)
    k_inertia<<<grid(s.n_free), 128, 0, st>>>(s.free_verts.p, s.n_free, s.inv_mass.p, s.x.p, s.xt.p, inv_h2,
                                            cb + 9 * s.cb_inertia, ge + 3 * s.gb_inertia);
  // all-pinned elements once (their contributions never change), then the active ones
  if (!s.static_done) {
    // the full element lists, built from identity index arrays
    std::vector<uint32_t> ids(std::max({s.n_stitch, s.n_spring, s.n_mem, s.n_shell, s.n_hinge, 1u}));
    for (uint32_t i = 0; i < ids.size(); ++i) ids[i] = i;
    DevBuf<uint32_t> all;
    MG_TRY(all.upload(ids.data(), ids.size(), st));
    if (s.n_stitch)
      k_stitch<<<grid(s.n_stitch), 128, 0, st>>>(all.p, s.n_stitch, s.stitch_idx.p, s.stitch_w.p, s.stitch_kl.p,
                                                 s.x.p, cb + 9 * s.cb_stitch, ge + 3 * s.gb_stitch, ex_stitch);
    if (s.n_spring)
      k_spring<<<grid(s.n_spring), 128, 0, st>>>(all.p, s.n_spring, s.spring_v.p, s.spring_rest.p, s.p.stiffness,
                                                 s.x.p, cb + 9 * s.cb_spring, ge + 3 * s.gb_spring, ex_spring,
                                                 s.spring_slr.p, s.edge_limit ? s.p.strain_limit_k : 0.f);
    if (s.n_mem)
      k_membrane<<<grid(s.n_mem), 128, 0, st>>>(all.p, s.n_mem, s.mem_v.p, s.mem_dm.p, s.mem_area.p,
                                                s.p.membrane_warp, s.p.membrane_weft, s.p.membrane_shear, s.x.p,
                                                cb + 9 * s.cb_mem, ge + 3 * s.gb_mem);
    if (s.n_shell)
      k_shell<<<grid(s.n_shell), 128, 0, st>>>(all.p, s.n_shell, s.shell_v.p, s.shell_dm.p, s.shell_area.p,
                                               s.shell_mu.p, s.shell_lam.p, s.p.eiganalysis_eps, s.x.p,
                                               cb + 9 * s.cb_shell, ge + 3 * s.gb_shell, ex_shell, s.vinst.p,
                                               0xffffffffu);
    if (s.n_hinge)
      k_hinge<<<grid(s.n_hinge), 128, 0, st>>>(all.p, s.n_hinge, s.hinge_v.p, s.hinge_rest.p, s.p.bend_stiffness,
                                               s.x.p, cb + 9 * s.cb_hinge, ge + 3 * s.gb_hinge, ex_hinge,
                                               s.vinst.p, 0xffffffffu);
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaStreamSynchronize(st));
    s.static_done = true;
  } else {
    if (s.n_act_stitch)
      k_stitch<<<grid(s.n_act_stitch), 128, 0, st>>>(s.act_stitch.p, s.n_act_stitch, s.stitch_idx.p, s.stitch_w.p,
                                                     s.stitch_kl.p, s.x.p, cb + 9 * s.cb_stitch, ge + 3 * s.gb_stitch, ex_stitch);
    if (s.n_act_spring)
      k_spring<<<grid(s.n_act_spring), 128, 0, st>>>(s.act_spring.p, s.n_act_spring, s.spring_v.p, s.spring_rest.p,
                                                     s.p.stiffness, s.x.p, cb + 9 * s.cb_spring, ge + 3 * s.gb_spring, ex_spring,
                                                     s.spring_slr.p, s.edge_limit ? s.p.strain_limit_k : 0.f);
    if (s.n_act_mem)
      k_membrane<<<grid(s.n_act_mem), 128, 0, st>>>(s.act_mem.p, s.n_act_mem, s.mem_v.p, s.mem_dm.p, s.mem_area.p,
                                                    s.p.membrane_warp, s.p.membrane_weft, s.p.membrane_shear, s.x.p,
                                                    cb + 9 * s.cb_mem, ge + 3 * s.gb_mem);
    if (s.n_act_shell)
      k_shell<<<grid(s.n_act_shell), 128, 0, st>>>(s.act_shell.p, s.n_act_shell, s.shell_v.p, s.shell_dm.p,
                                                   s.shell_area.p, s.shell_mu.p, s.shell_lam.p, s.p.eiganalysis_eps,
                                                   s.x.p, cb + 9 * s.cb_shell, ge + 3 * s.gb_shell, ex_shell, s.vinst.p,
                                               s.iter_active);
    if (s.n_act_hinge)
      k_hinge<<<grid(s.n_act_hinge), 128, 0, st>>>(s.act_hinge.p, s.n_act_hinge, s.hinge_v.p, s.hinge_rest.p,
                                                   s.p.bend_stiffness, s.x.p, cb + 9 * s.cb_hinge, ge + 3 * s.gb_hinge, ex_hinge,
                                               s.vinst.p, s.iter_active);
  }
  MG_CUDA(cudaGetLastError());
  uint32_t nslots = s.Ps.nnz + s.Pp.nnz;
  k_gather_blocks<<<grid(nslots), 128, 0, st>>>(s.slot_ptr.p, s.slot_list.p, cb, nslots, s.Ps.nnz, s.A->val.p,
                                                s.valp.p, s.slot_inst.p, s.iter_active);
  k_gather_grad<<<grid(s.nv), 128, 0, st>>>(s.gv_ptr.p, s.gv_list.p, ge, s.nv, s.grad.p, s.vinst.p, s.iter_active);
  k_pinned_identity<<<grid(s.nv), 128, 0, st>>>(s.Ps.row_ptr.p, s.Ps.col.p, s.pinned.p, s.nv, s.A->val.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// ---- analytic colliders (vertex_contact_full, contact.rs:1082-1125) -------------------------
template <class R>
__global__ void k_colliders(const uint32_t* __restrict__ free_verts, uint32_t n_free, const float* __restrict__ im,
                            const float* __restrict__ x, const float* __restrict__ x_start,
                            const float* __restrict__ cols, uint32_t ncol, const uint32_t* __restrict__ diag_slot,
                            float* __restrict__ vals, float* __restrict__ grad, float dhat, float kappa,
                            float coupling, int barrier_kind, int rayleigh, float mu, float feps) {
  uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_free) return;
  uint32_t i = free_verts[f];
  R m = R(1) / (R)im[i];
  V3<R> xi = ld3<R>(x, i);
  float* dblk = vals + 9 * (size_t)diag_slot[i];
  R el[1][9];
  for (int q = 0; q < 9; ++q) el[0][q] = (R)dblk[q];
  V3<R> gsum;
  R hs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t c = 0; c < ncol; ++c) {
    const float* cc = cols + 8 * c;
    R d;
    V3<R> n;
    V3<R> a((R)cc[1], (R)cc[2], (R)cc[3]);
    if (cc[0] == 0.f) {
      n = V3<R>((R)cc[4], (R)cc[5], (R)cc[6]);
      d = (xi - a).dot(n);
    } else {
      V3<R> v = xi - a;
      R l = v.length();
      if (l < R(1.0e-9)) {
        d = -(R)cc[7];
        n = V3<R>(0, 1, 0);
      } else {
        d = l - (R)cc[7];
        n = v / l;
      }
    }
    R k;
    if (rayleigh) {
      R one = 1;
      k = rayleigh_stiffness<R>(el, &m, &one, 1, n * d);
    } else {
      k = (R)kappa;
      if (coupling > 0 && m > 0) {
        R dd = rmax(rmax(d, R(0.1) * (R)dhat), R(1.0e-6));
        k = (R)kappa * (R(1) + (R)coupling * m / (dd * dd));
      }
    }
    R g, h;
    if (!barrier_of<R>(barrier_kind, d, (R)dhat, k, g, h)) continue;
    V3<R> f_c = n * g;
    gsum += f_c;
    R hp = rmax(h, R(0));
    for (int r = 0; r < 3; ++r)
      for (int c2 = 0; c2 < 3; ++c2) hs[3 * r + c2] += hp * n[r] * n[c2];
    if (mu > 0) {
      V3<R> fg;
      R fh[9];
      if (friction<R>(f_c, xi - ld3<R>(x_start, i), n, (R)mu, (R)feps, fg, fh)) {
        gsum += fg;
        for (int q = 0; q < 9; ++q) hs[q] += fh[q];
      }
    }
  }
  for (int q = 0; q < 9; ++q)
    if (hs[q] != 0) dblk[q] += (float)hs[q];
  grad[3 * i] += (float)gsum.x;
  grad[3 * i + 1] += (float)gsum.y;
  grad[3 * i + 2] += (float)gsum.z;
}

// ---- pins and pulls (implicit.rs:2809-2872) -----------------------------------------------
// One thread per vertex with pins or pulls, in push order (every pin of the vertex in the
// order they were set, then its pulls): a pin's stiffness reads the vertex's diagonal block
// as accumulated so far (the elastic blocks and the earlier pins), k = (H w).w / |w|^2 +
// m / gap^2 with w = x - target, gap = max(ghat - |w|, constraint_tol ghat), times the pin's
// stiffness when kinematic; gradient k w, k on the diagonal. A pull adds weight (x - target)
// and weight on the diagonal.
template <class R>
__global__ void k_pins_pulls(const uint32_t* __restrict__ pv, uint32_t n_pv, const uint32_t* __restrict__ pv_pin,
                             const uint32_t* __restrict__ pv_pull, const float* __restrict__ pin_target,
                             const float* __restrict__ pin_ghat, const uint8_t* __restrict__ pin_kin,
                             const float* __restrict__ pin_stiff, const float* __restrict__ pull_target,
                             const float* __restrict__ pull_weight, const float* __restrict__ im,
                             const float* __restrict__ x, const uint32_t* __restrict__ diag_slot,
                             float* __restrict__ vals, float* __restrict__ grad, float ctol) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_pv) return;
  const uint32_t i = pv[t];
  if (!(im[i] > 0.f)) return;
  const R m = R(1) / (R)im[i];
  const V3<R> xi = ld3<R>(x, i);
  float* dblk = vals + 9 * (size_t)diag_slot[i];
  R el[9];
  for (int q = 0; q < 9; ++q) el[q] = (R)dblk[q];
  V3<R> g;
  for (uint32_t p = pv_pin[t]; p < pv_pin[t + 1]; ++p) {
    const V3<R> w = xi - ld3<R>(pin_target, p);
    const R d = w.length();
    const R gh = (R)pin_ghat[p];
    const R gap = rmax(gh - d, (R)ctol * gh);
    const R d2 = w.length_squared();
    R tmp = 0;
    if (d2 > 0) {
      const V3<R> hw(el[0] * w.x + el[1] * w.y + el[2] * w.z, el[3] * w.x + el[4] * w.y + el[5] * w.z,
                     el[6] * w.x + el[7] * w.y + el[8] * w.z);
      tmp = hw.dot(w) / d2;
    }
    R kp = tmp + m / (gap * gap);
    if (pin_kin[p]) kp *= (R)pin_stiff[p];
    g += w * kp;
    el[0] += kp;
    el[4] += kp;
    el[8] += kp;
  }
  for (uint32_t q = pv_pull[t]; q < pv_pull[t + 1]; ++q) {
    const R wt = (R)pull_weight[q];
    g += (xi - ld3<R>(pull_target, q)) * wt;
    el[0] += wt;
    el[4] += wt;
    el[8] += wt;
  }
  dblk[0] = (float)el[0];
  dblk[4] = (float)el[4];
  dblk[8] = (float)el[8];
  grad[3 * i] += (float)g.x;
  grad[3 * i + 1] += (float)g.y;
  grad[3 * i + 2] += (float)g.z;
}

static int assemble_pins(Scene& s) {
  if (!s.n_pv) return MGUSO_OK;
  const unsigned g = ceil_div(s.n_pv, 128);
  const float ctol = s.p.constraint_tol > 0.f ? s.p.constraint_tol : 1.0e-2f;
  if (s.mixed)
    k_pins_pulls<double><<<g, 128, 0, s.st>>>(s.pv.p, s.n_pv, s.pv_pin.p, s.pv_pull.p, s.pin_target.p, s.pin_ghat.p,
                                              s.pin_kin.p, s.pin_stiff.p, s.pull_target.p, s.pull_weight.p,
                                              s.inv_mass.p, s.x.p, s.diag_slot.p, s.A->val.p, s.grad.p, ctol);
  else
    k_pins_pulls<float><<<g, 128, 0, s.st>>>(s.pv.p, s.n_pv, s.pv_pin.p, s.pv_pull.p, s.pin_target.p, s.pin_ghat.p,
                                             s.pin_kin.p, s.pin_stiff.p, s.pull_target.p, s.pull_weight.p,
                                             s.inv_mass.p, s.x.p, s.diag_slot.p, s.A->val.p, s.grad.p, ctol);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// ---- strain-limit barrier faces (implicit.rs:2743-2807) -----------------------------------
// One thread per face: its elastic stiffness w.(H w) from the blocks gathered so far (every
// elastic term and the inertia; w the face's positions about their centroid), then the
// barrier's gradient and 9x9 Hessian at the dynamic stiffness (sl_face_grad_hess) into the
// face's contribution (zeros when inactive). Every face reads the blocks before any face
// adds to them, as the reference does.
template <class R>
__global__ void __launch_bounds__(128) k_sl_faces(uint32_t n, const uint32_t* __restrict__ fv,
                                                  const float* __restrict__ fdm, const float* __restrict__ flim,
                                                  const float* __restrict__ fmass, const uint32_t* __restrict__ fslot,
                                                  const float* __restrict__ x, const float* __restrict__ vals,
                                                  const float* __restrict__ valp, uint32_t nnz_s, int kind, float eps,
                                                  float* __restrict__ out) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  V3<R> p[3];
  for (int a = 0; a < 3; ++a) p[a] = ld3<R>(x, fv[3 * f + a]);
  // centroid and offsets in FP32 (the reference's Vec3 arithmetic), then widened
  const V3<float> pf[3] = {ld3<float>(x, fv[3 * f]), ld3<float>(x, fv[3 * f + 1]), ld3<float>(x, fv[3 * f + 2])};
  const V3<float> cen = (pf[0] + pf[1] + pf[2]) / 3.0f;
  V3<R> w[3];
  for (int a = 0; a < 3; ++a) {
    const V3<float> d = pf[a] - cen;
    w[a] = V3<R>((R)d.x, (R)d.y, (R)d.z);
  }
  R ek = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const uint32_t sl = fslot[9 * f + 3 * a + b];
      if (sl == ~0u) continue;
      const float* blk = sl < nnz_s ? vals + 9 * (size_t)sl : valp + 9 * (size_t)(sl - nnz_s);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) ek += w[a][r] * (R)blk[3 * r + c] * w[b][c];
    }
  const M2<R> dm{(R)fdm[4 * f], (R)fdm[4 * f + 1], (R)fdm[4 * f + 2], (R)fdm[4 * f + 3]};
  V3<R> g[3];
  R h[81];
  float* o = out + 90 * (size_t)f;
  if (!sl_face_grad_hess<R>(p, dm, (R)flim[f], (R)fmass[f], ek, kind, (R)eps, g, h)) {
    for (int q = 0; q < 90; ++q) o[q] = 0.f;
    return;
  }
  for (int q = 0; q < 81; ++q) o[q] = (float)h[q];
  for (int a = 0; a < 3; ++a) {
    o[81 + 3 * a] = (float)g[a].x;
    o[82 + 3 * a] = (float)g[a].y;
    o[83 + 3 * a] = (float)g[a].z;
  }
}

// One thread per touched slot: the faces' blocks added to it in face order.
__global__ void k_sl_gather_blocks(uint32_t ns, const uint32_t* __restrict__ slots, const uint32_t* __restrict__ sptr,
                                   const uint32_t* __restrict__ slist, const float* __restrict__ c, uint32_t nnz_s,
                                   float* __restrict__ vals, float* __restrict__ valp) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns) return;
  const uint32_t sl = slots[t];
  float* blk = sl < nnz_s ? vals + 9 * (size_t)sl : valp + 9 * (size_t)(sl - nnz_s);
  float acc[9];
  for (int q = 0; q < 9; ++q) acc[q] = blk[q];
  for (uint32_t j = sptr[t]; j < sptr[t + 1]; ++j) {
    const uint32_t e = slist[j], f = e / 9, a = (e % 9) / 3, b = e % 3;
    const float* h = c + 90 * (size_t)f;
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) acc[3 * r + cc] += h[(3 * a + r) * 9 + 3 * b + cc];
  }
  for (int q = 0; q < 9; ++q) blk[q] = acc[q];
}

// One thread per touched vertex: the faces' gradient entries added in face order.
__global__ void k_sl_gather_grad(uint32_t nvt, const uint32_t* __restrict__ verts, const uint32_t* __restrict__ vptr,
                                 const uint32_t* __restrict__ vlist, const float* __restrict__ c,
                                 float* __restrict__ grad) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nvt) return;
  const uint32_t v = verts[t];
  float g0 = grad[3 * v], g1 = grad[3 * v + 1], g2 = grad[3 * v + 2];
  for (uint32_t j = vptr[t]; j < vptr[t + 1]; ++j) {
    const uint32_t e = vlist[j], f = e / 3, a = e % 3;
    const float* g = c + 90 * (size_t)f + 81 + 3 * a;
    g0 += g[0];
    g1 += g[1];
    g2 += g[2];
  }
  grad[3 * v] = g0;
  grad[3 * v + 1] = g1;
  grad[3 * v + 2] = g2;
}

static int assemble_strain_limit(Scene& s) {
  if (!s.n_sl) return MGUSO_OK;
  const unsigned g = ceil_div(s.n_sl, 128);
  if (s.mixed)
    k_sl_faces<double><<<g, 128, 0, s.st>>>(s.n_sl, s.sl_v.p, s.sl_dm.p, s.sl_limit.p, s.sl_mass.p, s.sl_slot.p,
                                            s.x.p, s.A->val.p, s.valp.p, s.Ps.nnz, s.p.barrier_kind,
                                            s.p.eiganalysis_eps, s.sl_c.p);
  else
    k_sl_faces<float><<<g, 128, 0, s.st>>>(s.n_sl, s.sl_v.p, s.sl_dm.p, s.sl_limit.p, s.sl_mass.p, s.sl_slot.p,
                                           s.x.p, s.A->val.p, s.valp.p, s.Ps.nnz, s.p.barrier_kind,
                                           s.p.eiganalysis_eps, s.sl_c.p);
  if (s.n_sl_slots)
    k_sl_gather_blocks<<<ceil_div(s.n_sl_slots, 128), 128, 0, s.st>>>(s.n_sl_slots, s.sl_slots.p, s.sl_sptr.p,
                                                                      s.sl_slist.p, s.sl_c.p, s.Ps.nnz, s.A->val.p,
                                                                      s.valp.p);
  k_sl_gather_grad<<<ceil_div(s.n_sl_verts, 128), 128, 0, s.st>>>(s.n_sl_verts, s.sl_verts.p, s.sl_vptr.p,
                                                                  s.sl_vlist.p, s.sl_c.p, s.grad.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int assemble_colliders(Scene& s) {
  MG_TRY(assemble_strain_limit(s));
  MG_TRY(assemble_pins(s));
  if (!s.n_col || !s.n_free) return MGUSO_OK;
  unsigned g = ceil_div(s.n_free, 128);
  float mu = s.p.friction;  // collider friction unset: the vertex coefficient stands
  if (s.mixed)
    k_colliders<double><<<g, 128, 0, s.st>>>(s.free_verts.p, s.n_free, s.inv_mass.p, s.x.p, s.x0.p, s.colliders.p,
                                             s.n_col, s.diag_slot.p, s.A->val.p, s.grad.p, s.p.contact_dhat,
                                             s.p.contact_kappa, s.p.contact_dynamic, s.p.barrier_kind,
                                             s.p.contact_rayleigh, mu, s.p.friction_eps);
  else
    k_colliders<float><<<g, 128, 0, s.st>>>(s.free_verts.p, s.n_free, s.inv_mass.p, s.x.p, s.x0.p, s.colliders.p,
                                            s.n_col, s.diag_slot.p, s.A->val.p, s.grad.p, s.p.contact_dhat,
                                            s.p.contact_kappa, s.p.contact_dynamic, s.p.barrier_kind,
                                            s.p.contact_rayleigh, mu, s.p.friction_eps);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// ---- self contact ------------------------------------------------------------------------------
// block (va, vb) of the gathered (pre-contact) Hessian: Ps when both vertices are free,
// else Pp; absent blocks read as zero.
__device__ __forceinline__ const float* find_block(uint32_t va, uint32_t vb, const uint8_t* pinned,
                                                   const uint32_t* ps_rp, const uint32_t* ps_col, const float* vals,
                                                   const uint32_t* pp_rp, const uint32_t* pp_col, const float* valp) {
  bool sys = !pinned[va] && !pinned[vb];
  const uint32_t* rp = sys ? ps_rp : pp_rp;
  const uint32_t* cl = sys ? ps_col : pp_col;
  uint32_t lo = rp[va], hi = rp[va + 1];
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (cl[mid] < vb)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < rp[va + 1] && cl[lo] == vb) return (sys ? vals : valp) + 9 * (size_t)lo;
  return nullptr;
}

constexpr unsigned long long INVALID_KEY = ~0ull;

// self_contact_rayleigh (implicit.rs:755-795): a stencil's barrier stiffness from the
// gathered blocks of its participants and their masses (kappa when the normal degenerates).
// km, when given, receives the masses' part of it, sum m w^2 / d^2 (its only part that
// depends on the gap d).
template <class R>
__device__ inline R stencil_stiffness(const Stencil& S, const V3<R> g[4], const float* __restrict__ im,
                                      const uint8_t* __restrict__ pinned, const uint32_t* __restrict__ ps_rp,
                                      const uint32_t* __restrict__ ps_col, const float* __restrict__ vals,
                                      const uint32_t* __restrict__ pp_rp, const uint32_t* __restrict__ pp_col,
                                      const float* __restrict__ valp, float kappa, R* km) {
  const R d = (R)S.d;
  if (km) *km = R(0);
  const R nlen = g[0].length();
  if (nlen < R(1.0e-12)) return (R)kappa;
  V3<R> nrm = g[0] / nlen;
  R wts[4], mass[4];
  R el[16][9];
  for (int a = 0; a < 4; ++a) {
    wts[a] = g[a].dot(nrm);
    R imv = (R)im[S.idx[a]];
    mass[a] = imv > 0 ? R(1) / imv : R(0);
  }
  for (int ia = 0; ia < 4; ++ia)
    for (int ib = 0; ib < 4; ++ib) {
      const float* b = find_block(S.idx[ia], S.idx[ib], pinned, ps_rp, ps_col, vals, pp_rp, pp_col, valp);
      for (int q = 0; q < 9; ++q) el[ia * 4 + ib][q] = b ? (R)b[q] : R(0);
    }
  R k = rayleigh_stiffness<R>(el, mass, wts, 4, nrm * d);
  if (!(k > 0)) return (R)kappa;
  if (km) {
    R m_max = 0, ws = 0, acc = 0;
    for (int a = 0; a < 4; ++a) m_max = rmax(m_max, mass[a]);
    for (int a = 0; a < 4; ++a) {
      ws += wts[a] * wts[a];
      acc += (mass[a] > 0 ? mass[a] : m_max) * wts[a] * wts[a];
    }
    *km = ws > 0 ? acc / ws / (d * d) : R(0);
  }
  return k;
}

template <class R>
__global__ void k_contact_assemble(const Stencil* __restrict__ sts, uint32_t nst, const float* __restrict__ im,
                                   const uint8_t* __restrict__ pinned, const float* __restrict__ x,
                                   const float* __restrict__ x_start, const uint32_t* __restrict__ ps_rp,
                                   const uint32_t* __restrict__ ps_col, const float* __restrict__ vals,
                                   const uint32_t* __restrict__ pp_rp, const uint32_t* __restrict__ pp_col,
                                   const float* __restrict__ valp, float kappa, int barrier_kind, float mu, float feps,
                                   const float* __restrict__ kin_dx, float* __restrict__ ccb,
                                   unsigned long long* __restrict__ ckeys,
                                   uint32_t* __restrict__ cids, float* __restrict__ cge,
                                   unsigned long long* __restrict__ gkeys, uint32_t* __restrict__ gids) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  const Stencil& S = sts[s];
  V3<R> g[4];
  for (int a = 0; a < 4; ++a) g[a] = V3<R>((R)S.g[3 * a], (R)S.g[3 * a + 1], (R)S.g[3 * a + 2]);
  R d = (R)S.d;
  const R k = stencil_stiffness<R>(S, g, im, pinned, ps_rp, ps_col, vals, pp_rp, pp_col, valp, kappa, (R*)nullptr);
  R nlen = g[0].length();
  int kind = d < 0 ? 1 : barrier_kind;
  R bg = 0, bh = 0;
  bool active = barrier_of<R>(kind, d, (R)S.ghat, k, bg, bh);
  R hp = rmax(bh, R(0));
  // friction (stencil_friction, contact.rs:659-705)
  bool fr = false;
  V3<R> fg;
  R fh[9];
  R w[4];
  if (active && mu > 0 && nlen >= R(1.0e-12)) {
    V3<R> n = g[0] / nlen;
    V3<R> slip;
    for (int a = 0; a < 4; ++a) {
      w[a] = g[a].dot(n);
      // the slip is relative: a re-posed collider vertex adds the move it was given before
      // this step (fdx_override, implicit.rs:3063-3078)
      V3<R> dxa = ld3<R>(x, S.idx[a]) - ld3<R>(x_start, S.idx[a]);
      if (kin_dx) dxa += ld3<R>(kin_dx, S.idx[a]);
      slip += dxa * w[a];
    }
    fr = friction<R>(n * bg, slip, n, (R)mu, (R)feps, fg, fh);
    if (fr && fg.x == 0 && fg.y == 0 && fg.z == 0) fr = false;
  }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      uint32_t ra = S.idx[a], cbv = S.idx[b];
      bool keep = !pinned[ra] && !pinned[cbv];
      size_t id = 32 * (size_t)s + 4 * a + b;
      float* o = ccb + 9 * id;
      bool any = false;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          float vh = active ? (float)(hp * g[a][r] * g[b][c]) : 0.f;
          o[3 * r + c] = vh;
          any = any || vh != 0.f;
        }
      ckeys[id] = (keep && any) ? (((unsigned long long)ra << 32) | cbv) : INVALID_KEY;
      cids[id] = (uint32_t)id;
      size_t id2 = id + 16;
      float* o2 = ccb + 9 * id2;
      bool any2 = false;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          float vh = fr ? (float)(w[a] * w[b] * fh[3 * r + c]) : 0.f;
          if (fr && w[a] * w[b] == 0) vh = 0.f;
          o2[3 * r + c] = vh;
          any2 = any2 || vh != 0.f;
        }
      ckeys[id2] = (keep && any2) ? (((unsigned long long)ra << 32) | cbv) : INVALID_KEY;
      cids[id2] = (uint32_t)id2;
    }
  for (int a = 0; a < 4; ++a) {
    size_t id = 8 * (size_t)s + a;
    V3<R> gb = g[a] * bg;
    cge[3 * id] = active ? (float)gb.x : 0.f;
    cge[3 * id + 1] = active ? (float)gb.y : 0.f;
    cge[3 * id + 2] = active ? (float)gb.z : 0.f;
    gkeys[id] = active ? S.idx[a] : INVALID_KEY;
    gids[id] = (uint32_t)id;
    size_t id2 = id + 4;
    V3<R> ff = fr ? fg * w[a] : V3<R>();
    cge[3 * id2] = (float)ff.x;
    cge[3 * id2 + 1] = (float)ff.y;
    cge[3 * id2 + 2] = (float)ff.z;
    gkeys[id2] = fr ? S.idx[a] : INVALID_KEY;
    gids[id2] = (uint32_t)id2;
  }
}

// The stencils' stiffnesses and their mass parts, 2 per stencil, as the step's assembly
// computes them from the gathered (projected) blocks.
template <class R>
__global__ void k_contact_stiffness(const Stencil* __restrict__ sts, uint32_t nst, const float* __restrict__ im,
                                    const uint8_t* __restrict__ pinned, const uint32_t* __restrict__ ps_rp,
                                    const uint32_t* __restrict__ ps_col, const float* __restrict__ vals,
                                    const uint32_t* __restrict__ pp_rp, const uint32_t* __restrict__ pp_col,
                                    const float* __restrict__ valp, float kappa, double* __restrict__ out) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  const Stencil& S = sts[s];
  V3<R> g[4];
  for (int a = 0; a < 4; ++a) g[a] = V3<R>((R)S.g[3 * a], (R)S.g[3 * a + 1], (R)S.g[3 * a + 2]);
  R km;
  R k = stencil_stiffness<R>(S, g, im, pinned, ps_rp, ps_col, vals, pp_rp, pp_col, valp, kappa, &km);
  out[2 * (size_t)s] = (double)k;
  out[2 * (size_t)s + 1] = (double)km;
}

// the stencil's gap and its gradient in FP64 at positions p (the signed vertex-triangle
// gap of a static collider triangle keeps the sign it had, `inside`)
__device__ inline double stencil_gap(uint32_t kind, bool inside, const V3<double> p[4], double g[12]) {
  V3<double> gg[4];
  double d = kind == 0 ? point_tri_distance_grad<double>(p[0], p[1], p[2], p[3], inside, gg)
                       : segment_segment_distance_grad<double>(p[0], p[1], p[2], p[3], gg);
  for (int a = 0; a < 4; ++a)
    for (int c = 0; c < 3; ++c) g[3 * a + c] = gg[a][c];
  return d;
}

// The exact Hessian of a stencil's barrier term b'(d; k(d)) grad d with the stiffness
// recorded by k_contact_stiffness: (b'' + b'/k dk/dd) grad d grad d^T + b' hess d, where
// dk/dd = -2 km / d (the stiffness's mass part goes as 1/d^2; its elastic part is held
// fixed) and hess d comes from FP64 central differences of the gap's gradient. Outputs as
// k_contact_assemble (no friction: the adjoint takes frictionless scenes).
__global__ void k_contact_exact(const Stencil* __restrict__ sts, uint32_t nst, const uint8_t* __restrict__ pinned,
                                const float* __restrict__ x, const double* __restrict__ kst, int barrier_kind,
                                float* __restrict__ ccb, unsigned long long* __restrict__ ckeys,
                                uint32_t* __restrict__ cids, float* __restrict__ cge,
                                unsigned long long* __restrict__ gkeys, uint32_t* __restrict__ gids) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  const Stencil& S = sts[s];
  const double d = S.d, k = kst[2 * (size_t)s], km = kst[2 * (size_t)s + 1];
  int kind = d < 0 ? 1 : barrier_kind;
  double bg = 0, bh = 0;
  bool active = barrier_of<double>(kind, d, S.ghat, k, bg, bh);
  double H[144];
  for (int q = 0; q < 144; ++q) H[q] = 0;
  if (active) {
    const double dkdd = d != 0 ? -2.0 * km / d : 0.0;
    const double coef = bh + bg / k * dkdd;
    for (int i = 0; i < 12; ++i)
      for (int j = 0; j < 12; ++j) H[12 * i + j] = coef * S.g[i] * S.g[j];
    V3<double> p[4];
    for (int a = 0; a < 4; ++a) p[a] = ld3<double>(x, S.idx[a]);
    // a small step: the gap gradient of nearly parallel edges (a seam's two sides) changes
    // region within 1e-4 |d|, and a difference across that switch is no derivative
    const double eps = fmax(1e-6 * fabs(d), 1e-12);
    const bool inside = d < 0;
    for (int i = 0; i < 12; ++i) {
      double gp[12], gm[12];
      V3<double> q[4] = {p[0], p[1], p[2], p[3]};
      q[i / 3][i % 3] = p[i / 3][i % 3] + eps;
      stencil_gap(S.kind, inside, q, gp);
      q[i / 3][i % 3] = p[i / 3][i % 3] - eps;
      stencil_gap(S.kind, inside, q, gm);
      for (int j = 0; j < 12; ++j) {
        const double hij = 0.5 * bg * (gp[j] - gm[j]) / (2 * eps);
        H[12 * i + j] += hij;
        H[12 * j + i] += hij;
      }
    }
  }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      uint32_t ra = S.idx[a], cbv = S.idx[b];
      bool keep = !pinned[ra] && !pinned[cbv];
      size_t id = 32 * (size_t)s + 4 * a + b;
      float* o = ccb + 9 * id;
      bool any = false;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          float vh = (float)H[12 * (3 * a + r) + 3 * b + c];
          o[3 * r + c] = vh;
          any = any || vh != 0.f;
        }
      ckeys[id] = (keep && any) ? (((unsigned long long)ra << 32) | cbv) : INVALID_KEY;
      cids[id] = (uint32_t)id;
      size_t id2 = id + 16;
      for (int q = 0; q < 9; ++q) ccb[9 * id2 + q] = 0.f;
      ckeys[id2] = INVALID_KEY;
      cids[id2] = (uint32_t)id2;
    }
  for (int a = 0; a < 4; ++a) {
    size_t id = 8 * (size_t)s + a;
    for (int c = 0; c < 3; ++c) cge[3 * id + c] = active ? (float)(S.g[3 * a + c] * bg) : 0.f;
    gkeys[id] = active ? S.idx[a] : INVALID_KEY;
    gids[id] = (uint32_t)id;
    size_t id2 = id + 4;
    for (int c = 0; c < 3; ++c) cge[3 * id2 + c] = 0.f;
    gkeys[id2] = INVALID_KEY;
    gids[id2] = (uint32_t)id2;
  }
}

int contact_stiffness(Scene& s, uint32_t nst) {
  if (nst == 0) return MGUSO_OK;
  MG_TRY(s.contact_k.grow(2 * (size_t)nst));
  unsigned g = ceil_div(nst, 64);
  if (s.mixed)
    k_contact_stiffness<double><<<g, 64, 0, s.st>>>(s.stencils_sorted.p, nst, s.inv_mass.p, s.pinned.p,
                                                    s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.Pp.row_ptr.p,
                                                    s.Pp.col.p, s.valp.p, s.p.contact_kappa, s.contact_k.p);
  else
    k_contact_stiffness<float><<<g, 64, 0, s.st>>>(s.stencils_sorted.p, nst, s.inv_mass.p, s.pinned.p,
                                                   s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.Pp.row_ptr.p,
                                                   s.Pp.col.p, s.valp.p, s.p.contact_kappa, s.contact_k.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// Segment heads of the sorted block keys: add onto Ps when the block exists there, else
// flag a new C entry (rank computed by the scan below).
__global__ void k_contact_heads(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ ids,
                                uint32_t m, const float* __restrict__ ccb, const uint32_t* __restrict__ ps_rp,
                                const uint32_t* __restrict__ ps_col, float* __restrict__ vals,
                                uint32_t* __restrict__ is_new) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  unsigned long long k = keys[i];
  bool head = k != INVALID_KEY && (i == 0 || keys[i - 1] != k);
  is_new[i] = 0;
  if (!head) return;
  uint32_t r = (uint32_t)(k >> 32), c = (uint32_t)k;
  uint32_t lo = ps_rp[r], hi = ps_rp[r + 1];
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (ps_col[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < ps_rp[r + 1] && ps_col[lo] == c) {
    float* v = vals + 9 * (size_t)lo;
    float a[9];
    for (int q = 0; q < 9; ++q) a[q] = v[q];
    for (uint32_t j = i; j < m && keys[j] == k; ++j) {
      const float* cc = ccb + 9 * (size_t)ids[j];
      for (int q = 0; q < 9; ++q)
        if (cc[q] != 0.f) a[q] += cc[q];
    }
    for (int q = 0; q < 9; ++q) v[q] = a[q];
  } else {
    is_new[i] = 1;
  }
}

__global__ void k_contact_new(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ ids,
                              uint32_t m, const float* __restrict__ ccb, const uint32_t* __restrict__ is_new,
                              const uint32_t* __restrict__ rank, uint32_t* __restrict__ c_row,
                              uint32_t* __restrict__ c_col, float* __restrict__ c_val) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || !is_new[i]) return;
  unsigned long long k = keys[i];
  uint32_t o = rank[i];
  float a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t j = i; j < m && keys[j] == k; ++j) {
    const float* cc = ccb + 9 * (size_t)ids[j];
    for (int q = 0; q < 9; ++q)
      if (cc[q] != 0.f) a[q] += cc[q];
  }
  c_row[o] = (uint32_t)(k >> 32);
  c_col[o] = (uint32_t)k;
  for (int q = 0; q < 9; ++q) c_val[9 * (size_t)o + q] = a[q];
}

__global__ void k_row_ptr_from_sorted(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ count,
                                      uint32_t nv, uint32_t* __restrict__ row_ptr) {
  uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > nv) return;
  uint32_t n = *count;
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (rows[mid] < r)
      lo = mid + 1;
    else
      hi = mid;
  }
  row_ptr[r] = lo;
}

__global__ void k_contact_grad(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ ids,
                               uint32_t m, const float* __restrict__ cge, float* __restrict__ grad) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  unsigned long long k = keys[i];
  if (k == INVALID_KEY || (i > 0 && keys[i - 1] == k)) return;
  uint32_t v = (uint32_t)k;
  float a0 = grad[3 * v], a1 = grad[3 * v + 1], a2 = grad[3 * v + 2];
  for (uint32_t j = i; j < m && keys[j] == k; ++j) {
    const float* g = cge + 3 * (size_t)ids[j];
    a0 += g[0];
    a1 += g[1];
    a2 += g[2];
  }
  grad[3 * v] = a0;
  grad[3 * v + 1] = a1;
  grad[3 * v + 2] = a2;
}

// exclusive scan of u32 flags (n <= 2^30), three passes
__global__ void k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                             uint32_t* __restrict__ block_sums) {
  __shared__ uint32_t s[1024];
  uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  uint32_t v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (uint32_t o = 1; o < 1024; o <<= 1) {
    uint32_t t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) block_sums[blockIdx.x] = s[1023];
}

__global__ void k_scan_sums(uint32_t* __restrict__ sums, uint32_t nb, uint32_t* __restrict__ total) {
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t b = 0; b < nb; ++b) {
      uint32_t v = sums[b];
      sums[b] = acc;
      acc += v;
    }
    *total = acc;
  }
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t n, const uint32_t* __restrict__ sums) {
  uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += sums[blockIdx.x];
}

static int scan_u32(Scene& s, const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total, DevBuf<uint32_t>& tmp) {
  uint32_t nb = std::max<uint32_t>(ceil_div(n, 1024), 1);
  MG_TRY(tmp.grow(nb + 1));
  if (n) k_scan_block<<<nb, 1024, 0, s.st>>>(in, out, n, tmp.p);
  else MG_CUDA(cudaMemsetAsync(tmp.p, 0, 4, s.st));
  k_scan_sums<<<1, 32, 0, s.st>>>(tmp.p, n ? nb : 1, total);
  if (n) k_scan_add<<<nb, 1024, 0, s.st>>>(out, n, tmp.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int assemble_contacts(Scene& s, uint32_t nst) {
  cudaStream_t st = s.st;
  // C starts empty every iteration
  MG_CUDA(cudaMemsetAsync(s.c_count.p, 0, 4, st));
  if (nst == 0) {
    MG_CUDA(cudaMemsetAsync(s.c_row_ptr.p, 0, 4 * ((size_t)s.nv + 1), st));
    return MGUSO_OK;
  }
  const uint32_t mb = 32 * nst, mg_ = 8 * nst;
  MG_TRY(s.ccblocks.grow(9 * (size_t)mb));
  MG_TRY(s.ckeys.grow(mb));
  MG_TRY(s.cids.grow(mb));
  MG_TRY(s.cgentries.grow(3 * (size_t)mg_));
  MG_TRY(s.gkeys.grow(mg_));
  MG_TRY(s.gids.grow(mg_));
  unsigned g = ceil_div(nst, 64);
  if (s.hess_mode == 2 && (s.exact_terms & EXACT_CONTACTS))
    k_contact_exact<<<g, 64, 0, st>>>(s.stencils_sorted.p, nst, s.pinned.p, s.x.p, s.contact_k.p, s.p.barrier_kind,
                                      s.ccblocks.p, s.ckeys.p, s.cids.p, s.cgentries.p, s.gkeys.p, s.gids.p);
  else if (s.mixed)
    k_contact_assemble<double><<<g, 64, 0, st>>>(s.stencils_sorted.p, nst, s.inv_mass.p, s.pinned.p, s.x.p, s.x0.p,
                                                 s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.Pp.row_ptr.p, s.Pp.col.p,
                                                 s.valp.p, s.p.contact_kappa, s.p.barrier_kind, s.p.friction,
                                                 s.p.friction_eps, s.kin_dx_set ? s.kin_dx.p : nullptr, s.ccblocks.p,
                                                 s.ckeys.p, s.cids.p, s.cgentries.p, s.gkeys.p, s.gids.p);
  else
    k_contact_assemble<float><<<g, 64, 0, st>>>(s.stencils_sorted.p, nst, s.inv_mass.p, s.pinned.p, s.x.p, s.x0.p,
                                                s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.Pp.row_ptr.p, s.Pp.col.p,
                                                s.valp.p, s.p.contact_kappa, s.p.barrier_kind, s.p.friction,
                                                s.p.friction_eps, s.kin_dx_set ? s.kin_dx.p : nullptr, s.ccblocks.p,
                                                s.ckeys.p, s.cids.p, s.cgentries.p, s.gkeys.p, s.gids.p);
  MG_CUDA(cudaGetLastError());
  // blocks: stable sort by (row, col); stencil order survives within equal keys
  MG_TRY(radix_sort_pairs(&s.sorter, s.ckeys.p, s.cids.p, mb, 64, st));
  DevBuf<uint32_t>& is_new = s.is_new;
  DevBuf<uint32_t>& rank = s.rank;
  DevBuf<uint32_t>& tmp = s.scan_tmp;
  MG_TRY(is_new.grow(mb));
  MG_TRY(rank.grow(mb));
  k_contact_heads<<<ceil_div(mb, 256), 256, 0, st>>>(s.ckeys.p, s.cids.p, mb, s.ccblocks.p, s.Ps.row_ptr.p,
                                                    s.Ps.col.p, s.A->val.p, is_new.p);
  MG_TRY(scan_u32(s, is_new.p, rank.p, mb, s.c_count.p, tmp));
  // C has at most one block per stencil block: sized by that bound, its count (c_count)
  // stays on the device
  if (mb > s.cap_c || !s.c_col.p) {
    s.cap_c = std::max(mb, 2 * s.cap_c);
    s.work.drop_graph();
  }
  MG_TRY(s.c_row.reserve(s.cap_c));
  MG_TRY(s.c_col.reserve(s.cap_c));
  MG_TRY(s.c_val.reserve(9 * (size_t)s.cap_c));
  k_contact_new<<<ceil_div(mb, 256), 256, 0, st>>>(s.ckeys.p, s.cids.p, mb, s.ccblocks.p, is_new.p, rank.p,
                                                  s.c_row.p, s.c_col.p, s.c_val.p);
  k_row_ptr_from_sorted<<<ceil_div(s.nv + 1, 256), 256, 0, st>>>(s.c_row.p, s.c_count.p, s.nv, s.c_row_ptr.p);
  // gradient entries: stable sort by vertex, then add in stencil order
  MG_TRY(radix_sort_pairs(&s.sorter, s.gkeys.p, s.gids.p, mg_, 64, st));
  k_contact_grad<<<ceil_div(mg_, 256), 256, 0, st>>>(s.gkeys.p, s.gids.p, mg_, s.cgentries.p, s.grad.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

__global__ void k_rhs(const float* __restrict__ grad, const uint8_t* __restrict__ pinned, uint32_t nv,
                      float* __restrict__ rhs) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nv) return;
  rhs[i] = pinned[i / 3] ? 0.f : -grad[i];
}

int finish_rhs(Scene& s) {
  k_rhs<<<ceil_div(3 * s.nv, 256), 256, 0, s.st>>>(s.grad.p, s.pinned.p, s.nv, s.work.b.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// y = (Ps + C) x over every block row in one pass, accumulated in Acc, then the fused
// dot(x, y). In mixed precision Acc is FP64: products of FP32 values are exact there, so
// the inertia term (m / h^2, ~0.04 for a 10 mg vertex) survives next to seam and barrier
// blocks of ~1e6 whose contributions cancel between neighbours. Storage stays FP32.
__device__ __forceinline__ float acc_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double acc_fma(double a, double b, double c) { return fma(a, b, c); }

// Eight lanes per block row: lane g takes blocks g, g + 8, ... of the row's fixed-pattern
// and contact lists (coalesced 288-byte runs of values), then a fixed xor tree over the
// eight lanes sums them, so the result is deterministic.
template <class Acc>
__global__ void __launch_bounds__(256) k_system_spmv(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ col,
                                                     const float* __restrict__ val, const uint32_t* __restrict__ c_rp,
                                                     const uint32_t* __restrict__ c_col,
                                                     const float* __restrict__ c_val, uint32_t nv,
                                                     const float* __restrict__ x, float* __restrict__ y, DotSink dot,
                                                     int with_dot) {
  if (with_dot && dot.sc->done) return;
  const uint32_t g = threadIdx.x & 7u;
  const unsigned gmask = 0xFFu << (threadIdx.x & 24u);
  Acc acc = 0;
  const uint32_t stride = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 3; r < nv; r += stride) {
    Acc y0 = 0, y1 = 0, y2 = 0;
    auto block = [&](const float* __restrict__ a, uint32_t c) {
      const Acc x0 = (Acc)__ldg(x + 3 * c), x1 = (Acc)__ldg(x + 3 * c + 1), x2 = (Acc)__ldg(x + 3 * c + 2);
      y0 = acc_fma((Acc)a[0], x0, y0);
      y0 = acc_fma((Acc)a[1], x1, y0);
      y0 = acc_fma((Acc)a[2], x2, y0);
      y1 = acc_fma((Acc)a[3], x0, y1);
      y1 = acc_fma((Acc)a[4], x1, y1);
      y1 = acc_fma((Acc)a[5], x2, y1);
      y2 = acc_fma((Acc)a[6], x0, y2);
      y2 = acc_fma((Acc)a[7], x1, y2);
      y2 = acc_fma((Acc)a[8], x2, y2);
    };
    const uint32_t ke = rp[r + 1];
    for (uint32_t k = rp[r] + g; k < ke; k += 8) block(val + 9 * (size_t)k, col[k]);
    const uint32_t ce = c_rp[r + 1];
    for (uint32_t k = c_rp[r] + g; k < ce; k += 8) block(c_val + 9 * (size_t)k, c_col[k]);
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      y0 += __shfl_xor_sync(gmask, y0, o, 8);
      y1 += __shfl_xor_sync(gmask, y1, o, 8);
      y2 += __shfl_xor_sync(gmask, y2, o, 8);
    }
    if (g == 0) {
      const float f0 = (float)y0, f1 = (float)y1, f2 = (float)y2;
      y[3 * r] = f0;
      y[3 * r + 1] = f1;
      y[3 * r + 2] = f2;
      acc += (Acc)x[3 * r] * (Acc)f0 + (Acc)x[3 * r + 1] * (Acc)f1 + (Acc)x[3 * r + 2] * (Acc)f2;
    }
  }
  if (with_dot) grid_dot_commit<Acc>(dot, acc);
}

int system_spmv(Scene& s, const float* p, float* ap, cudaStream_t st, const DotSink* d) {
  const int grid = (int)std::max<uint64_t>(
      1, std::min<uint64_t>(ceil_div(8ull * s.nv, 256), (uint64_t)s.ctx->sm_count * 8));
  DotSink dd = d ? *d : DotSink{};
  const uint32_t* c_col = s.c_col.p ? s.c_col.p : s.c_row_ptr.p;
  if (s.mixed)
    k_system_spmv<double><<<grid, 256, 0, st>>>(s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.c_row_ptr.p, c_col,
                                                s.c_val.p, s.nv, p, ap, dd, d ? 1 : 0);
  else
    k_system_spmv<float><<<grid, 256, 0, st>>>(s.Ps.row_ptr.p, s.Ps.col.p, s.A->val.p, s.c_row_ptr.p, c_col,
                                               s.c_val.p, s.nv, p, ap, dd, d ? 1 : 0);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

}  // namespace mg
