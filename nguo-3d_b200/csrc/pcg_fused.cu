// Fused two-kernel PCG for the Newton systems (linsolve.rs:350-411), replayed as CUDA
// graphs of 16 iterations, for systems large enough to fill the GPU (batches of drapes).
//
// Each iteration is two full-occupancy kernels:
//   rows:    p = z + beta p_old for the CTA's block rows (into the other p buffer), Ap with
//            every gathered p_j formed the same way, p.Ap; the last CTA to finish sums the
//            per-CTA partials of each instance in CTA order and sets alpha (or flags a
//            breakdown, pAp <= 0 or NaN, where the reference breaks out);
//   domains: one warp per Schwarz domain (block Jacobi: one thread per vertex) updates
//            x += alpha p, r -= alpha Ap on its rows, applies the preconditioner to them,
//            and accumulates r.r and r.z; the last CTA sets the residual, the convergence
//            flag, beta and rz.
// CTAs are partitioned by instance, so a CTA's partials belong to one instance and each
// instance's sums are deterministic. Kernels of converged instances skip their work, and a
// kernel launched after every instance converged returns at entry.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "reduce.cuh"
#include "scene.cuh"
#include "tiles.cuh"

namespace mg {

constexpr int FR_THREADS = 256;
constexpr int FD_WARPS = 4;        // Schwarz, one warp per domain: warps (domains) per CTA
constexpr int FD_THREADS = 256;    // block Jacobi: vertices per CTA
constexpr uint32_t FUSED_CHECK = 16;
constexpr int FR_BATCH = 4;  // blocks per lane whose loads the rows kernel issues together

// z and the search directions are stored with 4 floats per vertex (xyz, w unused): a
// neighbour's z and p_old are two 16-byte loads in the SpMV gather. x, r, b and Ap keep 3.
__device__ __forceinline__ uint32_t zpos(uint32_t e) { return 4 * (e / 3) + e % 3; }
__device__ __forceinline__ float4 ld_v4(const float* __restrict__ v, uint32_t i) {
  return __ldg(reinterpret_cast<const float4*>(v) + i);
}
__device__ __forceinline__ void st_v4(float* __restrict__ v, uint32_t i, float x, float y, float z) {
  reinterpret_cast<float4*>(v)[i] = make_float4(x, y, z, 0.f);
}

struct FusedArgs {
  uint32_t ninst;
  const uint32_t* lay;  // [0, K] rows, [9 ..] row-kernel CTAs, [18 ..] domain-kernel CTAs, [27 ..] domains
  const uint32_t *rp, *col;
  const float* val;
  const uint32_t *crp, *ccol;
  const float* cval;
  const float* bjinv;
  const uint32_t *dom_start, *dom_verts;
  const uint64_t* fac_off;
  const void* fac;         // float or __half tiles
  const float* fac_scale;  // per domain (FP16 tiles), else null
  const uint8_t* dom_diag;  // block-diagonal domains (per-vertex factors in vfac)
  const float* vfac;
  const uint32_t *sell_base, *sell_inst, *sell_col;  // SELL rows variant
  const float* sell_val;
  const float* b;
  float *x, *r, *z, *ap;
  float tol;
  uint32_t max_iter;
  FusedInst* inst;
  FusedCtl* ctl;
  double* part;  // row kernel: [cta]; domain kernel: [2 * cta + j]
};

constexpr int LAY = PCG_MAX_INST + 1;

__device__ __forceinline__ float fr_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fr_fma(double a, double b, double c) { return fma(a, b, c); }

__device__ __forceinline__ int cta_instance(const uint32_t* cta, uint32_t K) {
  int k = 0;
  while (k + 1 < (int)K && blockIdx.x >= __ldg(cta + k + 1)) ++k;
  return k;
}

// The last CTA of the grid to arrive returns true (after a fence, so all partials are visible).
__device__ __forceinline__ bool last_cta(uint32_t* counter) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// finish of the rows kernel: alpha per instance, partials summed in CTA order
__device__ __forceinline__ void rows_finish(const FusedArgs& a) {
  const uint32_t K = a.ninst;
  const int tid = threadIdx.x, lane = tid & 31;
  const int w = tid >> 5;
  for (uint32_t q = w; q < K; q += FR_THREADS / 32) {
    const uint32_t cb = a.lay[LAY + q], ce = a.lay[LAY + q + 1];
    double t = 0;
    for (uint32_t c = cb + lane; c < ce; c += 32) t += ((volatile double*)a.part)[c];
    t = warp_sum(t);
    if (lane == 0) {
      FusedInst& I = a.inst[q];
      I.upd = 0;
      if (!I.done) {
        if (!(t > 0.0)) {
          I.done = 1;
          I.status |= ST_PCG_BREAKDOWN;
        } else {
          I.alpha = I.rz / t;
          I.upd = 1;
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    a.ctl->counter[0] = 0;
    __threadfence();
  }
}

template <class Acc, int FR_LPR>
__global__ void __launch_bounds__(FR_THREADS) k_fr_rows(FusedArgs a, const float* __restrict__ po,
                                                        float* __restrict__ pn) {
  if (a.ctl->all_done) return;
  const uint32_t K = a.ninst;
  const int k = cta_instance(a.lay + LAY, K);
  const uint32_t c0 = __ldg(a.lay + LAY + k), nc = __ldg(a.lay + LAY + k + 1) - c0, lc = blockIdx.x - c0;
  const uint32_t row0 = __ldg(a.lay + k), row1 = __ldg(a.lay + k + 1);
  const bool done = a.inst[k].done != 0;
  const float be = (float)a.inst[k].beta;
  const int tid = threadIdx.x, lane = tid & 31;
  const uint32_t sub = tid % FR_LPR;
  const unsigned gmask = ((1u << FR_LPR) - 1u) << (lane & ~(FR_LPR - 1));
  Acc acc = 0;
  if (!done) {
    for (uint32_t row = row0 + (lc * FR_THREADS + tid) / FR_LPR; row < row1; row += nc * FR_THREADS / FR_LPR) {
      Acc y0 = 0, y1 = 0, y2 = 0;
      auto block_x = [&](const float* __restrict__ m9, const float4& zc, const float4& pc4) {
        const Acc x0 = (Acc)fmaf(be, pc4.x, zc.x);
        const Acc x1 = (Acc)fmaf(be, pc4.y, zc.y);
        const Acc x2 = (Acc)fmaf(be, pc4.z, zc.z);
        y0 = fr_fma((Acc)__ldg(m9 + 0), x0, y0);
        y0 = fr_fma((Acc)__ldg(m9 + 1), x1, y0);
        y0 = fr_fma((Acc)__ldg(m9 + 2), x2, y0);
        y1 = fr_fma((Acc)__ldg(m9 + 3), x0, y1);
        y1 = fr_fma((Acc)__ldg(m9 + 4), x1, y1);
        y1 = fr_fma((Acc)__ldg(m9 + 5), x2, y1);
        y2 = fr_fma((Acc)__ldg(m9 + 6), x0, y2);
        y2 = fr_fma((Acc)__ldg(m9 + 7), x1, y2);
        y2 = fr_fma((Acc)__ldg(m9 + 8), x2, y2);
      };
      auto block = [&](const float* __restrict__ m9, uint32_t c) { block_x(m9, ld_v4(a.z, c), ld_v4(po, c)); };
      const uint32_t ke = __ldg(a.rp + row + 1);
      // the row's blocks in batches of FR_BATCH per lane: every column, then every gather,
      // issued before the first product (the same blocks in the same order as one at a time)
      for (uint32_t kk = __ldg(a.rp + row) + sub; kk < ke; kk += FR_BATCH * FR_LPR) {
        uint32_t cc[FR_BATCH];
        bool ok[FR_BATCH];
#pragma unroll
        for (int u = 0; u < FR_BATCH; ++u) {
          ok[u] = kk + u * FR_LPR < ke;
          cc[u] = ok[u] ? __ldg(a.col + kk + u * FR_LPR) : row;
        }
        float4 zz[FR_BATCH], pp[FR_BATCH];
#pragma unroll
        for (int u = 0; u < FR_BATCH; ++u) {
          zz[u] = ld_v4(a.z, cc[u]);
          pp[u] = ld_v4(po, cc[u]);
        }
#pragma unroll
        for (int u = 0; u < FR_BATCH; ++u)
          if (ok[u]) block_x(a.val + 9 * (size_t)(kk + u * FR_LPR), zz[u], pp[u]);
      }
      const uint32_t ce = __ldg(a.crp + row + 1);
      for (uint32_t kk = __ldg(a.crp + row) + sub; kk < ce; kk += FR_LPR) block(a.cval + 9 * (size_t)kk, __ldg(a.ccol + kk));
#pragma unroll
      for (int o = FR_LPR / 2; o > 0; o >>= 1) {
        y0 += __shfl_xor_sync(gmask, y0, o, FR_LPR);
        y1 += __shfl_xor_sync(gmask, y1, o, FR_LPR);
        y2 += __shfl_xor_sync(gmask, y2, o, FR_LPR);
      }
      if (sub == 0) {
        const float f0 = (float)y0, f1 = (float)y1, f2 = (float)y2;
        const float4 zr = ld_v4(a.z, row), pr = ld_v4(po, row);
        const float q0 = fmaf(be, pr.x, zr.x);
        const float q1 = fmaf(be, pr.y, zr.y);
        const float q2 = fmaf(be, pr.z, zr.z);
        st_v4(pn, row, q0, q1, q2);
        a.ap[3 * row] = f0;
        a.ap[3 * row + 1] = f1;
        a.ap[3 * row + 2] = f2;
        acc += (Acc)q0 * (Acc)f0 + (Acc)q1 * (Acc)f1 + (Acc)q2 * (Acc)f2;
      }
    }
  }
  const Acc s = block_sum<Acc>(acc);
  if (tid == 0) a.part[blockIdx.x] = (double)s;
  if (!last_cta(&a.ctl->counter[0])) return;
  rows_finish(a);
}

// Rows kernel over the sliced-ELL copy of Ps: one warp per slice of 32 rows, one lane per
// row; each slot's column and nine values are read as coalesced 128-byte rows of the slice
// (padding slots have zero values and the row's own column), then the row's contact blocks.
// Same iteration and finish as k_fr_rows.
template <class Acc>
__global__ void __launch_bounds__(FR_THREADS, 4) k_fr_rows_sell(FusedArgs a, const float* __restrict__ po,
                                                             float* __restrict__ pn) {
  if (a.ctl->all_done) return;
  const uint32_t K = a.ninst;
  const int k = cta_instance(a.lay + LAY, K);
  const uint32_t c0 = __ldg(a.lay + LAY + k), lc = blockIdx.x - c0;
  const uint32_t row0 = __ldg(a.lay + k), row1 = __ldg(a.lay + k + 1);
  const bool done = a.inst[k].done != 0;
  const float be = (float)a.inst[k].beta;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  Acc acc = 0;
  const uint32_t sl = lc * (FR_THREADS / 32) + w;  // slice within the instance
  const uint32_t row = row0 + 32 * sl + lane;
  if (!done && row0 + 32 * sl < row1) {
    const uint32_t gs = __ldg(a.sell_inst + k) + sl;
    const uint32_t b0 = __ldg(a.sell_base + gs), b1 = __ldg(a.sell_base + gs + 1);
    Acc y0 = 0, y1 = 0, y2 = 0;
    auto gather = [&](uint32_t c, Acc& x0, Acc& x1, Acc& x2) {
      const float4 zc = ld_v4(a.z, c), pc4 = ld_v4(po, c);
      x0 = (Acc)fmaf(be, pc4.x, zc.x);
      x1 = (Acc)fmaf(be, pc4.y, zc.y);
      x2 = (Acc)fmaf(be, pc4.z, zc.z);
    };
    if (row < row1) {
      // the slice's slots in pairs: both columns, then both gathers, then the products (the
      // same slots in the same order as one at a time)
      for (uint32_t b = b0; b < b1; b += 2) {
        const bool two = b + 1 < b1;
        const uint32_t cA = __ldg(a.sell_col + 32 * (size_t)b + lane);
        const uint32_t cB = two ? __ldg(a.sell_col + 32 * (size_t)(b + 1) + lane) : cA;
        const float4 zA = ld_v4(a.z, cA), pA = ld_v4(po, cA), zB = ld_v4(a.z, cB), pB = ld_v4(po, cB);
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (u == 1 && !two) break;
          const float* m = a.sell_val + 288 * (size_t)(b + u) + lane;
          const float4& zc = u ? zB : zA;
          const float4& pc4 = u ? pB : pA;
          const Acc x0 = (Acc)fmaf(be, pc4.x, zc.x);
          const Acc x1 = (Acc)fmaf(be, pc4.y, zc.y);
          const Acc x2 = (Acc)fmaf(be, pc4.z, zc.z);
          y0 = fr_fma((Acc)__ldcs(m + 0), x0, y0);
          y0 = fr_fma((Acc)__ldcs(m + 32), x1, y0);
          y0 = fr_fma((Acc)__ldcs(m + 64), x2, y0);
          y1 = fr_fma((Acc)__ldcs(m + 96), x0, y1);
          y1 = fr_fma((Acc)__ldcs(m + 128), x1, y1);
          y1 = fr_fma((Acc)__ldcs(m + 160), x2, y1);
          y2 = fr_fma((Acc)__ldcs(m + 192), x0, y2);
          y2 = fr_fma((Acc)__ldcs(m + 224), x1, y2);
          y2 = fr_fma((Acc)__ldcs(m + 256), x2, y2);
        }
      }
      const uint32_t ce = __ldg(a.crp + row + 1);
      for (uint32_t kk = __ldg(a.crp + row); kk < ce; ++kk) {
        const float* m9 = a.cval + 9 * (size_t)kk;
        Acc x0, x1, x2;
        gather(__ldg(a.ccol + kk), x0, x1, x2);
        y0 = fr_fma((Acc)__ldg(m9 + 0), x0, y0);
        y0 = fr_fma((Acc)__ldg(m9 + 1), x1, y0);
        y0 = fr_fma((Acc)__ldg(m9 + 2), x2, y0);
        y1 = fr_fma((Acc)__ldg(m9 + 3), x0, y1);
        y1 = fr_fma((Acc)__ldg(m9 + 4), x1, y1);
        y1 = fr_fma((Acc)__ldg(m9 + 5), x2, y1);
        y2 = fr_fma((Acc)__ldg(m9 + 6), x0, y2);
        y2 = fr_fma((Acc)__ldg(m9 + 7), x1, y2);
        y2 = fr_fma((Acc)__ldg(m9 + 8), x2, y2);
      }
      const float f0 = (float)y0, f1 = (float)y1, f2 = (float)y2;
      const float4 zr = ld_v4(a.z, row), pr = ld_v4(po, row);
      const float q0 = fmaf(be, pr.x, zr.x);
      const float q1 = fmaf(be, pr.y, zr.y);
      const float q2 = fmaf(be, pr.z, zr.z);
      st_v4(pn, row, q0, q1, q2);
      a.ap[3 * row] = f0;
      a.ap[3 * row + 1] = f1;
      a.ap[3 * row + 2] = f2;
      acc = (Acc)q0 * (Acc)f0 + (Acc)q1 * (Acc)f1 + (Acc)q2 * (Acc)f2;
    }
  }
  const Acc s = block_sum<Acc>(acc);
  if (tid == 0) a.part[blockIdx.x] = (double)s;
  if (!last_cta(&a.ctl->counter[0])) return;
  rows_finish(a);
}

// Ps values into the sliced-ELL copy (after every assembly; padding slots stay zero)
__global__ void k_sell_pack(const float* __restrict__ val, const uint32_t* __restrict__ pos, uint32_t nnz,
                            float* __restrict__ sv, const uint8_t* __restrict__ slot_inst, uint32_t active) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 9 * nnz) return;
  const uint32_t k = i / 9, q = i - 9 * k;
  if (!((active >> slot_inst[k]) & 1u)) return;  // an instance the batch no longer iterates
  sv[pos[k] + 32 * q] = val[i];
}

// finish of the domain kernel (and of the initialisation): instance sums of r.r and r.z
__device__ __forceinline__ void fd_finish(const FusedArgs& a, bool init) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t K = a.ninst;
  for (uint32_t q = w; q < K; q += nw) {
    const uint32_t cb = a.lay[2 * LAY + q], ce = a.lay[2 * LAY + q + 1];
    double rr = 0, rz = 0;
    for (uint32_t c = cb + lane; c < ce; c += 32) {
      rr += ((volatile double*)a.part)[2 * c];
      rz += ((volatile double*)a.part)[2 * c + 1];
    }
    rr = warp_sum(rr);
    rz = warp_sum(rz);
    if (lane == 0) {
      FusedInst& I = a.inst[q];
      if (init) {
        I.bnorm = fmax(sqrt(rr), 1e-30);
        I.residual = sqrt(rr) / I.bnorm;
        I.rz = rz;
        I.beta = 0.0;
      } else if (I.upd) {
        I.iters += 1;
        I.residual = sqrt(rr) / I.bnorm;
        if (I.residual <= (double)a.tol || I.iters >= a.max_iter) {
          I.done = 1;
        } else {
          I.beta = rz / I.rz;
          I.rz = rz;
        }
        I.upd = 0;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t all = 1;
    for (uint32_t q = 0; q < K; ++q) all &= a.inst[q].done ? 1u : 0u;
    a.ctl->all_done = all;
    a.ctl->counter[1] = 0;
    __threadfence();
  }
}

// Schwarz domains: one warp per domain. init: x = 0, r = b, p_init = 0.
template <class Acc, class TS>
__global__ void __launch_bounds__(32 * FD_WARPS) k_fr_schwarz(FusedArgs a, const float* __restrict__ pc,
                                                             float* __restrict__ p_init, int init) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (!init && a.ctl->all_done) return;
  const uint32_t K = a.ninst;
  const int k = cta_instance(a.lay + 2 * LAY, K);
  const uint32_t c0 = __ldg(a.lay + 2 * LAY + k);
  const uint32_t d = __ldg(a.lay + 3 * LAY + k) + (blockIdx.x - c0) * FD_WARPS + (threadIdx.x >> 5);
  const uint32_t dend = __ldg(a.lay + 3 * LAY + k + 1);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool upd = !init && a.inst[k].upd != 0;
  const float al = (float)a.inst[k].alpha;
  const bool skip = !init && a.inst[k].done != 0 && !upd;
  uint64_t* bar = (uint64_t*)(smem + 16 * w);
  TS* buf = (TS*)(smem + 128 + (size_t)w * apply_slice_bytes<TS>());
  float* rd = (float*)(buf + 6 * TILE_FLOATS);
  Acc* yd = (Acc*)(rd + 96);
  Acc rr = 0, rz = 0;
  if (d < dend && !skip) {
    const uint32_t vs = a.dom_start[d], nvd = a.dom_start[d + 1] - vs;
    const int m = 3 * (int)nvd;
    const uint64_t off = a.fac_off[d];
    const uint32_t bytes = (uint32_t)((a.fac_off[d + 1] - off) * sizeof(TS));
    const bool diag = a.dom_diag[d] != 0;
    if (lane == 0 && !diag) {
      mbar_init(bar, 1);
      fence_mbar_init();
      fence_proxy_async();
      mbar_arrive_expect_tx(bar, bytes);
      bulk_g2s(buf, (const TS*)a.fac + off, bytes, bar);
    }
    for (int i = lane; i < 96; i += 32) {
      float v = 0.f;
      if (i < m) {
        const uint32_t e = 3 * a.dom_verts[vs + i / 3] + i % 3;
        if (init) {
          v = a.b[e];
          a.x[e] = 0.f;
          a.r[e] = v;
          p_init[zpos(e)] = 0.f;
        } else if (upd) {
          a.x[e] = fmaf(al, pc[zpos(e)], a.x[e]);
          v = fmaf(-al, a.ap[e], a.r[e]);
          a.r[e] = v;
        } else {
          v = a.r[e];
        }
      }
      rd[i] = v;
    }
    __syncwarp();
    if (diag) {
      if (lane < (int)nvd) {
        const uint32_t v = a.dom_verts[vs + lane];
        Acc zz[3];
        vertex_apply<Acc>(a.vfac + 6 * (size_t)v, rd + 3 * lane, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float zi = (float)zz[c];
          a.z[4 * v + c] = zi;
          rr += (Acc)rd[3 * lane + c] * (Acc)rd[3 * lane + c];
          rz += (Acc)rd[3 * lane + c] * (Acc)zi;
        }
      }
    } else if (!mbar_wait(bar, 0)) {
      if (lane == 0) atomicOr(&a.inst[k].status, ST_WAIT_TIMEOUT);
      mbar_wait(bar, 0);  // bounded again: the copy may still land
    } else {
      Acc zz[3];
      const int T = (m + 31) >> 5;
      if (T == 3)
        tiles_apply<3, Acc, TS>(buf, rd, yd, zz, lane);
      else if (T == 2)
        tiles_apply<2, Acc, TS>(buf, rd, yd, zz, lane);
      else
        tiles_apply<1, Acc, TS>(buf, rd, yd, zz, lane);
      const Acc sc = a.fac_scale ? (Acc)a.fac_scale[d] : (Acc)1;
#pragma unroll
      for (int J = 0; J < 3; ++J) {
        const int i = 32 * J + lane;
        if (i < m) {
          const float zi = (float)(zz[J] * sc * sc);
          a.z[4 * a.dom_verts[vs + i / 3] + i % 3] = zi;
          rr += (Acc)rd[i] * (Acc)rd[i];
          rz += (Acc)rd[i] * (Acc)zi;
        }
      }
    }
  }
  const Acc s0 = block_sum<Acc>(rr);
  const Acc s1 = block_sum<Acc>(rz);
  if (threadIdx.x == 0) {
    a.part[2 * blockIdx.x] = (double)s0;
    a.part[2 * blockIdx.x + 1] = (double)s1;
  }
  if (!last_cta(&a.ctl->counter[1])) return;
  fd_finish(a, init != 0);
}

// Schwarz domains on the tensor cores (FP16 tiles): one warp per domain, DOMS domains per CTA;
// the domain's apply is tc_apply (mma.sync over 16 x 16 blocks of its tiles, the vectors split
// into three FP16 terms, FP32 accumulation). Otherwise as k_fr_schwarz.
constexpr uint32_t TC_SLICE_BYTES = 6 * TILE_FLOATS * 2 + 3 * 96 * 4;  // tiles, r, y, z

template <class Acc, int DOMS>
__global__ void __launch_bounds__(32 * DOMS) k_fr_schwarz_tc(FusedArgs a, const float* __restrict__ pc,
                                                            float* __restrict__ p_init, int init) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (!init && a.ctl->all_done) return;
  const uint32_t K = a.ninst;
  const int k = cta_instance(a.lay + 2 * LAY, K);
  const uint32_t c0 = __ldg(a.lay + 2 * LAY + k);
  const uint32_t d = __ldg(a.lay + 3 * LAY + k) + (blockIdx.x - c0) * DOMS + (threadIdx.x >> 5);
  const uint32_t dend = __ldg(a.lay + 3 * LAY + k + 1);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const bool upd = !init && a.inst[k].upd != 0;
  const float al = (float)a.inst[k].alpha;
  const bool skip = !init && a.inst[k].done != 0 && !upd;
  uint64_t* bar = (uint64_t*)(smem + 16 * w);
  __half* buf = (__half*)(smem + 128 + (size_t)w * TC_SLICE_BYTES);
  float* rd = (float*)(buf + 6 * TILE_FLOATS);
  float* ys = rd + 96;
  float* zs = ys + 96;
  Acc rr = 0, rz = 0;
  if (d < dend && !skip) {
    const uint32_t vs = a.dom_start[d], nvd = a.dom_start[d + 1] - vs;
    const int m = 3 * (int)nvd;
    const uint64_t off = a.fac_off[d];
    const uint32_t bytes = (uint32_t)((a.fac_off[d + 1] - off) * sizeof(__half));
    const bool diag = a.dom_diag[d] != 0;
    if (lane == 0 && !diag) {
      mbar_init(bar, 1);
      fence_mbar_init();
      fence_proxy_async();
      mbar_arrive_expect_tx(bar, bytes);
      bulk_g2s(buf, (const __half*)a.fac + off, bytes, bar);
    }
    for (int i = lane; i < 96; i += 32) {
      float v = 0.f;
      if (i < m) {
        const uint32_t e = 3 * a.dom_verts[vs + i / 3] + i % 3;
        if (init) {
          v = a.b[e];
          a.x[e] = 0.f;
          a.r[e] = v;
          p_init[zpos(e)] = 0.f;
        } else if (upd) {
          a.x[e] = fmaf(al, pc[zpos(e)], a.x[e]);
          v = fmaf(-al, a.ap[e], a.r[e]);
          a.r[e] = v;
        } else {
          v = a.r[e];
        }
      }
      rd[i] = v;
    }
    __syncwarp();
    if (diag) {
      if (lane < (int)nvd) {
        const uint32_t v = a.dom_verts[vs + lane];
        Acc zz[3];
        vertex_apply<Acc>(a.vfac + 6 * (size_t)v, rd + 3 * lane, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float zi = (float)zz[c];
          a.z[4 * v + c] = zi;
          rr += (Acc)rd[3 * lane + c] * (Acc)rd[3 * lane + c];
          rz += (Acc)rd[3 * lane + c] * (Acc)zi;
        }
      }
    } else if (!mbar_wait(bar, 0)) {
      if (lane == 0) atomicOr(&a.inst[k].status, ST_WAIT_TIMEOUT);
      mbar_wait(bar, 0);  // bounded again: the copy may still land
    } else {
      float zz[3];
      tc_apply(buf, rd, ys, zs, m, zz, lane);
      const float sc = a.fac_scale[d];
#pragma unroll
      for (int J = 0; J < 3; ++J) {
        const int i = 32 * J + lane;
        if (i < m) {
          const float zi = (float)((Acc)zz[J] * (Acc)sc * (Acc)sc);
          a.z[4 * a.dom_verts[vs + i / 3] + i % 3] = zi;
          rr += (Acc)rd[i] * (Acc)rd[i];
          rz += (Acc)rd[i] * (Acc)zi;
        }
      }
    }
  }
  const Acc s0 = block_sum<Acc>(rr);
  const Acc s1 = block_sum<Acc>(rz);
  if (threadIdx.x == 0) {
    a.part[2 * blockIdx.x] = (double)s0;
    a.part[2 * blockIdx.x + 1] = (double)s1;
  }
  if (!last_cta(&a.ctl->counter[1])) return;
  fd_finish(a, init != 0);
}

// Schwarz domains with three warps per domain, DOMS domains per CTA. The domain's tiles
// (storage order (0,0), (1,0), (1,1), (2,0), (2,1), (2,2)) are split between the warps, warp
// q taking tiles q and q + 3: each warp forms its tiles' partial W r rows, the partials are
// summed per tile row in a fixed order into y = W r, each warp forms its tiles' partial
// W^T y columns, and those are summed per tile column into z. Compared with one warp per
// domain, the chain of dependent tile passes per domain is a third as long and three times
// as many warps share the same shared memory. The sums are deterministic.
// Accumulation type of the tile passes: FP32 over FP16 tiles (whose own rounding, 2^-11,
// dwarfs FP32 sums of 32 terms), else the precision's type. The dot products stay in Acc.
template <class Acc, class TS>
using ApplyAcc = typename std::conditional<sizeof(TS) == 2, float, Acc>::type;

template <class Acc, class TS>
__host__ __device__ constexpr uint32_t f3_slice_bytes() {
  return (6 * TILE_FLOATS * (uint32_t)sizeof(TS) + 96 * 4 + 3 * 2 * 32 * (uint32_t)sizeof(ApplyAcc<Acc, TS>) +
          96 * (uint32_t)sizeof(ApplyAcc<Acc, TS>) + 127) / 128 * 128;
}

__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// tile t's row and column block, and the tiles of warp q (slot 0, 1; -1 none) for T tile rows
__device__ __forceinline__ int f3_tile_i(int t) { return t >= 3 ? 2 : (t >= 1 ? 1 : 0); }
__device__ __forceinline__ int f3_tile_j(int t) { return t - f3_tile_i(t) * (f3_tile_i(t) + 1) / 2; }
__device__ __forceinline__ int f3_tile(int T, int q, int slot) {
  if (T == 3) return slot == 0 ? q : q + 3;
  if (T == 2) return slot == 0 ? q : -1;
  return (q == 0 && slot == 0) ? 0 : -1;
}

template <class Acc, class TS, int DOMS>
__global__ void __launch_bounds__(96 * DOMS) k_fr_schwarz3(FusedArgs a, const float* __restrict__ pc,
                                                          float* __restrict__ p_init, int init) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (!init && a.ctl->all_done) return;
  const uint32_t K = a.ninst;
  const int k = cta_instance(a.lay + 2 * LAY, K);
  const uint32_t c0 = __ldg(a.lay + 2 * LAY + k);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ld = wid / 3, q = wid - 3 * ld;
  const uint32_t d = __ldg(a.lay + 3 * LAY + k) + (blockIdx.x - c0) * DOMS + ld;
  const uint32_t dend = __ldg(a.lay + 3 * LAY + k + 1);
  const bool upd = !init && a.inst[k].upd != 0;
  const float al = (float)a.inst[k].alpha;
  const bool skip = !init && a.inst[k].done != 0 && !upd;
  const bool valid = d < dend && !skip;
  uint64_t* bar = (uint64_t*)(smem + 16 * ld);
  unsigned char* slice = smem + 128 + (size_t)ld * f3_slice_bytes<Acc, TS>();
  using AA = ApplyAcc<Acc, TS>;
  TS* buf = (TS*)slice;
  float* rd = (float*)(buf + 6 * TILE_FLOATS);
  AA* part = (AA*)(rd + 96);  // [3][2][32]
  AA* yd = part + 3 * 2 * 32;
  const int bid = 1 + ld;
  Acc rr = 0, rz = 0;
  uint32_t vs = 0;
  int m = 0;
  const bool diag = valid && a.dom_diag[d] != 0;
  if (valid) {
    vs = a.dom_start[d];
    m = 3 * (int)(a.dom_start[d + 1] - vs);
    if (q == 0 && lane == 0 && !diag) {
      const uint64_t off = a.fac_off[d];
      const uint32_t bytes = (uint32_t)((a.fac_off[d + 1] - off) * sizeof(TS));
      mbar_init(bar, 1);
      fence_mbar_init();
      fence_proxy_async();
      mbar_arrive_expect_tx(bar, bytes);
      bulk_g2s(buf, (const TS*)a.fac + off, bytes, bar);
    }
    const int i = 32 * q + lane;
    float v = 0.f;
    if (i < m) {
      const uint32_t e = 3 * a.dom_verts[vs + i / 3] + i % 3;
      if (init) {
        v = a.b[e];
        a.x[e] = 0.f;
        a.r[e] = v;
        p_init[zpos(e)] = 0.f;
      } else if (upd) {
        a.x[e] = fmaf(al, pc[zpos(e)], a.x[e]);
        v = fmaf(-al, a.ap[e], a.r[e]);
        a.r[e] = v;
      } else {
        v = a.r[e];
      }
    }
    rd[i] = v;
  }
  named_sync(bid, 96);  // rd complete, the barrier initialised
  if (diag && q == 0 && lane < m / 3) {
    // block-diagonal domain: one lane per vertex
    const uint32_t v = a.dom_verts[vs + lane];
    Acc zz[3];
    vertex_apply<Acc>(a.vfac + 6 * (size_t)v, rd + 3 * lane, zz);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float zi = (float)zz[c];
      a.z[4 * v + c] = zi;
      rr += (Acc)rd[3 * lane + c] * (Acc)rd[3 * lane + c];
      rz += (Acc)rd[3 * lane + c] * (Acc)zi;
    }
  }
  bool ok = true;
  if (valid && !diag) {
    ok = mbar_wait(bar, 0);
    if (!ok) {
      if (q == 0 && lane == 0) atomicOr(&a.inst[k].status, ST_WAIT_TIMEOUT);
      mbar_wait(bar, 0);  // bounded again: the copy may still land
    }
  }
  const int T = (m + 31) >> 5;
  const bool tiles = valid && ok && !diag;
  // pass 1: partial rows of W r
  if (tiles) {
#pragma unroll
    for (int slot = 0; slot < 2; ++slot) {
      const int t = f3_tile(T, q, slot);
      if (t < 0) continue;
      const TS* w = buf + t * TILE_FLOATS;
      const float* rj = rd + 32 * f3_tile_j(t);
      AA y = 0;
      if constexpr (sizeof(TS) == 2) {
        // row `lane` of an FP16 tile: element (lane, c) sits at c * 32 + off[(c >> 1) & 3] (the
        // chunk permutation repeats every 8 columns), so with the column loop unrolled every
        // load is a register base plus an immediate
        const __half* wh = reinterpret_cast<const __half*>(w);
        const __half* row[4];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) row[qq] = wh + ((((lane >> 3) ^ qq) & 3) << 3) + (lane & 7);
#pragma unroll
        for (int c0 = 0; c0 < 32; c0 += 4) {  // r_j as broadcast float4 loads, the sum in column order
          const float4 r4 = *reinterpret_cast<const float4*>(rj + c0);
          y += __half2float(row[(c0 >> 1) & 3][c0 * 32]) * r4.x;
          y += __half2float(row[((c0 + 1) >> 1) & 3][(c0 + 1) * 32]) * r4.y;
          y += __half2float(row[((c0 + 2) >> 1) & 3][(c0 + 2) * 32]) * r4.z;
          y += __half2float(row[((c0 + 3) >> 1) & 3][(c0 + 3) * 32]) * r4.w;
        }
      } else {
#pragma unroll 2
        for (int c0 = 0; c0 < 32; c0 += 4) {  // r_j as broadcast float4 loads, the sum in column order
          const float4 r4 = *reinterpret_cast<const float4*>(rj + c0);
          y += (AA)tile_ld(w, tile_off<TS>(lane, c0)) * (AA)r4.x;
          y += (AA)tile_ld(w, tile_off<TS>(lane, c0 + 1)) * (AA)r4.y;
          y += (AA)tile_ld(w, tile_off<TS>(lane, c0 + 2)) * (AA)r4.z;
          y += (AA)tile_ld(w, tile_off<TS>(lane, c0 + 3)) * (AA)r4.w;
        }
      }
      part[(2 * q + slot) * 32 + lane] = y;
    }
  }
  named_sync(bid, 96);
  if (tiles && q < T) {  // y_q = sum of the partials of tile row q
    AA y = 0;
    for (int p = 0; p < 3; ++p)
      for (int slot = 0; slot < 2; ++slot) {
        const int t = f3_tile(T, p, slot);
        if (t >= 0 && f3_tile_i(t) == q) y += part[(2 * p + slot) * 32 + lane];
      }
    yd[32 * q + lane] = y;
  }
  named_sync(bid, 96);
  // pass 2: partial columns of W^T y (into the partial buffer, now free)
  if (tiles) {
#pragma unroll
    for (int slot = 0; slot < 2; ++slot) {
      const int t = f3_tile(T, q, slot);
      if (t < 0) continue;
      const TS* w = buf + t * TILE_FLOATS;
      const AA* yi = yd + 32 * f3_tile_i(t);
      AA z = 0;
      if constexpr (sizeof(TS) == 2) {
        // FP16 tiles: column `lane` as four 16-byte chunks (rows 8 kk .. 8 kk + 7 each), read
        // in row order, their y entries as broadcast float4 loads; the sum runs over r in order
        const uint4* col = reinterpret_cast<const uint4*>(w + 32 * lane);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint4 v = col[kk ^ ((lane >> 1) & 3)];
          const float4 ya = *reinterpret_cast<const float4*>(yi + 8 * kk);
          const float4 yb = *reinterpret_cast<const float4*>(yi + 8 * kk + 4);
          float2 f = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
          z += f.x * ya.x;
          z += f.y * ya.y;
          f = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
          z += f.x * ya.z;
          z += f.y * ya.w;
          f = __half22float2(*reinterpret_cast<const __half2*>(&v.z));
          z += f.x * yb.x;
          z += f.y * yb.y;
          f = __half22float2(*reinterpret_cast<const __half2*>(&v.w));
          z += f.x * yb.z;
          z += f.y * yb.w;
        }
      } else {
#pragma unroll 8
        for (int r = 0; r < 32; ++r) z += (AA)tile_ld(w, tile_off<TS>(r, lane)) * yi[r];
      }
      part[(2 * q + slot) * 32 + lane] = z;
    }
  }
  named_sync(bid, 96);
  if (tiles && q < T) {  // z_q = sum of the partials of tile column q
    AA z = 0;
    for (int p = 0; p < 3; ++p)
      for (int slot = 0; slot < 2; ++slot) {
        const int t = f3_tile(T, p, slot);
        if (t >= 0 && f3_tile_j(t) == q) z += part[(2 * p + slot) * 32 + lane];
      }
    const int i = 32 * q + lane;
    if (i < m) {
      const AA sc = a.fac_scale ? (AA)a.fac_scale[d] : (AA)1;
      const float zi = (float)(z * sc * sc);
      a.z[4 * a.dom_verts[vs + i / 3] + i % 3] = zi;
      rr = (Acc)rd[i] * (Acc)rd[i];
      rz = (Acc)rd[i] * (Acc)zi;
    }
  }
  const Acc s0 = block_sum<Acc>(rr);
  const Acc s1 = block_sum<Acc>(rz);
  if (threadIdx.x == 0) {
    a.part[2 * blockIdx.x] = (double)s0;
    a.part[2 * blockIdx.x + 1] = (double)s1;
  }
  if (!last_cta(&a.ctl->counter[1])) return;
  fd_finish(a, init != 0);
}

// Block Jacobi: one thread per vertex. init: x = 0, r = b, p_init = 0.
template <class Acc>
__global__ void __launch_bounds__(FD_THREADS) k_fr_bj(FusedArgs a, const float* __restrict__ pc,
                                                     float* __restrict__ p_init, int init) {
  if (!init && a.ctl->all_done) return;
  const uint32_t K = a.ninst;
  const int k = cta_instance(a.lay + 2 * LAY, K);
  const uint32_t c0 = __ldg(a.lay + 2 * LAY + k);
  const uint32_t v = __ldg(a.lay + k) + (blockIdx.x - c0) * FD_THREADS + threadIdx.x;
  const uint32_t vend = __ldg(a.lay + k + 1);
  const bool upd = !init && a.inst[k].upd != 0;
  const float al = (float)a.inst[k].alpha;
  const bool skip = !init && a.inst[k].done != 0 && !upd;
  Acc rr = 0, rz = 0;
  if (v < vend && !skip) {
    float q[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const uint32_t e = 3 * v + c;
      if (init) {
        q[c] = a.b[e];
        a.x[e] = 0.f;
        a.r[e] = q[c];
        p_init[zpos(e)] = 0.f;
      } else if (upd) {
        a.x[e] = fmaf(al, pc[zpos(e)], a.x[e]);
        q[c] = fmaf(-al, a.ap[e], a.r[e]);
        a.r[e] = q[c];
      } else {
        q[c] = a.r[e];
      }
    }
    const float* m9 = a.bjinv + 9 * (size_t)v;
    const float z0 = m9[0] * q[0] + m9[1] * q[1] + m9[2] * q[2];
    const float z1 = m9[3] * q[0] + m9[4] * q[1] + m9[5] * q[2];
    const float z2 = m9[6] * q[0] + m9[7] * q[1] + m9[8] * q[2];
    a.z[4 * v] = z0;
    a.z[4 * v + 1] = z1;
    a.z[4 * v + 2] = z2;
    rr = (Acc)q[0] * (Acc)q[0] + (Acc)q[1] * (Acc)q[1] + (Acc)q[2] * (Acc)q[2];
    rz = (Acc)q[0] * (Acc)z0 + (Acc)q[1] * (Acc)z1 + (Acc)q[2] * (Acc)z2;
  }
  const Acc s0 = block_sum<Acc>(rr);
  const Acc s1 = block_sum<Acc>(rz);
  if (threadIdx.x == 0) {
    a.part[2 * blockIdx.x] = (double)s0;
    a.part[2 * blockIdx.x + 1] = (double)s1;
  }
  if (!last_cta(&a.ctl->counter[1])) return;
  fd_finish(a, init != 0);
}

namespace {
// The fused kernels' variants the autotuner chooses between (per scene, cached per system
// size): rows kernel with 2, 1 or 4 lanes per block row over the BSR, or one lane per row over
// the sliced-ELL copy; Schwarz domain kernel with one warp per domain (4 domains per CTA),
// three warps per domain (1, 2 or 4 domains per CTA), or, for FP16 tiles, one warp per domain
// on the tensor cores (4 or 8 domains per CTA; with FP32 tiles these two fall back to the
// first).
constexpr int N_ROWS_VARIANTS = 4;
constexpr int N_DOM_VARIANTS = 6;
constexpr int DOM_TC4 = 4, DOM_TC8 = 5;
constexpr int ROWS_LPR[N_ROWS_VARIANTS] = {2, 1, 4, 1};
constexpr int ROWS_SELL = 3;

struct Launch {
  void* rows;
  void* dom;
  size_t dom_smem;
  uint32_t grid_rows, grid_dom;
  uint32_t lpr, dom_threads, doms_per_cta;
};

template <class Acc>
void* rows_fn(int rv) {
  switch (rv) {
    case 1: return (void*)k_fr_rows<Acc, 1>;
    case 2: return (void*)k_fr_rows<Acc, 4>;
    case 3: return (void*)k_fr_rows_sell<Acc>;
    default: return (void*)k_fr_rows<Acc, 2>;
  }
}

template <class Acc, class TS>
void dom_fn(int dv, Launch& L) {
  if (sizeof(TS) == 2 && (dv == DOM_TC4 || dv == DOM_TC8)) {
    const int n = dv == DOM_TC4 ? 4 : 8;
    L.dom = n == 4 ? (void*)k_fr_schwarz_tc<Acc, 4> : (void*)k_fr_schwarz_tc<Acc, 8>;
    L.doms_per_cta = n;
    L.dom_threads = 32 * n;
    L.dom_smem = 128 + (size_t)n * TC_SLICE_BYTES;
    return;
  }
  switch (dv) {
    case 1:
      L.dom = (void*)k_fr_schwarz3<Acc, TS, 1>;
      L.doms_per_cta = 1;
      L.dom_threads = 96;
      L.dom_smem = 128 + f3_slice_bytes<Acc, TS>();
      break;
    case 2:
      L.dom = (void*)k_fr_schwarz3<Acc, TS, 2>;
      L.doms_per_cta = 2;
      L.dom_threads = 192;
      L.dom_smem = 128 + 2 * (size_t)f3_slice_bytes<Acc, TS>();
      break;
    case 3:
      L.dom = (void*)k_fr_schwarz3<Acc, TS, 4>;
      L.doms_per_cta = 4;
      L.dom_threads = 384;
      L.dom_smem = 128 + 4 * (size_t)f3_slice_bytes<Acc, TS>();
      break;
    default:
      L.dom = (void*)k_fr_schwarz<Acc, TS>;
      L.doms_per_cta = FD_WARPS;
      L.dom_threads = 32 * FD_WARPS;
      L.dom_smem = 128 + (size_t)FD_WARPS * apply_slice_bytes<TS>();
  }
}

Launch fused_kernels(const Scene& s, int rv, int dv) {
  Launch L{};
  const bool sch = s.schwarz != nullptr;
  L.rows = s.mixed ? rows_fn<double>(rv) : rows_fn<float>(rv);
  L.lpr = ROWS_LPR[rv];
  if (sch && s.schwarz->half) {
    if (s.mixed) dom_fn<double, __half>(dv, L); else dom_fn<float, __half>(dv, L);
  } else if (sch) {
    if (s.mixed) dom_fn<double, float>(dv, L); else dom_fn<float, float>(dv, L);
  } else {
    L.dom = s.mixed ? (void*)k_fr_bj<double> : (void*)k_fr_bj<float>;
    L.dom_smem = 0;
    L.dom_threads = FD_THREADS;
    L.doms_per_cta = FD_THREADS;  // vertices per CTA
  }
  return L;
}
}  // namespace

// The sliced-ELL copy of Ps (built once per scene: the pattern is fixed): slices of 32
// consecutive rows of one instance, each as wide as its longest row.
static int sell_build(Scene& s) {
  const auto& rp = s.Ps.h_row_ptr;
  const auto& cl = s.Ps.h_col;
  const uint32_t K = s.ninst;
  std::vector<uint32_t> base(1, 0), inst(K + 1, 0), col, pos(std::max<uint32_t>(s.Ps.nnz, 1), 0);
  for (uint32_t k = 0; k < K; ++k) {
    inst[k] = (uint32_t)base.size() - 1;
    for (uint32_t r0 = s.inst_vert[k]; r0 < s.inst_vert[k + 1]; r0 += 32) {
      const uint32_t r1 = std::min<uint32_t>(r0 + 32, s.inst_vert[k + 1]);
      uint32_t w = 0;
      for (uint32_t r = r0; r < r1; ++r) w = std::max<uint32_t>(w, rp[r + 1] - rp[r]);
      const uint32_t b = base.back();
      col.resize(32 * (size_t)(b + w));
      for (uint32_t j = 0; j < w; ++j)
        for (uint32_t l = 0; l < 32; ++l) {
          const uint32_t r = r0 + l;
          const bool has = r < r1 && rp[r] + j < rp[r + 1];
          col[32 * (size_t)(b + j) + l] = has ? cl[rp[r] + j] : (r < r1 ? r : r0);
          if (has) pos[rp[r] + j] = 288 * (b + j) + l;
        }
      base.push_back(b + w);
    }
  }
  inst[K] = (uint32_t)base.size() - 1;
  cudaStream_t st = s.st;
  MG_TRY(s.sell_base.upload(base.data(), base.size(), st));
  MG_TRY(s.sell_inst.upload(inst.data(), inst.size(), st));
  MG_TRY(s.sell_col.upload(col.data(), std::max<size_t>(col.size(), 1), st));
  MG_TRY(s.sell_pos.upload(pos.data(), pos.size(), st));
  MG_TRY(s.sell_val.reserve(std::max<size_t>(288 * (size_t)base.back(), 1)));
  MG_CUDA(cudaMemsetAsync(s.sell_val.p, 0, 4 * std::max<size_t>(288 * (size_t)base.back(), 1), st));
  MG_CUDA(cudaStreamSynchronize(st));
  s.sell_built = true;
  return MGUSO_OK;
}

__global__ void k_fr_reset(FusedInst* __restrict__ inst, FusedCtl* __restrict__ ctl, uint32_t K, uint32_t active) {
  const uint32_t k = threadIdx.x;
  if (k < K) {
    inst[k] = FusedInst{};
    inst[k].done = ((active >> k) & 1u) ? 0u : 1u;
  }
  if (k == 0) *ctl = FusedCtl{};
}

// Layout of the fused kernels over the scene's instances and the arguments of both; resets
// the per-instance state (instances outside `active` start done) on the scene's stream.
static int fused_prepare(Scene& s, const uint32_t* h_inst_row, uint32_t K, uint32_t active, FusedArgs& a, Launch& L) {
  MG_CHECK_ARG(K >= 1 && K <= PCG_MAX_INST, "fused PCG: 1..8 instances");
  cudaStream_t st = s.st;
  PcgWork& w = s.work;
  L = fused_kernels(s, s.fr_rows_variant, s.fr_dom_variant);
  // layout: rows, row-kernel CTAs, domain-kernel CTAs, domains (per instance)
  std::vector<uint32_t> key(h_inst_row, h_inst_row + K + 1);
  key.push_back((uint32_t)s.fr_rows_variant);
  key.push_back((uint32_t)s.fr_dom_variant);
  if (key != s.fr_key) {
    std::vector<uint32_t> lay(4 * LAY, 0);
    for (uint32_t k = 0; k <= K; ++k) lay[k] = h_inst_row[k];
    uint32_t* dom = lay.data() + 3 * LAY;
    if (s.schwarz) {
      mguso_schwarz* sw = s.schwarz.get();
      uint32_t kk = 0;
      for (uint32_t d = 0; d < sw->ndom; ++d) {
        const uint32_t v0 = sw->h_dom_verts[sw->h_dom_start[d]];
        while (kk < K && v0 >= h_inst_row[kk + 1]) dom[++kk] = d;
        MG_CHECK_ARG(kk < K, "fused PCG: Schwarz domains are not grouped by instance");
      }
      while (kk < K) dom[++kk] = sw->ndom;
    }
    for (uint32_t k = 0; k < K; ++k) {
      const uint32_t rows = h_inst_row[k + 1] - h_inst_row[k];
      const uint32_t cr = std::max<uint32_t>(1, ceil_div(rows * L.lpr, FR_THREADS));
      const uint32_t cd = s.schwarz ? std::max<uint32_t>(1, ceil_div(dom[k + 1] - dom[k], L.doms_per_cta))
                                    : std::max<uint32_t>(1, ceil_div(rows, FD_THREADS));
      lay[LAY + k + 1] = lay[LAY + k] + cr;
      lay[2 * LAY + k + 1] = lay[2 * LAY + k] + cd;
    }
    MG_TRY(s.fr_lay.upload(lay.data(), lay.size(), st));
    s.fr_grid_rows = lay[LAY + K];
    s.fr_grid_dom = lay[2 * LAY + K];
    s.fr_key = key;
    s.fr_graph_key.clear();
  }
  L.grid_rows = s.fr_grid_rows;
  L.grid_dom = s.fr_grid_dom;
  MG_TRY(w.p2.reserve(4 * ((size_t)w.n / 3 + 1)));  // the second direction, 4 floats per vertex
  MG_TRY(s.fr_inst.reserve(PCG_MAX_INST));
  MG_TRY(s.fr_ctl.reserve(1));
  MG_TRY(s.fr_part.reserve(2ull * std::max(L.grid_rows, L.grid_dom)));
  // per-instance state and loop control reset on the device (no host copy to wait for)
  k_fr_reset<<<1, 32, 0, st>>>(s.fr_inst.p, s.fr_ctl.p, K, active);
  MG_CUDA(cudaGetLastError());

  a = FusedArgs{};
  a.ninst = K;
  a.lay = s.fr_lay.p;
  a.rp = s.Ps.row_ptr.p;
  a.col = s.Ps.col.p;
  a.val = s.A->val.p;
  a.crp = s.c_row_ptr.p;
  a.ccol = s.c_col.p ? s.c_col.p : s.c_row_ptr.p;
  a.cval = s.c_val.p;
  a.bjinv = s.bjinv.p;
  if (s.schwarz) {
    mguso_schwarz* sw = s.schwarz.get();
    a.dom_start = sw->dom_start.p;
    a.dom_verts = sw->dom_verts.p;
    a.fac_off = sw->fac_off.p;
    a.fac = sw->half ? (const void*)sw->fac_h.p : (const void*)sw->fac.p;
    a.fac_scale = sw->half ? sw->fac_scale.p : nullptr;
    a.dom_diag = sw->dom_diag.p;
    a.vfac = sw->vfac.p;
  }
  if (s.fr_rows_variant == ROWS_SELL) {
    if (!s.sell_built) MG_TRY(sell_build(s));
    // the system's current values into the sliced-ELL copy
    k_sell_pack<<<ceil_div(9 * (size_t)s.Ps.nnz, 256), 256, 0, st>>>(s.A->val.p, s.sell_pos.p, s.Ps.nnz, s.sell_val.p,
                                                                    s.slot_inst.p, s.iter_active);
    MG_CUDA(cudaGetLastError());
    a.sell_base = s.sell_base.p;
    a.sell_inst = s.sell_inst.p;
    a.sell_col = s.sell_col.p;
    a.sell_val = s.sell_val.p;
  }
  a.b = w.b.p;
  a.x = w.x.p;
  a.r = w.r.p;
  a.z = w.z.p;
  a.ap = w.ap.p;
  a.tol = s.p.cg_tol;
  a.max_iter = s.p.cg_max_iter;
  a.inst = s.fr_inst.p;
  a.ctl = s.fr_ctl.p;
  a.part = s.fr_part.p;
  if (L.dom_smem) MG_CUDA(cudaFuncSetAttribute(L.dom, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.dom_smem));
  return MGUSO_OK;
}

// The device-driven loop's condition: after each body of FUSED_CHECK iterations, go on while
// an instance is still iterating and fewer than max_rounds bodies have run (the bound the
// host-driven loop had: cg_max_iter + FUSED_CHECK iterations launched).
__global__ void k_fr_continue(FusedCtl* __restrict__ ctl, cudaGraphConditionalHandle h, uint32_t max_rounds) {
  const uint32_t r = ctl->rounds + 1;
  ctl->rounds = r;
  cudaGraphSetConditional(h, (!ctl->all_done && r < max_rounds) ? 1u : 0u);
}

static int launch_dom(const Scene& s, const Launch& L, FusedArgs& a, const float* pc, float* pinit, int init) {
  void* args[] = {(void*)&a, (void*)&pc, (void*)&pinit, (void*)&init};
  MG_CUDA(cudaLaunchKernel(L.dom, dim3(L.grid_dom), dim3(L.dom_threads), args, L.dom_smem, s.st));
  return MGUSO_OK;
}

static int launch_rows(const Scene& s, const Launch& L, FusedArgs& a, const float* po, float* pn) {
  void* args[] = {(void*)&a, (void*)&po, (void*)&pn};
  MG_CUDA(cudaLaunchKernel(L.rows, dim3(L.grid_rows), dim3(FR_THREADS), args, 0, s.st));
  return MGUSO_OK;
}

// Solves the scene's current system (work.b) into work.x; instance k covers block rows
// [h_inst_row[k], h_inst_row[k+1]); instances outside `active` keep x = 0. out[k] gets each
// instance's result. Schwarz domains must be grouped by instance.
int pcg_fused(Scene& s, const uint32_t* h_inst_row, uint32_t K, uint32_t active, PcgInstResult* out) {
  cudaStream_t st = s.st;
  FusedArgs a;
  Launch L;
  MG_TRY(fused_prepare(s, h_inst_row, K, active, a, L));
  float* p0 = s.work.p.p;
  float* p1 = s.work.p2.p;
  // x = 0, r = b, p0 = 0, z = M^-1 r, norms
  MG_TRY(launch_dom(s, L, a, p0, p0, 1));
  // one graph of FUSED_CHECK iterations (p alternates between the two buffers)
  std::vector<unsigned char> gk(sizeof(FusedArgs) + 2 * sizeof(void*) + 2 * sizeof(uint32_t));
  std::memcpy(gk.data(), &a, sizeof(FusedArgs));
  std::memcpy(gk.data() + sizeof(FusedArgs), &p0, sizeof(void*));
  std::memcpy(gk.data() + sizeof(FusedArgs) + sizeof(void*), &p1, sizeof(void*));
  std::memcpy(gk.data() + sizeof(FusedArgs) + 2 * sizeof(void*), &L.grid_rows, 4);
  std::memcpy(gk.data() + sizeof(FusedArgs) + 2 * sizeof(void*) + 4, &L.grid_dom, 4);
  // The whole solve is one graph launch: a conditional while node whose body runs FUSED_CHECK
  // iterations and then k_fr_continue, which decides on the device whether to go on, so the
  // host neither waits nor reads anything until the solve has finished.
  const uint32_t max_rounds = ceil_div(s.p.cg_max_iter + FUSED_CHECK, FUSED_CHECK);
  if (plain_launches()) {
    // every kernel launched on its own and the loop driven by the host (profilers cannot see
    // the kernels inside conditional graphs): the same iterations and the same bound
    FusedCtl h{};
    for (uint32_t r = 0; r < max_rounds; ++r) {
      for (uint32_t i = 0; i < FUSED_CHECK; ++i) {
        const float* po = (i & 1) ? p1 : p0;
        float* pn = (i & 1) ? p0 : p1;
        MG_TRY(launch_rows(s, L, a, po, pn));
        MG_TRY(launch_dom(s, L, a, pn, pn, 0));
      }
      MG_CUDA(cudaMemcpyAsync(&h, s.fr_ctl.p, sizeof(FusedCtl), cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaStreamSynchronize(st));
      if (h.all_done) break;
    }
    MG_TRY(s.fr_out.reserve(PCG_MAX_INST));
    MG_CUDA(cudaMemcpyAsync(s.fr_out.p, s.fr_inst.p, sizeof(FusedInst) * K, cudaMemcpyDeviceToHost, st));
    if (!out) return MGUSO_OK;
    return pcg_fused_results(s, K, out);
  }
  if (gk != s.fr_graph_key || !s.fr_exec) {
    if (s.fr_exec) cudaGraphExecDestroy(s.fr_exec);
    s.fr_exec = nullptr;
    cudaGraph_t g = nullptr;
    MG_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = cond;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    }
    if (e == cudaSuccess)
      e = cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      MG_CUDA(e);
    }
    int rc = MGUSO_OK;
    for (uint32_t i = 0; i < FUSED_CHECK && rc == MGUSO_OK; ++i) {
      const float* po = (i & 1) ? p1 : p0;
      float* pn = (i & 1) ? p0 : p1;
      rc = launch_rows(s, L, a, po, pn);
      if (rc == MGUSO_OK) rc = launch_dom(s, L, a, pn, pn, 0);
    }
    if (rc == MGUSO_OK) {
      k_fr_continue<<<1, 1, 0, st>>>(s.fr_ctl.p, cond, max_rounds);
      if (cudaGetLastError() != cudaSuccess) rc = MGUSO_ERR_CUDA;
    }
    cudaGraph_t body = nullptr;
    e = cudaStreamEndCapture(st, &body);
    if (rc != MGUSO_OK || e != cudaSuccess) {
      cudaGraphDestroy(g);
      if (rc != MGUSO_OK) return rc;
      MG_CUDA(e);
    }
    cudaError_t ie = cudaGraphInstantiate(&s.fr_exec, g, 0);
    cudaGraphDestroy(g);
    MG_CUDA(ie);
    s.fr_graph_key = gk;
  }
  MG_CUDA(cudaGraphLaunch(s.fr_exec, st));
  MG_TRY(s.fr_out.reserve(PCG_MAX_INST));
  MG_CUDA(cudaMemcpyAsync(s.fr_out.p, s.fr_inst.p, sizeof(FusedInst) * K, cudaMemcpyDeviceToHost, st));
  if (!out) return MGUSO_OK;  // deferred: the caller syncs the stream, then pcg_fused_results
  return pcg_fused_results(s, K, out);
}

// The per-instance results of the last pcg_fused, once the stream has passed its copy.
int pcg_fused_results(Scene& s, uint32_t K, PcgInstResult* out) {
  MG_CUDA(cudaStreamSynchronize(s.st));
  const FusedInst* hi = s.fr_out.p;
  for (uint32_t k = 0; k < K; ++k) {
    out[k].iters = hi[k].iters;
    out[k].residual = hi[k].residual;
    out[k].status = hi[k].status;
    out[k].done = hi[k].done;
    if (hi[k].status & ST_WAIT_TIMEOUT) {
      set_error("fused PCG: a bounded bulk-copy wait timed out");
      return MGUSO_ERR_TIMEOUT;
    }
  }
  return MGUSO_OK;
}

// Device time of the two fused kernels inside a PCG solve of the scene's current system:
// `iters` iterations of every instance (tolerance 0, so none stops early unless it breaks
// down), each kernel launch bracketed by its own CUDA events on the scene's stream, in the
// order and with the cache state of the solve. us2 = mean microseconds per launch of
// {rows kernel, domain kernel}; the solution left in work.x is not the system's.
int pcg_fused_profile(Scene& s, uint32_t iters, float* us2) {
  MG_CHECK_ARG(iters >= 1 && iters <= 4096, "profile: 1..4096 iterations");
  const uint32_t K = s.ninst;
  const uint32_t all = (K >= 32) ? ~0u : ((1u << K) - 1u);
  const float tol = s.p.cg_tol;
  const uint32_t mx = s.p.cg_max_iter;
  s.p.cg_tol = 0.f;
  s.p.cg_max_iter = iters + 1;
  FusedArgs a;
  Launch L;
  int rc = fused_prepare(s, s.inst_vert.data(), K, all, a, L);
  s.p.cg_tol = tol;
  s.p.cg_max_iter = mx;
  MG_TRY(rc);
  std::vector<cudaEvent_t> ev(4 * iters, nullptr);
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) rc = MGUSO_ERR_CUDA;
  float* p0 = s.work.p.p;
  float* p1 = s.work.p2.p;
  if (rc == MGUSO_OK) rc = launch_dom(s, L, a, p0, p0, 1);
  for (uint32_t i = 0; i < iters && rc == MGUSO_OK; ++i) {
    const float* po = (i & 1) ? p1 : p0;
    float* pn = (i & 1) ? p0 : p1;
    if (cudaEventRecord(ev[4 * i], s.st) != cudaSuccess) rc = MGUSO_ERR_CUDA;
    if (rc == MGUSO_OK) rc = launch_rows(s, L, a, po, pn);
    if (rc == MGUSO_OK && cudaEventRecord(ev[4 * i + 1], s.st) != cudaSuccess) rc = MGUSO_ERR_CUDA;
    if (rc == MGUSO_OK && cudaEventRecord(ev[4 * i + 2], s.st) != cudaSuccess) rc = MGUSO_ERR_CUDA;
    if (rc == MGUSO_OK) rc = launch_dom(s, L, a, pn, pn, 0);
    if (rc == MGUSO_OK && cudaEventRecord(ev[4 * i + 3], s.st) != cudaSuccess) rc = MGUSO_ERR_CUDA;
  }
  if (rc == MGUSO_OK && cudaStreamSynchronize(s.st) != cudaSuccess) rc = MGUSO_ERR_CUDA;
  double t_rows = 0, t_dom = 0;
  for (uint32_t i = 0; i < iters && rc == MGUSO_OK; ++i) {
    float m0 = 0, m1 = 0;
    if (cudaEventElapsedTime(&m0, ev[4 * i], ev[4 * i + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&m1, ev[4 * i + 2], ev[4 * i + 3]) != cudaSuccess)
      rc = MGUSO_ERR_CUDA;
    t_rows += m0;
    t_dom += m1;
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (rc == MGUSO_ERR_CUDA) set_error("fused PCG profile: a CUDA event call failed");
  MG_TRY(rc);
  us2[0] = (float)(1000.0 * t_rows / iters);
  us2[1] = (float)(1000.0 * t_dom / iters);
  return MGUSO_OK;
}

// Autotuner of the fused kernels: every rows-kernel variant (with the current domain
// kernel), then every domain-kernel variant (with the fastest rows kernel), each timed over
// 12 iterations inside a solve of the scene's current system by pcg_fused_profile; the
// fastest of each is kept. Choices are cached per system shape (vertices, pattern blocks,
// instances, precision, factor storage, domains), so scenes of the same size share one
// tuning. The solve that follows starts from scratch, so tuning leaves no trace in results
// beyond the choice of kernels.
static int fused_autotune(Scene& s) {
  static std::mutex mu;
  static std::map<std::vector<uint64_t>, std::pair<int, int>> cache;
  std::vector<uint64_t> key = {s.nv, s.Ps.nnz, s.ninst, s.mixed ? 1u : 0u,
                               s.schwarz ? (s.schwarz->half ? 2u : 1u) : 0u, s.schwarz ? s.schwarz->ndom : 0u,
                               (uint64_t)s.ctx->device};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      s.fr_rows_variant = it->second.first;
      s.fr_dom_variant = it->second.second;
      return MGUSO_OK;
    }
  }
  float us2[2];
  float best = 0;
  int br = 0;
  s.fr_dom_variant = 0;
  for (int rv = 0; rv < N_ROWS_VARIANTS; ++rv) {
    s.fr_rows_variant = rv;
    MG_TRY(pcg_fused_profile(s, 2, us2));  // warm-up (graph-free launches, attributes set)
    MG_TRY(pcg_fused_profile(s, 12, us2));
    if (rv == 0 || us2[0] < best) {
      best = us2[0];
      br = rv;
    }
  }
  s.fr_rows_variant = br;
  int bd = 0;
  if (s.schwarz) {
    for (int dv = 0; dv < (s.schwarz->half ? N_DOM_VARIANTS : DOM_TC4); ++dv) {
      s.fr_dom_variant = dv;
      MG_TRY(pcg_fused_profile(s, 2, us2));
      MG_TRY(pcg_fused_profile(s, 12, us2));
      if (dv == 0 || us2[1] < best) {
        best = us2[1];
        bd = dv;
      }
    }
  }
  s.fr_dom_variant = bd;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = {br, bd};
  return MGUSO_OK;
}

int pcg_fused_select(Scene& s) {
  if (s.fr_tuned) return MGUSO_OK;
  if (s.p.pcg_variant > 0) {
    const int v = s.p.pcg_variant - 1;
    s.fr_rows_variant = (v / N_DOM_VARIANTS) % N_ROWS_VARIANTS;
    s.fr_dom_variant = s.schwarz ? v % N_DOM_VARIANTS : 0;
  } else {
    MG_TRY(fused_autotune(s));
  }
  s.fr_tuned = true;
  return MGUSO_OK;
}

}  // namespace mg
