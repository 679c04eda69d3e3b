// Persistent PCG for the Newton systems of the implicit step: one cooperative launch runs
// every iteration of a solve (linsolve.rs:350-411: x0 = 0, r = b, z = M^-1 r, p = z; Ap,
// alpha = rz / pAp with a break on pAp <= 0 or NaN, x += alpha p, r -= alpha Ap, stop at
// ||r|| / ||b|| <= tol or max_iter, z = M^-1 r, beta = rz' / rz, p = z + beta p).
//
// The drape's systems (tens of thousands of block rows) sit in L2, so a PCG iteration of
// separate kernels is bound by launch and tail latency. Here one CTA per SM stays resident
// and the phases are separated by a grid barrier (bounded spin: a barrier that times out sets
// an error bit and the kernel returns). The launch is cooperative, so all CTAs are resident.
//
// The system may hold several independent instances (disjoint block-row ranges
// inst_row[k] .. inst_row[k+1]), each with its own scalars, convergence test and done flag;
// a finished instance stops updating while the others go on. Dot products are deterministic:
// per-thread sums in a fixed order, a fixed-tree CTA sum per instance, and every CTA sums
// the per-CTA partials in the same order after the barrier, so all CTAs hold identical
// scalars and take identical branches.
//
// Data written by other CTAs during the solve (p, z, r, partials) is read with ld.global.cg
// (L2), never through L1 or the read-only path.
#include <algorithm>
#include <vector>
#include <cstdio>
#include <cstdlib>

#include "reduce.cuh"
#include "scene.cuh"
#include "tiles.cuh"

namespace mg {

__device__ __forceinline__ float pp_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double pp_fma(double a, double b, double c) { return fma(a, b, c); }

constexpr int PP_THREADS = 256;
constexpr int PP_WARPS = PP_THREADS / 32;

struct PersistentArgs {
  uint32_t nv, ninst;
  const uint32_t* inst_row;   // ninst + 1 block-row offsets
  const uint32_t* cta_start;  // ninst + 1 CTA offsets (CTAs of instance k)
  const uint32_t* dom_range;  // ninst + 1 Schwarz-domain offsets (domains of instance k)
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
  uint32_t ndom;
  const float* b;
  float *x, *r, *z, *p, *p2, *ap;
  float tol;
  uint32_t max_iter;
  uint32_t active;  // bit k: instance k is solved; the others keep x = 0
  PcgInstResult* out;
  void* partials;     // gridDim.x * PCG_MAX_INST accumulators
  uint32_t* bar;      // [0] arrivals, [1] generation, [2] error bits
  unsigned long long* probe;  // optional: globaltimer stamps of iteration 8's phases (CTA 0)
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded grid barrier on one monotonically growing arrival counter: a CTA arrives with an
// atomic add and waits until the counter reaches the next multiple of the grid size (no
// reset, no release flag). False when the wait gave up (error bit set).
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t& target) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    target += gridDim.x;
    __threadfence();
    atomicAdd(bar, 1u);
    volatile uint32_t* c = bar;
    int ok = 1;
    uint32_t spins = 0;
    while ((int)(*c - target) < 0) {
      if (++spins > (1u << 26)) {
        atomicOr(bar + 2, ST_WAIT_TIMEOUT);
        ok = 0;
        break;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Every CTA works on one instance: CTAs [cta[k], cta[k+1]) own instance k's block rows
// [row[k], row[k+1]) and, for Schwarz, its domains [dom[k], dom[k+1]). A thread therefore
// accumulates one value per dot product, and the partials of instance k are the entries of
// its CTA range.
//
// Block-sums the NV accumulators, publishes them, crosses the grid barrier and leaves every
// instance's totals in tot[NV][PCG_MAX_INST] (each CTA computes all of them, in the same
// order, so all CTAs agree). Two alternating partial buffers: a CTA overwrites a buffer only
// after the next barrier, which every CTA reaches only once it has read the previous
// contents. False when the barrier gave up.
constexpr int PP_MAX_NV = 2;

template <class Acc, int NV>
__device__ bool grid_dots(const Acc (&v)[NV], int ninst, const uint32_t* cta, Acc* base, int& parity, uint32_t* bar,
                          uint32_t& target, Acc (*tot)[PCG_MAX_INST]) {
  Acc* part = base + (size_t)parity * gridDim.x * PP_MAX_NV;  // same stride for every NV
  parity ^= 1;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    Acc s = block_sum<Acc>(v[j]);
    if (threadIdx.x == 0) __stcg(part + (size_t)blockIdx.x * NV + j, s);
  }
  if (!grid_barrier(bar, target)) return false;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // warp w sums (instance, value) pairs w, w + 8, ...
  for (int q = w; q < ninst * NV; q += PP_WARPS) {
    const int k = q / NV, j = q - k * NV;
    Acc s = 0;
    for (uint32_t c = cta[k] + lane; c < cta[k + 1]; c += 32) s += __ldcg(part + (size_t)c * NV + j);
    s = warp_sum(s);
    if (lane == 0) tot[j][k] = s;
  }
  __syncthreads();
  return true;
}

constexpr int PP_LPR = 2;  // lanes per block row in the SpMV phase

// Each iteration has two grid-wide synchronisations:
//   phase 1 (rows):    p = z + beta p_old for the CTA's rows into the other p buffer, and
//                      Ap with every gathered p_j formed the same way on the fly; p.Ap;
//   phase 2 (domains): each warp owns whole preconditioner domains (block Jacobi: single
//                      vertices), so it updates x += alpha p, r -= alpha Ap on its domain's
//                      rows and applies the preconditioner to them with no barrier in
//                      between; r.r and r.z together.
// This is the reference's iteration with its arithmetic unchanged; only the scheduling and
// the order of the partial sums of the dot products differ.
template <int PRE, class Acc, class TS>
__global__ void __launch_bounds__(PP_THREADS, 1) k_pcg_persistent(PersistentArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint32_t s_row[PCG_MAX_INST + 1], s_cta[PCG_MAX_INST + 1], s_dom[PCG_MAX_INST + 1];
  __shared__ Acc s_tot[2][PCG_MAX_INST];
  __shared__ double s_rz[PCG_MAX_INST], s_alpha[PCG_MAX_INST], s_beta[PCG_MAX_INST], s_bnorm[PCG_MAX_INST],
      s_res[PCG_MAX_INST];
  __shared__ uint32_t s_iters[PCG_MAX_INST], s_done[PCG_MAX_INST], s_status[PCG_MAX_INST], s_upd[PCG_MAX_INST];
  __shared__ int s_abort;  // a bounded bulk-copy wait gave up: leave at the next barrier
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int K = (int)a.ninst;
  Acc* partials = (Acc*)a.partials;
  if (tid <= K) {
    s_row[tid] = a.inst_row[tid];
    s_cta[tid] = a.cta_start[tid];
    s_dom[tid] = a.dom_range[tid];
  }
  if (tid == 0) s_abort = 0;
  int parity = 0;
  uint32_t target = 0;
  if (tid < K) {
    s_iters[tid] = 0;
    s_done[tid] = ((a.active >> tid) & 1u) ? 0u : 1u;
    s_status[tid] = 0;
    s_beta[tid] = 0.0;
    s_alpha[tid] = 0.0;
    s_upd[tid] = 0;
  }
  __syncthreads();
  int k = 0;  // this CTA's instance
  while (k + 1 < K && blockIdx.x >= s_cta[k + 1]) ++k;
  const uint32_t lc = blockIdx.x - s_cta[k], nc = s_cta[k + 1] - s_cta[k];
  const uint32_t row0 = s_row[k], row1 = s_row[k + 1];
  const uint32_t lthreads = nc * PP_THREADS, ltid = lc * PP_THREADS + tid;

  uint64_t* mbar = (uint64_t*)(smem + 16 * w);
  TS* buf = (TS*)(smem + 128 + (size_t)w * apply_slice_bytes<TS>());
  uint32_t mphase = 0;
  if (PRE == MGUSO_PRECOND_SCHWARZ && lane == 0) {
    mbar_init(mbar, 1);
    fence_mbar_init();
  }
  __syncwarp();

  int cur = 0;  // which p buffer holds the current search direction
  Acc acc[2];

  // Phase 2 body. init: x = 0, r = b, p = 0 and no update. acc: [0] r.r, [1] r.z.
  auto domain_phase = [&](bool init, const float* __restrict__ pc) {
    const bool upd = s_upd[k] != 0;
    const float al = (float)s_alpha[k];
    acc[0] = 0;
    acc[1] = 0;
    if (PRE == MGUSO_PRECOND_SCHWARZ) {
      float* rd = (float*)(buf + 6 * TILE_FLOATS);
      Acc* yd = (Acc*)(rd + 96);
      for (uint32_t d = s_dom[k] + lc * PP_WARPS + w; d < s_dom[k + 1]; d += nc * PP_WARPS) {
        const uint32_t vs = a.dom_start[d], nvd = a.dom_start[d + 1] - vs;
        const int m = 3 * (int)nvd;
        const uint64_t off = a.fac_off[d];
        const uint32_t bytes = (uint32_t)((a.fac_off[d + 1] - off) * sizeof(TS));
        const bool diag = a.dom_diag[d] != 0;
        if (lane == 0 && !diag) {
          fence_proxy_async();
          mbar_arrive_expect_tx(mbar, bytes);
          bulk_g2s(buf, (const TS*)a.fac + off, bytes, mbar);
        }
        for (int i = lane; i < 96; i += 32) {
          float v = 0.f;
          if (i < m) {
            const uint32_t e = 3 * a.dom_verts[vs + i / 3] + i % 3;
            if (init) {
              v = a.b[e];
              a.x[e] = 0.f;
              a.r[e] = v;
              a.p[e] = 0.f;
            } else if (upd) {
              a.x[e] = fmaf(al, __ldcg(pc + e), a.x[e]);
              v = fmaf(-al, __ldcg(a.ap + e), a.r[e]);
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
              a.z[3 * v + c] = zi;
              acc[0] += (Acc)rd[3 * lane + c] * (Acc)rd[3 * lane + c];
              acc[1] += (Acc)rd[3 * lane + c] * (Acc)zi;
            }
          }
          __syncwarp();
          continue;
        }
        if (!mbar_wait(mbar, mphase)) {
          if (lane == 0) {
            atomicOr(a.bar + 2, ST_WAIT_TIMEOUT);
            s_abort = 1;
          }
          mbar_wait(mbar, mphase);  // bounded again: the copy may still land
          break;
        }
        mphase ^= 1;
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
            a.z[3 * a.dom_verts[vs + i / 3] + i % 3] = zi;
            acc[0] += (Acc)rd[i] * (Acc)rd[i];
            acc[1] += (Acc)rd[i] * (Acc)zi;
          }
        }
        __syncwarp();
      }
    } else {
      for (uint32_t v = row0 + ltid; v < row1; v += lthreads) {
        float rr[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const uint32_t e = 3 * v + c;
          if (init) {
            rr[c] = a.b[e];
            a.x[e] = 0.f;
            a.r[e] = rr[c];
            a.p[e] = 0.f;
          } else if (upd) {
            a.x[e] = fmaf(al, __ldcg(pc + e), a.x[e]);
            rr[c] = fmaf(-al, __ldcg(a.ap + e), a.r[e]);
            a.r[e] = rr[c];
          } else {
            rr[c] = a.r[e];
          }
        }
        const float* m9 = a.bjinv + 9 * (size_t)v;
        const float z0 = m9[0] * rr[0] + m9[1] * rr[1] + m9[2] * rr[2];
        const float z1 = m9[3] * rr[0] + m9[4] * rr[1] + m9[5] * rr[2];
        const float z2 = m9[6] * rr[0] + m9[7] * rr[1] + m9[8] * rr[2];
        a.z[3 * v] = z0;
        a.z[3 * v + 1] = z1;
        a.z[3 * v + 2] = z2;
        acc[0] += (Acc)rr[0] * (Acc)rr[0] + (Acc)rr[1] * (Acc)rr[1] + (Acc)rr[2] * (Acc)rr[2];
        acc[1] += (Acc)rr[0] * (Acc)z0 + (Acc)rr[1] * (Acc)z1 + (Acc)rr[2] * (Acc)z2;
      }
    }
  };

  // x = 0, r = b, z = M^-1 r; ||b|| and r.z
  domain_phase(true, a.p);
  if (!grid_dots<Acc, 2>(acc, K, s_cta, partials, parity, a.bar, target, s_tot) || s_abort) return;
  if (tid < K) {
    s_bnorm[tid] = fmax(sqrt((double)s_tot[0][tid]), 1e-30);
    s_res[tid] = sqrt((double)s_tot[0][tid]) / s_bnorm[tid];
    s_rz[tid] = (double)s_tot[1][tid];
  }
  __syncthreads();

  const uint32_t sub = tid % PP_LPR;
  const unsigned gmask = ((1u << PP_LPR) - 1u) << (lane & ~(PP_LPR - 1));
  uint32_t it_no = 0;
  for (;;) {
    if (a.probe && blockIdx.x == 0 && tid == 0 && it_no == 8) a.probe[0] = globaltimer();
    // phase 1: p = z + beta p_old (own rows, into the other buffer); Ap from the same
    // formula for every gathered column; p.Ap
    {
      const float* __restrict__ po = cur ? a.p2 : a.p;
      float* __restrict__ pn = cur ? a.p : a.p2;
      const float be = (float)s_beta[k];
      acc[0] = 0;
      for (uint32_t row = row0 + ltid / PP_LPR; row < row1; row += lthreads / PP_LPR) {
        Acc y0 = 0, y1 = 0, y2 = 0;
        auto block = [&](const float* __restrict__ m9, uint32_t c) {
          // same fused multiply-add order as the standalone system SpMV
          const Acc x0 = (Acc)fmaf(be, __ldcg(po + 3 * c), __ldcg(a.z + 3 * c));
          const Acc x1 = (Acc)fmaf(be, __ldcg(po + 3 * c + 1), __ldcg(a.z + 3 * c + 1));
          const Acc x2 = (Acc)fmaf(be, __ldcg(po + 3 * c + 2), __ldcg(a.z + 3 * c + 2));
          y0 = pp_fma((Acc)__ldg(m9 + 0), x0, y0);
          y0 = pp_fma((Acc)__ldg(m9 + 1), x1, y0);
          y0 = pp_fma((Acc)__ldg(m9 + 2), x2, y0);
          y1 = pp_fma((Acc)__ldg(m9 + 3), x0, y1);
          y1 = pp_fma((Acc)__ldg(m9 + 4), x1, y1);
          y1 = pp_fma((Acc)__ldg(m9 + 5), x2, y1);
          y2 = pp_fma((Acc)__ldg(m9 + 6), x0, y2);
          y2 = pp_fma((Acc)__ldg(m9 + 7), x1, y2);
          y2 = pp_fma((Acc)__ldg(m9 + 8), x2, y2);
        };
        const uint32_t ke = __ldg(a.rp + row + 1);
#pragma unroll 4
        for (uint32_t kk = __ldg(a.rp + row) + sub; kk < ke; kk += PP_LPR) block(a.val + 9 * (size_t)kk, __ldg(a.col + kk));
        const uint32_t ce = __ldg(a.crp + row + 1);
        for (uint32_t kk = __ldg(a.crp + row) + sub; kk < ce; kk += PP_LPR)
          block(a.cval + 9 * (size_t)kk, __ldg(a.ccol + kk));
#pragma unroll
        for (int o = PP_LPR / 2; o > 0; o >>= 1) {
          y0 += __shfl_xor_sync(gmask, y0, o, PP_LPR);
          y1 += __shfl_xor_sync(gmask, y1, o, PP_LPR);
          y2 += __shfl_xor_sync(gmask, y2, o, PP_LPR);
        }
        if (sub == 0) {
          const float f0 = (float)y0, f1 = (float)y1, f2 = (float)y2;
          const float q0 = fmaf(be, __ldcg(po + 3 * row), __ldcg(a.z + 3 * row));
          const float q1 = fmaf(be, __ldcg(po + 3 * row + 1), __ldcg(a.z + 3 * row + 1));
          const float q2 = fmaf(be, __ldcg(po + 3 * row + 2), __ldcg(a.z + 3 * row + 2));
          pn[3 * row] = q0;
          pn[3 * row + 1] = q1;
          pn[3 * row + 2] = q2;
          a.ap[3 * row] = f0;
          a.ap[3 * row + 1] = f1;
          a.ap[3 * row + 2] = f2;
          acc[0] += (Acc)q0 * (Acc)f0 + (Acc)q1 * (Acc)f1 + (Acc)q2 * (Acc)f2;
        }
      }
    }
    cur ^= 1;
    if (a.probe && blockIdx.x == 0 && tid == 0 && it_no == 8) a.probe[1] = globaltimer();
    if (!grid_dots<Acc, 1>(*(Acc(*)[1])acc, K, s_cta, partials, parity, a.bar, target, s_tot) || s_abort) return;
    if (a.probe && blockIdx.x == 0 && tid == 0 && it_no == 8) a.probe[2] = globaltimer();
    if (tid < K) {
      s_upd[tid] = 0;
      if (!s_done[tid]) {
        const double pap = (double)s_tot[0][tid];
        if (!(pap > 0.0)) {  // the reference breaks out (linsolve.rs:386)
          s_done[tid] = 1;
          s_status[tid] |= ST_PCG_BREAKDOWN;
        } else {
          s_alpha[tid] = s_rz[tid] / pap;
          s_upd[tid] = 1;
        }
      }
    }
    __syncthreads();
    // phase 2: x += alpha p, r -= alpha Ap, z = M^-1 r; r.r and r.z
    domain_phase(false, cur ? a.p2 : a.p);
    if (a.probe && blockIdx.x == 0 && tid == 0 && it_no == 8) a.probe[3] = globaltimer();
    if (!grid_dots<Acc, 2>(acc, K, s_cta, partials, parity, a.bar, target, s_tot) || s_abort) return;
    if (a.probe && blockIdx.x == 0 && tid == 0 && it_no == 8) a.probe[4] = globaltimer();
    if (tid < K && s_upd[tid]) {
      s_iters[tid] += 1;
      s_res[tid] = sqrt((double)s_tot[0][tid]) / s_bnorm[tid];
      if (s_res[tid] <= (double)a.tol || s_iters[tid] >= a.max_iter) {
        s_done[tid] = 1;
      } else {
        const double rz = (double)s_tot[1][tid];
        s_beta[tid] = rz / s_rz[tid];
        s_rz[tid] = rz;
      }
    }
    __syncthreads();
    ++it_no;
    bool all = true;
    for (int q = 0; q < K; ++q) all = all && s_done[q];
    if (all) break;
  }
  if (blockIdx.x == 0 && tid < K) {
    PcgInstResult o;
    o.iters = s_iters[tid];
    o.residual = s_res[tid];
    o.status = s_status[tid];
    o.done = s_done[tid];
    a.out[tid] = o;
  }
}

static void* persistent_kernel(const Scene& s) {
  if (!s.schwarz)
    return s.mixed ? (void*)k_pcg_persistent<MGUSO_PRECOND_BLOCK_JACOBI, double, float>
                   : (void*)k_pcg_persistent<MGUSO_PRECOND_BLOCK_JACOBI, float, float>;
  if (s.schwarz->half)
    return s.mixed ? (void*)k_pcg_persistent<MGUSO_PRECOND_SCHWARZ, double, __half>
                   : (void*)k_pcg_persistent<MGUSO_PRECOND_SCHWARZ, float, __half>;
  return s.mixed ? (void*)k_pcg_persistent<MGUSO_PRECOND_SCHWARZ, double, float>
                 : (void*)k_pcg_persistent<MGUSO_PRECOND_SCHWARZ, float, float>;
}

int pcg_persistent_configure(Scene& s, int* grid_out) {
  const bool sch = s.schwarz != nullptr;
  const size_t smem = !sch ? 0
                     : 128 + (size_t)PP_WARPS * (s.schwarz->half ? apply_slice_bytes<__half>() : apply_slice_bytes<float>());
  void* fn = persistent_kernel(s);
  if (smem) MG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PP_THREADS, smem));
  *grid_out = per_sm >= 1 ? s.ctx->sm_count : 0;
  return MGUSO_OK;
}

// Solves the scene's current system (work.b) into work.x with one cooperative launch.
// h_inst_row (host, ninst + 1 block-row offsets) splits the rows into instances; results go
// to out[0 .. ninst). Returns MGUSO_ERR_UNSUPPORTED when the kernel cannot be resident on
// every SM or a Schwarz domain spans two instances (the caller then uses the per-kernel PCG).
int pcg_persistent(Scene& s, const uint32_t* h_inst_row, uint32_t ninst, uint32_t active, PcgInstResult* out) {
  MG_CHECK_ARG(ninst >= 1 && ninst <= PCG_MAX_INST, "persistent PCG: 1..8 instances");
  if (s.pp_grid < 0) MG_TRY(pcg_persistent_configure(s, &s.pp_grid));
  if (s.pp_grid == 0 || (int)ninst > s.pp_grid) return MGUSO_ERR_UNSUPPORTED;
  cudaStream_t st = s.st;
  PcgWork& w = s.work;
  std::vector<uint32_t> key(h_inst_row, h_inst_row + ninst + 1);
  if (key != s.pp_key) {
    // CTAs per instance in proportion to its rows (at least one each)
    const uint32_t G = (uint32_t)s.pp_grid, nv = h_inst_row[ninst] - h_inst_row[0];
    std::vector<uint32_t> cnt(ninst, 1);
    uint32_t used = ninst;
    for (uint32_t k = 0; k < ninst; ++k) {
      const uint64_t want = (uint64_t)(G - ninst) * (h_inst_row[k + 1] - h_inst_row[k]) / std::max<uint32_t>(nv, 1);
      cnt[k] += (uint32_t)want;
      used += (uint32_t)want;
    }
    for (uint32_t k = 0; used < G; k = (k + 1) % ninst, ++used) cnt[k]++;
    std::vector<uint32_t> lay(3 * (PCG_MAX_INST + 1), 0);
    for (uint32_t k = 0; k <= ninst; ++k) lay[k] = h_inst_row[k];
    for (uint32_t k = 0; k < ninst; ++k) lay[PCG_MAX_INST + 1 + k + 1] = lay[PCG_MAX_INST + 1 + k] + cnt[k];
    uint32_t* dom = lay.data() + 2 * (PCG_MAX_INST + 1);
    if (s.schwarz) {
      // domains must be grouped by instance: domain d lies in one instance, in order
      mguso_schwarz* sw = s.schwarz.get();
      uint32_t kk = 0;
      dom[0] = 0;
      for (uint32_t d = 0; d < sw->ndom; ++d) {
        const uint32_t v0 = sw->h_dom_verts[sw->h_dom_start[d]];
        while (kk < ninst && v0 >= h_inst_row[kk + 1]) dom[++kk] = d;
        if (kk >= ninst) return MGUSO_ERR_UNSUPPORTED;
        for (uint32_t i = sw->h_dom_start[d]; i < sw->h_dom_start[d + 1]; ++i) {
          const uint32_t v = sw->h_dom_verts[i];
          if (v < h_inst_row[kk] || v >= h_inst_row[kk + 1]) return MGUSO_ERR_UNSUPPORTED;
        }
      }
      while (kk < ninst) dom[++kk] = sw->ndom;
    }
    MG_TRY(s.pp_inst.upload(lay.data(), lay.size(), st));
    s.pp_key = key;
  }
  MG_TRY(s.pp_bar.reserve(4));
  MG_TRY(s.pp_out.reserve(PCG_MAX_INST));
  MG_CUDA(cudaMemsetAsync(s.pp_bar.p, 0, 16, st));
  PersistentArgs a{};
  a.nv = s.nv;
  a.ninst = ninst;
  a.inst_row = s.pp_inst.p;
  a.cta_start = s.pp_inst.p + (PCG_MAX_INST + 1);
  a.dom_range = s.pp_inst.p + 2 * (PCG_MAX_INST + 1);
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
    a.ndom = sw->ndom;
  }
  a.b = w.b.p;
  a.x = w.x.p;
  a.r = w.r.p;
  a.z = w.z.p;
  a.p = w.p.p;
  MG_TRY(w.p2.reserve(w.n));
  a.p2 = w.p2.p;
  a.ap = w.ap.p;
  a.tol = s.p.cg_tol;
  a.active = active;
  a.max_iter = s.p.cg_max_iter;
  a.out = s.pp_out.p;
  // two alternating buffers x grid x (r.r, r.z)
  MG_TRY(s.pp_part.reserve(2ull * 2 * s.pp_grid));
  a.partials = s.pp_part.p;
  a.bar = s.pp_bar.p;
  static const bool probe = std::getenv("MGUSO_TRACE") != nullptr;
  if (probe) {
    MG_TRY(s.pp_probe.reserve(16));
    MG_CUDA(cudaMemsetAsync(s.pp_probe.p, 0, 16 * 8, st));
    a.probe = (unsigned long long*)s.pp_probe.p;
  }
  const bool sch = s.schwarz != nullptr;
  const size_t smem = !sch ? 0
                     : 128 + (size_t)PP_WARPS * (s.schwarz->half ? apply_slice_bytes<__half>() : apply_slice_bytes<float>());
  void* fn = persistent_kernel(s);
  void* args[] = {(void*)&a};
  MG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(s.pp_grid), dim3(PP_THREADS), args, smem, st));
  uint32_t err[4] = {0, 0, 0, 0};
  MG_CUDA(cudaMemcpyAsync(out, s.pp_out.p, sizeof(PcgInstResult) * ninst, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpyAsync(err, s.pp_bar.p, 16, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  if (probe) {
    unsigned long long t[16];
    MG_CUDA(cudaMemcpy(t, s.pp_probe.p, 16 * 8, cudaMemcpyDeviceToHost));
    if (t[4] > t[0])
      std::fprintf(stderr, "[mguso]   pcg iteration 8 us: p+Ap %.2f dot %.2f x,r+precond %.2f dots %.2f"
                   "\n", (t[1] - t[0]) * 1e-3, (t[2] - t[1]) * 1e-3, (t[3] - t[2]) * 1e-3, (t[4] - t[3]) * 1e-3);
  }
  if (err[2] & ST_WAIT_TIMEOUT) {
    set_error("persistent PCG: a bounded grid-barrier or bulk-copy wait timed out");
    return MGUSO_ERR_TIMEOUT;
  }
  return MGUSO_OK;
}

}  // namespace mg
