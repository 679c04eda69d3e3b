// 3x3 block-sparse (BSR) operator: scalar-CSR -> BSR conversion and the FP32 SpMV.
//
// The reference multiplies a scalar CSR with one thread per scalar row
// (engine-gpu/src/shaders/pcg_ops.wgsl:76-93). Its matrix is 3x3-block structured
// (implicit.rs:2394-3103 pushes 9 entries per vertex pair), so here it is stored as BSR:
// values 9 floats per block (row-major), one u32 column per block. The main kernel stages
// each tile's value and column ranges into shared memory with 1-D TMA bulk copies
// (16-byte aligned, 128-bit transactions), double-buffered per persistent CTA, and
// multiplies one block row per thread; x is gathered through the read-only path (it is
// L2 resident at every size this library targets).
#include <algorithm>
#include <cstring>

#include "reduce.cuh"

namespace mg {

int device_sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// ---------------------------------------------------------------------------------------
// Host conversion of the reference's scalar CSR into BSR.
// ---------------------------------------------------------------------------------------
int bsr_build_host_from_csr(const mguso_csr* a, uint32_t& nb, std::vector<uint32_t>& row_ptr,
                            std::vector<uint32_t>& col, std::vector<float>& val) {
  MG_CHECK_ARG(a && a->row_ptr && (a->row_ptr[a->n] == 0 || (a->col_idx && a->values)), "null CSR");
  MG_CHECK_ARG(a->n % 3 == 0, "CSR order must be a multiple of 3 (3 DOFs per vertex)");
  nb = a->n / 3;
  row_ptr.assign(nb + 1, 0);
  col.clear();
  val.clear();
  std::vector<uint32_t> cols;
  for (uint32_t v = 0; v < nb; ++v) {
    cols.clear();
    for (int r = 0; r < 3; ++r) {
      uint32_t row = 3 * v + r;
      for (uint32_t k = a->row_ptr[row]; k < a->row_ptr[row + 1]; ++k) {
        uint32_t c = a->col_idx[k];
        MG_CHECK_ARG(c < a->n, "CSR column index out of range");
        cols.push_back(c / 3);
      }
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    size_t base = col.size();
    col.insert(col.end(), cols.begin(), cols.end());
    val.resize(9 * col.size(), 0.0f);
    for (int r = 0; r < 3; ++r) {
      uint32_t row = 3 * v + r;
      for (uint32_t k = a->row_ptr[row]; k < a->row_ptr[row + 1]; ++k) {
        uint32_t cb = a->col_idx[k] / 3;
        size_t j = std::lower_bound(cols.begin(), cols.end(), cb) - cols.begin();
        val[9 * (base + j) + 3 * r + a->col_idx[k] % 3] += a->values[k];
      }
    }
    row_ptr[v + 1] = (uint32_t)col.size();
  }
  return MGUSO_OK;
}

int bsr_upload(mguso_bsr* m, uint32_t nb, const std::vector<uint32_t>& row_ptr, const std::vector<uint32_t>& col,
               const float* val_host) {
  cudaStream_t s = m->ctx->stream;
  m->nb = nb;
  m->nnzb = row_ptr[nb];
  m->h_row_ptr = row_ptr;
  m->h_col = col;
  MG_TRY(m->row_ptr.upload(row_ptr.data(), nb + 1, s));
  MG_TRY(m->col.upload(col.data(), m->nnzb, s));
  MG_TRY(m->val.reserve((size_t)9 * m->nnzb));
  if (m->nnzb)
    MG_CUDA(cudaMemcpyAsync(m->val.p, val_host, sizeof(float) * 9 * m->nnzb, cudaMemcpyHostToDevice, s));
  MG_TRY(m->status.reserve(4));
  MG_CUDA(cudaMemsetAsync(m->status.p, 0, 16, s));
  m->tilings.clear();
  m->sell.ready = false;
  if (m->nnzb) m->h_val_keep.assign(val_host, val_host + (size_t)9 * m->nnzb);
  MG_TRY(bsr_prepare_tilings(m));
  MG_CUDA(cudaStreamSynchronize(s));
  return MGUSO_OK;
}

// ---------------------------------------------------------------------------------------
// SpMV kernels
// ---------------------------------------------------------------------------------------
template <class Acc>
struct DotAcc {
  Acc v = 0;
  __device__ void add(float a, float b) { v += (Acc)a * (Acc)b; }
};

// One block row: y_r = sum_k A_k x[col_k]; 4 independent chains for gather latency.
__device__ __forceinline__ void row_mul(const float* __restrict__ a, const uint32_t* __restrict__ c, uint32_t nblk,
                                        const float* __restrict__ x, float& y0, float& y1, float& y2) {
  float s0 = 0.f, s1 = 0.f, s2 = 0.f;
  uint32_t k = 0;
  for (; k + 2 <= nblk; k += 2) {
    uint32_t c0 = c[k], c1 = c[k + 1];
    float xa0 = __ldg(x + 3 * c0), xa1 = __ldg(x + 3 * c0 + 1), xa2 = __ldg(x + 3 * c0 + 2);
    float xb0 = __ldg(x + 3 * c1), xb1 = __ldg(x + 3 * c1 + 1), xb2 = __ldg(x + 3 * c1 + 2);
    const float* p = a + 9 * k;
    s0 = fmaf(p[0], xa0, s0); s0 = fmaf(p[1], xa1, s0); s0 = fmaf(p[2], xa2, s0);
    s1 = fmaf(p[3], xa0, s1); s1 = fmaf(p[4], xa1, s1); s1 = fmaf(p[5], xa2, s1);
    s2 = fmaf(p[6], xa0, s2); s2 = fmaf(p[7], xa1, s2); s2 = fmaf(p[8], xa2, s2);
    s0 = fmaf(p[9], xb0, s0); s0 = fmaf(p[10], xb1, s0); s0 = fmaf(p[11], xb2, s0);
    s1 = fmaf(p[12], xb0, s1); s1 = fmaf(p[13], xb1, s1); s1 = fmaf(p[14], xb2, s1);
    s2 = fmaf(p[15], xb0, s2); s2 = fmaf(p[16], xb1, s2); s2 = fmaf(p[17], xb2, s2);
  }
  if (k < nblk) {
    uint32_t c0 = c[k];
    float xa0 = __ldg(x + 3 * c0), xa1 = __ldg(x + 3 * c0 + 1), xa2 = __ldg(x + 3 * c0 + 2);
    const float* p = a + 9 * k;
    s0 = fmaf(p[0], xa0, s0); s0 = fmaf(p[1], xa1, s0); s0 = fmaf(p[2], xa2, s0);
    s1 = fmaf(p[3], xa0, s1); s1 = fmaf(p[4], xa1, s1); s1 = fmaf(p[5], xa2, s1);
    s2 = fmaf(p[6], xa0, s2); s2 = fmaf(p[7], xa1, s2); s2 = fmaf(p[8], xa2, s2);
  }
  y0 = s0;
  y1 = s1;
  y2 = s2;
}

// Persistent TMA-staged SpMV. Shared memory: STAGES mbarriers, then per stage the value
// bytes (val_stage_bytes) and the column bytes (col_stage_bytes) of one tile.
template <int STAGES, class Acc>
__global__ void k_spmv_tma(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                           const float* __restrict__ val, const uint32_t* __restrict__ tile_row, uint32_t ntiles,
                           uint32_t val_stage_bytes, uint32_t col_stage_bytes, const float* __restrict__ x,
                           float* __restrict__ y, uint32_t* status, DotSink dot, int with_dot) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (with_dot && dot.sc->done) return;
  uint64_t* bar = (uint64_t*)smem;
  unsigned char* stage_base = smem + 128;
  const uint32_t stage_bytes = val_stage_bytes + col_stage_bytes;
  const int tid = threadIdx.x;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  auto issue = [&](uint32_t tile, int s) {
    uint32_t b0 = row_ptr[tile_row[tile]], b1 = row_ptr[tile_row[tile + 1]];
    uint64_t vs = (uint64_t)b0 * 36u, ve = (uint64_t)b1 * 36u;
    uint64_t vs_al = vs & ~15ull, ve_al = (ve + 15ull) & ~15ull;
    uint64_t cs = (uint64_t)b0 * 4u, ce = (uint64_t)b1 * 4u;
    uint64_t cs_al = cs & ~15ull, ce_al = (ce + 15ull) & ~15ull;
    uint32_t vbytes = (uint32_t)(ve_al - vs_al), cbytes = (uint32_t)(ce_al - cs_al);
    unsigned char* st = stage_base + (size_t)s * stage_bytes;
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[s], vbytes + cbytes);
    if (vbytes) bulk_g2s(st, (const unsigned char*)val + vs_al, vbytes, &bar[s]);
    if (cbytes) bulk_g2s(st + val_stage_bytes, (const unsigned char*)col + cs_al, cbytes, &bar[s]);
  };

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      uint32_t t = blockIdx.x + (uint32_t)s * gridDim.x;
      if (t < ntiles) issue(t, s);
    }
  }

  DotAcc<Acc> acc;
  for (uint32_t k = 0;; ++k) {
    uint32_t t = blockIdx.x + k * gridDim.x;
    if (t >= ntiles) break;
    int s = (int)(k % STAGES);
    uint32_t phase = (k / STAGES) & 1u;
    bool ok = mbar_wait(&bar[s], phase);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(status, ST_WAIT_TIMEOUT);
      return;
    }
    uint32_t r0 = tile_row[t], r1 = tile_row[t + 1];
    uint32_t b0 = row_ptr[r0];
    const unsigned char* st = stage_base + (size_t)s * stage_bytes;
    const float* sv = (const float*)(st + ((uint64_t)b0 * 36u - (((uint64_t)b0 * 36u) & ~15ull)));
    const uint32_t* sc = (const uint32_t*)(st + val_stage_bytes + ((uint64_t)b0 * 4u - (((uint64_t)b0 * 4u) & ~15ull)));
    for (uint32_t r = r0 + tid; r < r1; r += blockDim.x) {
      uint32_t kb = row_ptr[r] - b0, ke = row_ptr[r + 1] - b0;
      float y0, y1, y2;
      row_mul(sv + 9 * kb, sc + kb, ke - kb, x, y0, y1, y2);
      y[3 * r] = y0;
      y[3 * r + 1] = y1;
      y[3 * r + 2] = y2;
      if (with_dot) {
        acc.add(x[3 * r], y0);
        acc.add(x[3 * r + 1], y1);
        acc.add(x[3 * r + 2], y2);
      }
    }
    __syncthreads();
    if (tid == 0) {
      uint32_t t2 = t + (uint32_t)STAGES * gridDim.x;
      if (t2 < ntiles) issue(t2, s);
    }
  }
  if (with_dot) grid_dot_commit<Acc>(dot, acc.v);
}

// Direct variant: one block row per thread, values read straight from global memory.
template <class Acc>
__global__ void k_spmv_direct(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                              const float* __restrict__ val, uint32_t nb, const float* __restrict__ x,
                              float* __restrict__ y, DotSink dot, int with_dot) {
  if (with_dot && dot.sc->done) return;
  DotAcc<Acc> acc;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nb; r += gridDim.x * blockDim.x) {
    uint32_t kb = row_ptr[r], ke = row_ptr[r + 1];
    float y0, y1, y2;
    row_mul(val + 9 * (size_t)kb, col + kb, ke - kb, x, y0, y1, y2);
    y[3 * r] = y0;
    y[3 * r + 1] = y1;
    y[3 * r + 2] = y2;
    if (with_dot) {
      acc.add(x[3 * r], y0);
      acc.add(x[3 * r + 1], y1);
      acc.add(x[3 * r + 2], y2);
    }
  }
  if (with_dot) grid_dot_commit<Acc>(dot, acc.v);
}

// Sliced-ELL variant: one block row per thread, 32 rows per warp-aligned slice; values and
// columns are streamed with evict-first loads, x is gathered through the read-only path.
template <class Acc>
__global__ void __launch_bounds__(256) k_spmv_sell(const uint32_t* __restrict__ slice_base,
                                                   const uint32_t* __restrict__ scol, const float* __restrict__ sval,
                                                   uint32_t nb, const float* __restrict__ x, float* __restrict__ y,
                                                   DotSink dot, int with_dot) {
  if (with_dot && dot.sc->done) return;
  DotAcc<Acc> acc;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < ((nb + 31u) & ~31u); r += gridDim.x * blockDim.x) {
    const uint32_t sl = r >> 5, lane = r & 31u;
    const uint32_t b0 = slice_base[sl], b1 = slice_base[sl + 1];
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    const uint32_t* cp = scol + (size_t)b0 * 32 + lane;
    const float* vp = sval + (size_t)b0 * 288 + lane;
#pragma unroll 2
    for (uint32_t k = b0; k < b1; ++k) {
      uint32_t c = __ldcs(cp);
      float a0 = __ldcs(vp), a1 = __ldcs(vp + 32), a2 = __ldcs(vp + 64);
      float a3 = __ldcs(vp + 96), a4 = __ldcs(vp + 128), a5 = __ldcs(vp + 160);
      float a6 = __ldcs(vp + 192), a7 = __ldcs(vp + 224), a8 = __ldcs(vp + 256);
      float x0 = __ldg(x + 3 * c), x1 = __ldg(x + 3 * c + 1), x2 = __ldg(x + 3 * c + 2);
      s0 = fmaf(a0, x0, s0); s0 = fmaf(a1, x1, s0); s0 = fmaf(a2, x2, s0);
      s1 = fmaf(a3, x0, s1); s1 = fmaf(a4, x1, s1); s1 = fmaf(a5, x2, s1);
      s2 = fmaf(a6, x0, s2); s2 = fmaf(a7, x1, s2); s2 = fmaf(a8, x2, s2);
      cp += 32;
      vp += 288;
    }
    if (r < nb) {
      y[3 * r] = s0;
      y[3 * r + 1] = s1;
      y[3 * r + 2] = s2;
      if (with_dot) {
        acc.add(x[3 * r], s0);
        acc.add(x[3 * r + 1], s1);
        acc.add(x[3 * r + 2], s2);
      }
    }
  }
  if (with_dot) grid_dot_commit<Acc>(dot, acc.v);
}

int bsr_build_sell(mguso_bsr* m) {
  SellLayout& L = m->sell;
  if (L.ready) return MGUSO_OK;
  const uint32_t nb = m->nb;
  L.nslices = (nb + 31) / 32;
  std::vector<uint32_t> base(L.nslices + 1, 0);
  for (uint32_t sl = 0; sl < L.nslices; ++sl) {
    uint32_t mx = 0;
    for (uint32_t r = sl * 32; r < std::min(nb, sl * 32 + 32); ++r)
      mx = std::max(mx, m->h_row_ptr[r + 1] - m->h_row_ptr[r]);
    base[sl + 1] = base[sl] + mx;
  }
  L.total_k = base[L.nslices];
  std::vector<uint32_t> col((size_t)32 * L.total_k, 0);
  std::vector<float> val((size_t)288 * L.total_k, 0.0f);
  for (uint32_t r = 0; r < L.nslices * 32; ++r) {
    uint32_t sl = r >> 5, lane = r & 31;
    uint32_t len = base[sl + 1] - base[sl];
    uint32_t kb = r < nb ? m->h_row_ptr[r] : 0, ke = r < nb ? m->h_row_ptr[r + 1] : 0;
    for (uint32_t k = 0; k < len; ++k) {
      size_t g = (size_t)base[sl] + k;
      if (kb + k < ke) {
        col[g * 32 + lane] = m->h_col[kb + k];
        for (int e = 0; e < 9; ++e) val[(g * 9 + e) * 32 + lane] = m->h_val_keep[9 * (size_t)(kb + k) + e];
      } else {
        col[g * 32 + lane] = r < nb ? r : 0;
      }
    }
  }
  cudaStream_t s = m->ctx->stream;
  MG_TRY(L.slice_base.upload(base.data(), base.size(), s));
  MG_TRY(L.col.upload(col.data(), col.size(), s));
  MG_TRY(L.val.upload(val.data(), val.size(), s));
  MG_CUDA(cudaStreamSynchronize(s));
  L.ready = true;
  return MGUSO_OK;
}

// ---------------------------------------------------------------------------------------
// Tilings
// ---------------------------------------------------------------------------------------
static const int kTilingShapes[][2] = {{128, 2}, {256, 2}, {128, 3}, {64, 4}};

template <int STAGES>
static void* tma_kernel_ptr(bool mixed) {
  return mixed ? (void*)k_spmv_tma<STAGES, double> : (void*)k_spmv_tma<STAGES, float>;
}
static void* tma_kernel(int stages, bool mixed) {
  switch (stages) {
    case 2: return tma_kernel_ptr<2>(mixed);
    case 3: return tma_kernel_ptr<3>(mixed);
    default: return tma_kernel_ptr<4>(mixed);
  }
}

int bsr_prepare_tilings(mguso_bsr* m) {
  int sms = m->ctx ? m->ctx->sm_count : 148;
  uint32_t max_row = 0;
  for (uint32_t r = 0; r < m->nb; ++r) max_row = std::max(max_row, m->h_row_ptr[r + 1] - m->h_row_ptr[r]);
  for (auto& sh : kTilingShapes) {
    auto t = std::make_unique<SpmvTiling>();
    t->rows = sh[0];
    t->stages = sh[1];
    t->cap = (uint32_t)t->rows * 8u;
    t->val_stage_bytes = ((t->cap * 36u + 32u) + 127u) & ~127u;
    t->col_stage_bytes = ((t->cap * 4u + 32u) + 127u) & ~127u;
    size_t smem = 128 + (size_t)t->stages * (t->val_stage_bytes + t->col_stage_bytes);
    t->ok = max_row <= t->cap && smem <= 227 * 1024;
    if (t->ok) {
      std::vector<uint32_t> tr;
      tr.push_back(0);
      uint32_t r = 0;
      while (r < m->nb) {
        uint32_t r0 = r, b0 = m->h_row_ptr[r];
        while (r < m->nb && r - r0 < (uint32_t)t->rows && m->h_row_ptr[r + 1] - b0 <= t->cap) ++r;
        tr.push_back(r);
      }
      t->ntiles = (uint32_t)tr.size() - 1;
      MG_TRY(t->tile_row.upload(tr.data(), tr.size(), m->ctx->stream));
      void* fn = tma_kernel(t->stages, false);
      MG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      MG_CUDA(cudaFuncSetAttribute(tma_kernel(t->stages, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
      int per_sm = 0;
      MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, t->rows, smem));
      per_sm = std::max(per_sm, 1);
      t->grid = (int)std::min<uint64_t>((uint64_t)sms * per_sm, std::max<uint32_t>(t->ntiles, 1));
      t->grid = std::min(t->grid, MAX_PARTIALS);
    }
    m->tilings.push_back(std::move(t));
  }
  // default choice: first usable tiling
  m->tiling_choice = -1;
  for (size_t i = 0; i < m->tilings.size(); ++i)
    if (m->tilings[i]->ok) {
      m->tiling_choice = (int)i;
      break;
    }
  return MGUSO_OK;
}

static int launch_spmv(mguso_bsr* m, int variant, int tiling, const float* x, float* y, cudaStream_t s,
                       const DotSink* dot) {
  DotSink d{};
  int with_dot = dot ? 1 : 0;
  if (dot) d = *dot;
  bool mixed = dot && dot->mixed;
  if (m->nb == 0) return MGUSO_OK;
  if (variant == SPMV_SELL && m->sell.ready) {
    int threads = 256;
    uint32_t rows = m->sell.nslices * 32;
    int grid = (int)std::min<uint64_t>(ceil_div(rows, threads), with_dot ? MAX_PARTIALS : 1u << 20);
    const SellLayout& L = m->sell;
    if (mixed)
      k_spmv_sell<double><<<grid, threads, 0, s>>>(L.slice_base.p, L.col.p, L.val.p, m->nb, x, y, d, with_dot);
    else
      k_spmv_sell<float><<<grid, threads, 0, s>>>(L.slice_base.p, L.col.p, L.val.p, m->nb, x, y, d, with_dot);
    MG_CUDA(cudaGetLastError());
    return MGUSO_OK;
  }
  if (variant == SPMV_TMA && tiling >= 0 && m->tilings[tiling]->ok) {
    SpmvTiling& t = *m->tilings[tiling];
    size_t smem = 128 + (size_t)t.stages * (t.val_stage_bytes + t.col_stage_bytes);
    void* fn = tma_kernel(t.stages, mixed);
    const uint32_t* rp = m->row_ptr.p;
    const uint32_t* cl = m->col.p;
    const float* vl = m->val.p;
    const uint32_t* trp = t.tile_row.p;
    uint32_t nt = t.ntiles, vsb = t.val_stage_bytes, csb = t.col_stage_bytes;
    uint32_t* stp = m->status.p;
    void* args[] = {(void*)&rp, (void*)&cl, (void*)&vl, (void*)&trp, (void*)&nt, (void*)&vsb, (void*)&csb,
                    (void*)&x, (void*)&y, (void*)&stp, (void*)&d, (void*)&with_dot};
    MG_CUDA(cudaLaunchKernel(fn, dim3(t.grid), dim3(t.rows), args, smem, s));
  } else {
    int threads = 256;
    int grid = (int)std::min<uint64_t>(ceil_div(m->nb, threads), with_dot ? MAX_PARTIALS : 1u << 20);
    if (mixed)
      k_spmv_direct<double><<<grid, threads, 0, s>>>(m->row_ptr.p, m->col.p, m->val.p, m->nb, x, y, d, with_dot);
    else
      k_spmv_direct<float><<<grid, threads, 0, s>>>(m->row_ptr.p, m->col.p, m->val.p, m->nb, x, y, d, with_dot);
    MG_CUDA(cudaGetLastError());
  }
  return MGUSO_OK;
}

int bsr_spmv(mguso_bsr* m, const float* x, float* y, cudaStream_t s, const DotSink* dot) {
  int variant = m->variant;
  if (variant == SPMV_AUTO) variant = m->tiling_choice >= 0 ? SPMV_TMA : SPMV_DIRECT;
  return launch_spmv(m, variant, m->tiling_choice, x, y, s, dot);
}

// Times every variant/tiling with CUDA events on the context stream and keeps the best.
int bsr_autotune(mguso_bsr* m, float* best_us) {
  cudaStream_t s = m->ctx->stream;
  DevBuf<float> x, y;
  MG_TRY(x.reserve((size_t)3 * m->nb));
  MG_TRY(y.reserve((size_t)3 * m->nb));
  MG_CUDA(cudaMemsetAsync(x.p, 0, sizeof(float) * 3 * m->nb, s));
  cudaEvent_t e0, e1;
  MG_CUDA(cudaEventCreate(&e0));
  MG_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_var = SPMV_DIRECT, best_til = -1;
  const int reps = 20;
  auto time_it = [&](int var, int til) -> float {
    for (int i = 0; i < 3; ++i) launch_spmv(m, var, til, x.p, y.p, s, nullptr);
    cudaEventRecord(e0, s);
    for (int i = 0; i < reps; ++i) launch_spmv(m, var, til, x.p, y.p, s, nullptr);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return 1000.f * ms / reps;
  };
  float us = time_it(SPMV_DIRECT, -1);
  best = us;
  if (bsr_build_sell(m) == MGUSO_OK) {
    us = time_it(SPMV_SELL, -1);
    if (us < best) {
      best = us;
      best_var = SPMV_SELL;
    }
  }
  for (size_t i = 0; i < m->tilings.size(); ++i) {
    if (!m->tilings[i]->ok) continue;
    us = time_it(SPMV_TMA, (int)i);
    if (us < best) {
      best = us;
      best_var = SPMV_TMA;
      best_til = (int)i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MG_CUDA(cudaGetLastError());
  m->variant = best_var;
  if (best_til >= 0) m->tiling_choice = best_til;
  if (best_us) *best_us = best;
  return MGUSO_OK;
}

}  // namespace mg
