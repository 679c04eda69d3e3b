// One-level additive Schwarz preconditioner and 3x3 block Jacobi on the GPU.
//
// Reference: SchwarzTopology::{build, factorize, apply} (engine-core/src/linsolve.rs:
// 126-258): greedy BFS domains of <= D vertices over the block graph, per-domain dense
// block with the diagonal floor 1e-6*(tr/m) + 1e-8, Cholesky in f64 (fallback to the
// diagonal when a pivot is <= 1e-14), and z = (L L^T)^-1 r per domain.
//
// B200 layout: factorisation is one CTA per domain in FP64 shared memory (right-looking
// Cholesky, then W = L^-1), and what is stored is W in FP32 as swizzled 32 x 32 tiles of
// its lower block-triangle (4 KB aligned per tile). The apply is two dense triangular
// matvecs per domain, z = W^T (W r), with no sequential triangular sweeps: one warp per
// domain stages its tiles into shared memory with a single 1-D TMA bulk copy.
#include <algorithm>
#include <deque>

#include "reduce.cuh"
#include "tiles.cuh"

namespace mg {

int schwarz_configure();
int schwarz_build_coarse(mguso_schwarz* s);
int schwarz_factor_with(mguso_schwarz* s, const uint32_t* c_rp, const uint32_t* c_col, const float* c_val,
                        cudaStream_t st);

// ---------------------------------------------------------------------------------------
// Host: BFS domains over the block pattern (linsolve.rs:152-173).
// ---------------------------------------------------------------------------------------
int schwarz_build(mguso_schwarz* s) {
  mguso_bsr* a = s->a;
  uint32_t nb = a->nb;
  const auto& rp = a->h_row_ptr;
  const auto& cl = a->h_col;
  std::vector<uint8_t> assigned(nb, 0);
  s->h_dom_start.assign(1, 0);
  s->h_dom_verts.clear();
  s->h_dom_verts.reserve(nb);
  s->h_dom_of.assign(nb, 0);
  std::vector<uint32_t> loc(nb, 0);
  uint32_t D = std::max<uint32_t>(s->domain, 1);
  uint32_t max_m = 0;
  // Vertices with no off-diagonal block (pinned collider vertices, unconnected points)
  // would each be a one-vertex domain; they are packed D at a time instead. Their blocks
  // do not couple, so the packed domain's factor is block diagonal and the preconditioner
  // is unchanged (only the diagonal floor averages over the packed vertices).
  std::vector<uint32_t> singles;
  for (uint32_t v = 0; v < nb && s->pack_singles; ++v) {
    bool iso = true;
    for (uint32_t k = rp[v]; k < rp[v + 1] && iso; ++k) iso = cl[k] == v;
    if (iso) {
      singles.push_back(v);
      assigned[v] = 1;
    }
  }
  s->h_dom_diag.clear();
  auto close_domain = [&](size_t base, bool diag = false) {
    uint32_t d = (uint32_t)s->h_dom_start.size() - 1;
    s->h_dom_diag.push_back(diag ? 1 : 0);
    for (size_t i = base; i < s->h_dom_verts.size(); ++i) {
      s->h_dom_of[s->h_dom_verts[i]] = d;
      loc[s->h_dom_verts[i]] = (uint32_t)(i - base);
    }
    s->h_dom_start.push_back((uint32_t)s->h_dom_verts.size());
    max_m = std::max<uint32_t>(max_m, 3 * (uint32_t)(s->h_dom_verts.size() - base));
  };
  // instance by instance (vertex ranges; one range for a single scene), so that each
  // domain lies in one instance and the domains of an instance are contiguous
  std::vector<uint32_t> ranges = s->inst_vert;
  if (ranges.size() < 2) ranges = {0, nb};
  size_t si = 0;
  for (size_t r = 0; r + 1 < ranges.size(); ++r) {
  for (uint32_t seed = ranges[r]; seed < ranges[r + 1]; ++seed) {
    if (assigned[seed]) continue;
    size_t base = s->h_dom_verts.size();
    s->h_dom_verts.push_back(seed);
    assigned[seed] = 1;
    size_t fi = base;
    while (s->h_dom_verts.size() - base < D && fi < s->h_dom_verts.size()) {
      uint32_t v = s->h_dom_verts[fi++];
      // block columns are sorted and unique per row: the reference's sorted, deduped
      // adjacency minus the vertex itself.
      for (uint32_t k = rp[v]; k < rp[v + 1]; ++k) {
        uint32_t nbv = cl[k];
        if (nbv == v) continue;
        if (!assigned[nbv] && s->h_dom_verts.size() - base < D) {
          assigned[nbv] = 1;
          s->h_dom_verts.push_back(nbv);
        }
      }
    }
    close_domain(base);
  }
  // this instance's isolated vertices, D per domain
  size_t se = si;
  while (se < singles.size() && singles[se] < ranges[r + 1]) ++se;
  for (size_t i = si; i < se; i += D) {
    size_t base = s->h_dom_verts.size();
    for (size_t j = i; j < std::min(se, i + D); ++j) s->h_dom_verts.push_back(singles[j]);
    close_domain(base, true);
  }
  si = se;
  }
  s->ndom = (uint32_t)s->h_dom_start.size() - 1;
  s->max_m = max_m;
  std::vector<uint64_t> off(s->ndom + 1, 0);
  for (uint32_t d = 0; d < s->ndom; ++d) {
    uint64_t m = 3ull * (s->h_dom_start[d + 1] - s->h_dom_start[d]);
    uint64_t t = s->h_dom_diag[d] ? 0 : (m + 31) / 32;
    off[d + 1] = off[d] + t * (t + 1) / 2 * TILE_FLOATS;
  }
  s->fac_floats = off[s->ndom];
  MG_TRY(s->dom_diag.upload(s->h_dom_diag.data(), std::max<size_t>(s->h_dom_diag.size(), 1), a->ctx->stream));
  // each domain's instance (the range of its first vertex), for factorisations that skip
  // the instances a batch no longer iterates
  std::vector<uint8_t> dom_inst(std::max<uint32_t>(s->ndom, 1), 0);
  for (uint32_t d = 0; d < s->ndom; ++d) {
    const uint32_t v = s->h_dom_verts[s->h_dom_start[d]];
    dom_inst[d] = (uint8_t)(std::upper_bound(ranges.begin(), ranges.end(), v) - ranges.begin() - 1);
  }
  MG_TRY(s->dom_inst.upload(dom_inst.data(), dom_inst.size(), a->ctx->stream));
  MG_TRY(s->vfac.reserve(6 * (size_t)std::max<uint32_t>(nb, 1)));
  cudaStream_t st = a->ctx->stream;
  MG_TRY(s->dom_start.upload(s->h_dom_start.data(), s->h_dom_start.size(), st));
  MG_TRY(s->dom_verts.upload(s->h_dom_verts.data(), s->h_dom_verts.size(), st));
  MG_TRY(s->dom_of.upload(s->h_dom_of.data(), nb, st));
  MG_TRY(s->loc.upload(loc.data(), nb, st));
  MG_TRY(s->fac_off.upload(off.data(), off.size(), st));
  if (s->half) {
    MG_TRY(s->fac_h.reserve(std::max<uint64_t>(s->fac_floats, 8)));
    MG_TRY(s->fac_scale.reserve(std::max<uint32_t>(s->ndom, 1)));
  } else {
    MG_TRY(s->fac.reserve(std::max<uint64_t>(s->fac_floats, 4)));
  }
  MG_TRY(s->status.reserve(4));
  MG_CUDA(cudaMemsetAsync(s->status.p, 0, 16, st));
  if (s->levels == 2) MG_TRY(schwarz_build_coarse(s));
  MG_CUDA(cudaStreamSynchronize(st));
  MG_TRY(schwarz_configure());
  return MGUSO_OK;
}

// Coarse level of the two-level form (MultilevelSchwarz::build, linsolve.rs:555-608): coarse
// node G = level-0 domain G; G and H are adjacent when some block (i, j) of the pattern has
// i in G and j in H; coarse domains are the reference's greedy BFS over that adjacency
// (seeds in node order, neighbours in ascending order, <= domain nodes each).
int schwarz_build_coarse(mguso_schwarz* s) {
  mguso_bsr* a = s->a;
  const uint32_t nb = a->nb, nd = s->ndom;
  const auto& rp = a->h_row_ptr;
  const auto& cl = a->h_col;
  std::vector<std::vector<uint32_t>> adj(nd);
  for (uint32_t v = 0; v < nb; ++v) {
    const uint32_t g = s->h_dom_of[v];
    for (uint32_t k = rp[v]; k < rp[v + 1]; ++k) {
      const uint32_t h = s->h_dom_of[cl[k]];
      if (h != g) adj[g].push_back(h);
    }
  }
  for (auto& x : adj) {
    std::sort(x.begin(), x.end());
    x.erase(std::unique(x.begin(), x.end()), x.end());
  }
  const uint32_t D = std::max<uint32_t>(s->domain, 1);
  std::vector<uint8_t> assigned(nd, 0);
  std::vector<uint32_t> cdom_of(nd, 0), cloc(nd, 0);
  s->h_cdom_start.assign(1, 0);
  s->h_cdom_nodes.clear();
  s->max_m1 = 0;
  for (uint32_t seed = 0; seed < nd; ++seed) {
    if (assigned[seed]) continue;
    const size_t base = s->h_cdom_nodes.size();
    s->h_cdom_nodes.push_back(seed);
    assigned[seed] = 1;
    size_t fi = base;
    while (s->h_cdom_nodes.size() - base < D && fi < s->h_cdom_nodes.size()) {
      const uint32_t g = s->h_cdom_nodes[fi++];
      for (uint32_t h : adj[g])
        if (!assigned[h] && s->h_cdom_nodes.size() - base < D) {
          assigned[h] = 1;
          s->h_cdom_nodes.push_back(h);
        }
    }
    const uint32_t d1 = (uint32_t)s->h_cdom_start.size() - 1;
    for (size_t i = base; i < s->h_cdom_nodes.size(); ++i) {
      cdom_of[s->h_cdom_nodes[i]] = d1;
      cloc[s->h_cdom_nodes[i]] = (uint32_t)(i - base);
    }
    s->h_cdom_start.push_back((uint32_t)s->h_cdom_nodes.size());
    s->max_m1 = std::max<uint32_t>(s->max_m1, 3 * (uint32_t)(s->h_cdom_nodes.size() - base));
  }
  s->ncdom = (uint32_t)s->h_cdom_start.size() - 1;
  std::vector<uint64_t> off(s->ncdom + 1, 0);
  for (uint32_t d = 0; d < s->ncdom; ++d) {
    const uint64_t m = 3ull * (s->h_cdom_start[d + 1] - s->h_cdom_start[d]);
    const uint64_t t = (m + 31) / 32;
    off[d + 1] = off[d] + t * (t + 1) / 2 * TILE_FLOATS;
  }
  std::vector<uint32_t> sorted(s->h_dom_verts);
  for (uint32_t d = 0; d < nd; ++d)
    std::sort(sorted.begin() + s->h_dom_start[d], sorted.begin() + s->h_dom_start[d + 1]);
  cudaStream_t st = a->ctx->stream;
  MG_TRY(s->cdom_start.upload(s->h_cdom_start.data(), s->h_cdom_start.size(), st));
  MG_TRY(s->cdom_nodes.upload(s->h_cdom_nodes.data(), std::max<size_t>(s->h_cdom_nodes.size(), 1), st));
  MG_TRY(s->cdom_of.upload(cdom_of.data(), std::max<size_t>(nd, 1), st));
  MG_TRY(s->cloc.upload(cloc.data(), std::max<size_t>(nd, 1), st));
  MG_TRY(s->dom_sorted.upload(sorted.data(), std::max<size_t>(sorted.size(), 1), st));
  MG_TRY(s->cfac_off.upload(off.data(), off.size(), st));
  MG_TRY(s->cfac.reserve(std::max<uint64_t>(off[s->ncdom], 4)));
  MG_TRY(s->ec.reserve(std::max<uint64_t>(3ull * nd, 4)));
  MG_CUDA(cudaStreamSynchronize(st));
  return MGUSO_OK;
}

// ---------------------------------------------------------------------------------------
// Factorisation: one CTA per domain, FP64 in shared memory, in place in one m x ld buffer
// (ld = m + 1, so column walks are free of bank conflicts):
//   1. gather the dense block and add the reference's diagonal floor;
//   2. blocked right-looking Cholesky on the lower triangle over 32-column panels. The k-th
//      pivot is the k-th Schur complement diagonal, the value the reference's row-by-row
//      Cholesky tests against 1e-14 (linsolve.rs:88-92), so the same blocks fall back to the
//      diagonal;
//   3. W = L^-1, the diagonal blocks inverted per panel, the others by block forward
//      substitution, written transposed into the upper triangle.
// Stored: W in FP32 as swizzled tiles (layout above). The apply forms z = W^T (W r), so
// the FP32 preconditioner W~^T W~ is symmetric positive definite for any rounding of W.
// (An explicitly stored FP32 inverse is not: with stiff seams a domain block reaches a
// condition number near 1e7 and rounding the inverse to FP32 can make it indefinite.)
// ---------------------------------------------------------------------------------------
constexpr int FACTOR_THREADS = 256;

template <class TS>
__device__ __forceinline__ TS to_tile(double v) {
  return (TS)v;
}
template <>
__device__ __forceinline__ __half to_tile<__half>(double v) {
  return __float2half_rn((float)v);
}

// Largest |W_ij| over the domain's lower triangle (W_ij at A[j * ld + i], j <= i < m), or
// over diag when the factorisation failed; every thread gets it.
__device__ double factor_amax(const double* A, int ld, int m, const double* diag, bool failed) {
  __shared__ double s_w[FACTOR_THREADS / 32];
  const int tid = threadIdx.x, nt = blockDim.x;
  double mx = 0.0;
  if (failed) {
    for (int r = tid; r < m; r += nt) mx = fmax(mx, diag[r] > 1e-14 ? 1.0 / sqrt(diag[r]) : 1.0);
  } else {
    for (int e = tid; e < m * m; e += nt) {
      const int i = e / m, j = e - i * m;
      if (j <= i) mx = fmax(mx, fabs(A[j * ld + i]));
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) s_w[tid >> 5] = mx;
  __syncthreads();
  double r = 0.0;
  for (int q = 0; q < nt / 32; ++q) r = fmax(r, s_w[q]);
  __syncthreads();
  return r > 0.0 ? r : 1.0;
}

// acc[r][c] += sum over k in [k0, k1) of a(i0 + r, k) b(k, j0 + c): a 4 x 4 register tile of
// a small FP64 product in shared memory (a and b return 0 outside their structure)
__device__ __forceinline__ void mt4_zero(double (&acc)[4][4]) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
}
template <class FA, class FB>
__device__ __forceinline__ void mt4(double (&acc)[4][4], int i0, int j0, int k0, int k1, FA&& a, FB&& b) {
  for (int k = k0; k < k1; ++k) {
    double av[4], bv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) av[r] = a(i0 + r, k);
#pragma unroll
    for (int c = 0; c < 4; ++c) bv[c] = b(k, j0 + c);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
  }
}

// Steps 2-3 of the factorisation and the store, on the dense block A (m x m, leading
// dimension ld, FP64 shared memory, lower triangle filled) of one domain: the reference's
// diagonal floor, right-looking Cholesky with its pivot test (falling back to the floored
// diagonal), W = L^-1, and W written to `out` as tiles (FP16 tiles: W / scale with the
// scale in *scale_out). dinv and diag0 are m doubles of shared scratch each.
template <class TS>
__device__ void factor_dense_store(double* A, int ld, int m, double* dinv, double* diag0, TS* __restrict__ out,
                                   float* scale_out, uint32_t* status) {
  constexpr bool scaled = sizeof(TS) == 2;
  __shared__ double s_floor;
  __shared__ int s_fail;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) {
    double tr = 0.0;
    for (int k = 0; k < m; ++k) tr += A[k * ld + k];
    s_floor = 1e-6 * (tr / (double)m) + 1e-8;
    s_fail = 0;
  }
  __syncthreads();
  for (int k = tid; k < m; k += nt) {
    A[k * ld + k] += s_floor;
    diag0[k] = A[k * ld + k];
  }
  // the strict upper triangle receives W's off-diagonal entries (W_ij at A[j * ld + i], i > j)
  for (int e = tid; e < m * m; e += nt) {
    const int i = e / m, j = e - i * m;
    if (j > i) A[i * ld + j] = 0.0;
  }
  __syncthreads();
  // Blocked right-looking Cholesky A = L L^T over 32-column panels, L in the lower triangle:
  // per panel, warp 0 factors the diagonal block column by column (the k-th pivot is the
  // k-th Schur complement diagonal, tested against 1e-14 as the reference's row-by-row
  // Cholesky does) and inverts it (W_PP = L_PP^-1, one lane per column); then the rows below
  // become L_IP = A_IP W_PP^T and the trailing blocks lose L_IP L_JP^T, as 4 x 4 register
  // tiles per thread. About four barriers per panel instead of one per column.
  const int tx = tid & 31, ty = tid >> 5;
  const int T = (m + 31) >> 5;
  for (int P = 0; P < T; ++P) {
    const int c0 = 32 * P, nb = min(32, m - c0), r0 = c0 + nb, R = m - r0;
    if (ty == 0) {
      // the diagonal block in registers, lane i holding row i; column k of the factor is
      // broadcast by shuffles, so a step costs no shared-memory round trips
      double row[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) row[j] = (tx < nb && j <= tx) ? A[(c0 + tx) * ld + c0 + j] : 0.0;
      bool fail = false;
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        if (k < nb && !fail) {  // uniform
          const double p = __shfl_sync(0xffffffffu, row[k], k);
          if (!(p > 1e-14)) {  // every lane sees the same pivot
            fail = true;
          } else {
            const double il = rsqrt(p), lkk = p * il;  // 1 / L_kk and L_kk
            const double lik = tx > k ? row[k] * il : (tx == k ? lkk : 0.0);
            if (tx >= k) row[k] = lik;
            if (tx == k) dinv[c0 + k] = il;
#pragma unroll
            for (int j = k + 1; j < 32; ++j) {
              const double ljk = __shfl_sync(0xffffffffu, lik, j);
              if (tx >= j) row[j] = fma(-lik, ljk, row[j]);
            }
          }
        }
      }
      if (!fail) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (tx < nb && j <= tx) A[(c0 + tx) * ld + c0 + j] = row[j];
        __syncwarp();
        // W_PP = L_PP^-1, lane j holding column j: W_jj = 1 / L_jj and, for i > j,
        // W_ij = -(sum_{j <= q < i} L_iq W_qj) / L_ii, L's rows read as broadcasts
        double wcol[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          if (i < nb) {
            const double* li = A + (size_t)(c0 + i) * ld + c0;
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int q = 0; q < i; ++q) {
              const double t = q >= tx ? wcol[q] : 0.0;
              if (q & 1)
                a1 = fma(li[q], t, a1);
              else
                a0 = fma(li[q], t, a0);
            }
            const double di = dinv[c0 + i];
            wcol[i] = i == tx ? di : (i > tx ? -(a0 + a1) * di : 0.0);
          } else {
            wcol[i] = 0.0;
          }
        }
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (i > tx && i < nb) A[(c0 + tx) * ld + c0 + i] = wcol[i];
      }
      if (tx == 0) s_fail = fail ? 1 : 0;
    }
    __syncthreads();
    if (s_fail) break;  // uniform
    if (R > 0) {
      // panel: L_ij = sum_{c <= j} A_ic W_jc for the rows below (nb = 32 here)
      const int ntr = (R + 3) >> 2, items = ntr * 8;
      double acc[4][4];
      const int t = tid;
      const int ti = t >> 3, tj = t & 7;
      const int i0 = r0 + 4 * ti, j0 = 4 * tj;
      const bool mine = t < items;
      if (mine) {
        mt4_zero(acc);
        mt4(acc, i0, j0, 0, j0 + 4,
            [&](int i, int c) { return i < m ? A[i * ld + c0 + c] : 0.0; },
            [&](int c, int j) { return c == j ? dinv[c0 + j] : (c < j ? A[(c0 + c) * ld + c0 + j] : 0.0); });
      }
      __syncthreads();
      if (mine)
        for (int r = 0; r < 4; ++r)
          if (i0 + r < m)
            for (int c = 0; c < 4; ++c) A[(i0 + r) * ld + c0 + j0 + c] = acc[r][c];
      __syncthreads();
      // trailing update of the lower triangle: A_ij -= sum_c L_ic L_jc (i >= j >= r0)
      const int pairs = ntr * (ntr + 1) / 2;
      for (int u = tid; u < pairs; u += nt) {
        int a = (int)((sqrtf(8.f * (float)u + 1.f) - 1.f) * 0.5f);
        while ((a + 1) * (a + 2) / 2 <= u) ++a;
        while (a * (a + 1) / 2 > u) --a;
        const int b = u - a * (a + 1) / 2;  // tile row a >= tile column b
        const int ii = r0 + 4 * a, jj = r0 + 4 * b;
        double up[4][4];
        mt4_zero(up);
        mt4(up, ii, jj, 0, 32, [&](int i, int c) { return i < m ? A[i * ld + c0 + c] : 0.0; },
            [&](int c, int j) { return j < m ? A[j * ld + c0 + c] : 0.0; });
        for (int r = 0; r < 4; ++r)
          for (int c = 0; c < 4; ++c)
            if (ii + r < m && jj + c <= ii + r) A[(ii + r) * ld + jj + c] -= up[r][c];
      }
      __syncthreads();
    }
  }
  __syncthreads();
  if (!s_fail) {
    // off-diagonal blocks of W = L^-1, block row by block row:
    // W_IJ = -W_II S_IJ with S_IJ = sum_{J <= K < I} L_IK W_KJ; S is formed in W_IJ's place
    for (int I = 1; I < T; ++I) {
      const int i0 = 32 * I, ni = min(32, m - i0), ntr = (ni + 3) >> 2, items = I * ntr * 8;
      for (int u = tid; u < items; u += nt) {
        const int J = u / (ntr * 8), rem = u - J * ntr * 8, ti = rem >> 3, tj = rem & 7;
        const int j0 = 32 * J, ia = i0 + 4 * ti, ja = j0 + 4 * tj;
        double acc[4][4];
        mt4_zero(acc);
        mt4(acc, ia, ja, j0, i0, [&](int i, int k) { return i < m ? A[i * ld + k] : 0.0; },
            [&](int k, int j) { return k == j ? dinv[k] : (k > j ? A[j * ld + k] : 0.0); });
        for (int r = 0; r < 4; ++r)
          if (ia + r < m)
            for (int c = 0; c < 4; ++c) A[(ja + c) * ld + ia + r] = acc[r][c];
      }
      __syncthreads();
      double res[4][4];
      int ia = 0, ja = 0;
      const bool mine = tid < items;
      if (mine) {
        const int J = tid / (ntr * 8), rem = tid - J * ntr * 8, ti = rem >> 3, tj = rem & 7;
        ia = i0 + 4 * ti;
        ja = 32 * J + 4 * tj;
        mt4_zero(res);
        mt4(res, ia, ja, i0, min(m, ia + 4),
            [&](int i, int q) { return (i < m && q <= i) ? (q == i ? dinv[i] : A[q * ld + i]) : 0.0; },
            [&](int q, int j) { return A[j * ld + q]; });
      }
      __syncthreads();
      if (mine)
        for (int r = 0; r < 4; ++r)
          if (ia + r < m)
            for (int c = 0; c < 4; ++c) A[(ja + c) * ld + ia + r] = -res[r][c];
      __syncthreads();
    }
  }
  __syncthreads();
  const int nfl = T * (T + 1) / 2 * TILE_FLOATS;
  if (s_fail) {
    // reference fallback: L = diag(sqrt(ad_pp)) (1 where ad_pp <= 1e-14), i.e.
    // W = diag(1 / sqrt(ad_pp))
    const double sc = scaled ? factor_amax(A, ld, m, diag0, true) : 1.0;
    if (scaled && tid == 0) *scale_out = (float)sc;
    for (int e = tid; e < nfl; e += nt) out[e] = to_tile<TS>(0.0);
    __syncthreads();
    for (int r = tid; r < m; r += nt) {
      double a = diag0[r];
      const int I = r >> 5, lr = r & 31;
      out[tile_index(I, I) * TILE_FLOATS + tile_off<TS>(lr, lr)] = to_tile<TS>((a > 1e-14 ? 1.0 / sqrt(a) : 1.0) / sc);
    }
    if (tid == 0) atomicOr(status, 1u << 8);
    return;
  }
  for (int i = tid; i < m; i += nt) A[i * ld + i] = dinv[i];  // W's diagonal joins its upper-triangle copy
  __syncthreads();
  const double inv_sc = scaled ? 1.0 / factor_amax(A, ld, m, diag0, false) : 1.0;
  if (scaled && tid == 0) *scale_out = (float)(1.0 / inv_sc);
  // tiles in storage order; e walks each tile's swizzled offsets so the stores coalesce
  for (int e = tid; e < nfl; e += nt) {
    const int t = e / TILE_FLOATS, o = e - t * TILE_FLOATS;
    const int I = t >= 3 ? 2 : (t >= 1 ? 1 : 0), J = t - I * (I + 1) / 2;
    int r, c;
    tile_rc<TS>(o, r, c);
    const int gi = 32 * I + r, gj = 32 * J + c;
    out[e] = to_tile<TS>((gi < m && gj <= gi) ? A[gj * ld + gi] * inv_sc : 0.0);
  }
}

// One vertex as its own domain (m = 3): the reference's floor 1e-6 (tr / 3) + 1e-8 on the
// diagonal, the row-by-row Cholesky with its pivot test (linsolve.rs:80-99; a failed pivot
// falls back to L = diag(sqrt(a_pp)), 1 where a_pp <= 1e-14), and W = L^-1 stored as its
// lower triangle (w00 w10 w11 w20 w21 w22).
__device__ void vertex_factor(double* a, float* __restrict__ w6, uint32_t* status) {
  const double fl = 1e-6 * ((a[0] + a[4] + a[8]) / 3.0) + 1e-8;
  a[0] += fl;
  a[4] += fl;
  a[8] += fl;
  double l[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  bool ok = true;
  for (int i = 0; i < 3 && ok; ++i)
    for (int j = 0; j <= i; ++j) {
      double sum = a[3 * i + j];
      for (int k = 0; k < j; ++k) sum -= l[3 * i + k] * l[3 * j + k];
      if (i == j) {
        if (!(sum > 1e-14)) {
          ok = false;
          break;
        }
        l[3 * i + i] = sqrt(sum);
      } else {
        l[3 * i + j] = sum / l[3 * j + j];
      }
    }
  if (!ok) {
    for (int e = 0; e < 9; ++e) l[e] = 0.0;
    for (int p = 0; p < 3; ++p) l[4 * p] = a[4 * p] > 1e-14 ? sqrt(a[4 * p]) : 1.0;
    atomicOr(status, 1u << 8);
  }
  const double w00 = 1.0 / l[0], w11 = 1.0 / l[4], w22 = 1.0 / l[8];
  const double w10 = -l[3] * w00 * w11;
  const double w21 = -l[7] * w11 * w22;
  const double w20 = -(l[6] * w00 + l[7] * w10) * w22;
  w6[0] = (float)w00;
  w6[1] = (float)w10;
  w6[2] = (float)w11;
  w6[3] = (float)w20;
  w6[4] = (float)w21;
  w6[5] = (float)w22;
}

template <class TS>
__global__ void __launch_bounds__(FACTOR_THREADS, 2) k_schwarz_factor(
    const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col, const float* __restrict__ val,
    const uint32_t* __restrict__ dom_start, const uint32_t* __restrict__ dom_verts,
    const uint32_t* __restrict__ dom_of, const uint32_t* __restrict__ loc, const uint64_t* __restrict__ fac_off,
    TS* __restrict__ fac, float* __restrict__ fac_scale, uint32_t* status, const uint32_t* __restrict__ c_rp,
    const uint32_t* __restrict__ c_col, const float* __restrict__ c_val, const uint8_t* __restrict__ dom_diag,
    float* __restrict__ vfac, const uint8_t* __restrict__ dom_inst, uint32_t active) {
  // FP16 tiles hold W / scale (scale: the domain's largest |W|); FP32 tiles hold W
  extern __shared__ __align__(16) double sA[];
  const uint32_t d = blockIdx.x;
  if (!((active >> dom_inst[d]) & 1u)) return;  // an instance the batch no longer iterates
  const uint32_t vs = dom_start[d], nvd = dom_start[d + 1] - vs;
  if (dom_diag[d]) {
    for (uint32_t p = threadIdx.x; p < nvd; p += blockDim.x) {
      const uint32_t v = dom_verts[vs + p];
      double A9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (uint32_t k = row_ptr[v]; k < row_ptr[v + 1]; ++k)
        if (col[k] == v)
          for (int e = 0; e < 9; ++e) A9[e] = (double)val[9 * (size_t)k + e];
      vertex_factor(A9, vfac + 6 * (size_t)v, status);
    }
    return;
  }
  const int m = 3 * (int)nvd;
  const int ld = m + 1;
  double* A = sA;
  double* dinv = sA + (size_t)m * ld;  // 1 / L_kk
  double* diag0 = dinv + m;           // floored diagonal (fallback)
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < m * ld; i += nt) A[i] = 0.0;
  __syncthreads();
  const int lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  for (uint32_t p = w; p < nvd; p += nw) {
    uint32_t v = dom_verts[vs + p];
    for (uint32_t k = row_ptr[v] + lane; k < row_ptr[v + 1]; k += 32) {
      uint32_t c = col[k];
      if (dom_of[c] != d) continue;
      uint32_t q = loc[c];
      const float* b = val + 9 * (size_t)k;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) A[(3 * p + i) * ld + 3 * q + j] = (double)b[3 * i + j];
    }
  }
  __syncthreads();
  // contact blocks outside the fixed pattern (distinct (row, col) from the loop above)
  if (c_rp) {
    for (uint32_t p = w; p < nvd; p += nw) {
      uint32_t v = dom_verts[vs + p];
      for (uint32_t k = c_rp[v] + lane; k < c_rp[v + 1]; k += 32) {
        uint32_t c = c_col[k];
        if (dom_of[c] != d) continue;
        uint32_t q = loc[c];
        const float* b = c_val + 9 * (size_t)k;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) A[(3 * p + i) * ld + 3 * q + j] = (double)b[3 * i + j];
      }
    }
    __syncthreads();
  }
  factor_dense_store<TS>(A, ld, m, dinv, diag0, fac + fac_off[d], fac_scale ? fac_scale + d : nullptr, status);
}

// Coarse factorisation of the two-level form, one CTA per coarse domain: thread t owns
// row t = 3a + r of the domain's dense Galerkin block (coarse node a, component r) and adds,
// for every vertex i of node a in ascending order and every block (i, j) of the pattern and
// of the contact matrix in column order whose column vertex lies in this coarse domain, the
// block's row r. The sums run in FP32, entry by entry in the order of the fine values, as
// the reference's coarse_matrix does (linsolve.rs:618-630); the block is then factored and
// stored like a level-0 domain.
__global__ void __launch_bounds__(FACTOR_THREADS) k_coarse_factor(
    const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col, const float* __restrict__ val,
    const uint32_t* __restrict__ c_rp, const uint32_t* __restrict__ c_col, const float* __restrict__ c_val,
    const uint32_t* __restrict__ dom_start, const uint32_t* __restrict__ dom_sorted,
    const uint32_t* __restrict__ dom_of, const uint32_t* __restrict__ cdom_start,
    const uint32_t* __restrict__ cdom_nodes, const uint32_t* __restrict__ cdom_of, const uint32_t* __restrict__ cloc,
    const uint64_t* __restrict__ cfac_off, float* __restrict__ cfac, uint32_t* status) {
  extern __shared__ __align__(16) double sA[];
  const uint32_t d1 = blockIdx.x;
  const uint32_t n0 = cdom_start[d1], mn = cdom_start[d1 + 1] - n0;
  const int m = 3 * (int)mn, ld = m + 1;
  double* A = sA;
  double* dinv = sA + (size_t)m * ld;
  double* diag0 = dinv + m;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < m * ld; i += nt) A[i] = 0.0;
  __syncthreads();
  for (int t = tid; t < m; t += nt) {
    const int a = t / 3, r = t - 3 * a;
    const uint32_t g = cdom_nodes[n0 + a];
    double* row = A + (size_t)t * ld;
    for (uint32_t p = dom_start[g]; p < dom_start[g + 1]; ++p) {
      const uint32_t i = dom_sorted[p];
      uint32_t k1 = row_ptr[i];
      const uint32_t e1 = row_ptr[i + 1];
      uint32_t k2 = c_rp ? c_rp[i] : 0;
      const uint32_t e2 = c_rp ? c_rp[i + 1] : 0;
      while (k1 < e1 || k2 < e2) {
        const bool from_c = k1 >= e1 || (k2 < e2 && c_col[k2] < col[k1]);
        const uint32_t j = from_c ? c_col[k2] : col[k1];
        const float* b = from_c ? c_val + 9 * (size_t)k2++ : val + 9 * (size_t)k1++;
        const uint32_t h = dom_of[j];
        if (cdom_of[h] != d1) continue;
        const int q = 3 * (int)cloc[h];
#pragma unroll
        for (int c = 0; c < 3; ++c) row[q + c] = (double)((float)row[q + c] + b[3 * r + c]);
      }
    }
  }
  __syncthreads();
  factor_dense_store<float>(A, ld, m, dinv, diag0, cfac + cfac_off[d1], nullptr, status);
}

int schwarz_factor(mguso_schwarz* s, cudaStream_t st) {
  return schwarz_factor_with(s, nullptr, nullptr, nullptr, st);
}

int schwarz_factor_with(mguso_schwarz* s, const uint32_t* c_rp, const uint32_t* c_col, const float* c_val,
                        cudaStream_t st) {
  if (s->ndom == 0) return MGUSO_OK;
  mguso_bsr* a = s->a;
  size_t smem = sizeof(double) * ((size_t)s->max_m * (s->max_m + 1) + 2 * (size_t)s->max_m);
  if (s->half)
    k_schwarz_factor<__half><<<s->ndom, FACTOR_THREADS, smem, st>>>(
        a->row_ptr.p, a->col.p, a->val.p, s->dom_start.p, s->dom_verts.p, s->dom_of.p, s->loc.p, s->fac_off.p,
        s->fac_h.p, s->fac_scale.p, s->status.p, c_col ? c_rp : nullptr, c_col, c_val, s->dom_diag.p, s->vfac.p,
        s->dom_inst.p, s->active);
  else
    k_schwarz_factor<float><<<s->ndom, FACTOR_THREADS, smem, st>>>(
        a->row_ptr.p, a->col.p, a->val.p, s->dom_start.p, s->dom_verts.p, s->dom_of.p, s->loc.p, s->fac_off.p,
        s->fac.p, nullptr, s->status.p, c_col ? c_rp : nullptr, c_col, c_val, s->dom_diag.p, s->vfac.p,
        s->dom_inst.p, s->active);
  MG_CUDA(cudaGetLastError());
  if (s->levels == 2 && s->ncdom) {
    size_t smem1 = sizeof(double) * ((size_t)s->max_m1 * (s->max_m1 + 1) + 2 * (size_t)s->max_m1);
    k_coarse_factor<<<s->ncdom, FACTOR_THREADS, smem1, st>>>(
        a->row_ptr.p, a->col.p, a->val.p, c_col ? c_rp : nullptr, c_col, c_val, s->dom_start.p, s->dom_sorted.p,
        s->dom_of.p, s->cdom_start.p, s->cdom_nodes.p, s->cdom_of.p, s->cloc.p, s->cfac_off.p, s->cfac.p,
        s->status.p);
    MG_CUDA(cudaGetLastError());
  }
  return MGUSO_OK;
}

// ---------------------------------------------------------------------------------------
// Apply: one warp per domain (grid-stride over domains). The warp bulk-copies its domain's
// W tiles into its shared slice, gathers r, then
//   pass 1: y = W r    lane = row within a row tile, loop over columns c;
//   pass 2: z = W^T y  lane = column within a column tile, loop over rows r.
// The FP32 tile layout (c*32 + (r ^ c)) makes both passes free of bank conflicts. Every
// lane carries one accumulator per tile row/column (<= 3), so there are no long serial
// chains. Acc = double (mixed precision) accumulates in FP64.
// ---------------------------------------------------------------------------------------
constexpr int APPLY_WARPS = 4;

template <int WARPS, class Acc, class TS>
__global__ void __launch_bounds__(32 * WARPS) k_schwarz_apply(
    const uint32_t* __restrict__ dom_start, const uint32_t* __restrict__ dom_verts,
    const uint64_t* __restrict__ fac_off, const TS* __restrict__ fac, const float* __restrict__ fac_scale,
    const float* __restrict__ r, float* __restrict__ z, uint32_t ndom, uint32_t* status, DotSink dot, int with_dot,
    const uint8_t* __restrict__ dom_diag, const float* __restrict__ vfac) {
  extern __shared__ __align__(128) unsigned char smem[];
  if (with_dot && dot.sc->done) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t* bar = (uint64_t*)(smem + 16 * w);
  TS* buf = (TS*)(smem + 128 + (size_t)w * apply_slice_bytes<TS>());
  float* rd = (float*)(buf + 6 * TILE_FLOATS);
  Acc* yd = (Acc*)(rd + 96);
  Acc acc = 0;
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
  uint32_t phase = 0;
  for (uint32_t d = blockIdx.x * WARPS + w; d < ndom; d += gridDim.x * WARPS) {
    const uint32_t vs = dom_start[d], nvd = dom_start[d + 1] - vs;
    const int m = 3 * (int)nvd;
    const uint64_t off = fac_off[d];
    const uint32_t bytes = (uint32_t)((fac_off[d + 1] - off) * sizeof(TS));
    const bool diag = dom_diag[d] != 0;
    if (lane == 0 && !diag) {
      fence_proxy_async();
      mbar_arrive_expect_tx(bar, bytes);
      bulk_g2s(buf, fac + off, bytes, bar);
    }
    for (int i = lane; i < 96; i += 32) {
      float v = 0.f;
      if (i < m) v = r[3 * dom_verts[vs + i / 3] + i % 3];
      rd[i] = v;
    }
    __syncwarp();
    if (diag) {
      if (lane < (int)nvd) {
        const uint32_t v = dom_verts[vs + lane];
        Acc zz[3];
        vertex_apply<Acc>(vfac + 6 * (size_t)v, rd + 3 * lane, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float zi = (float)zz[c];
          z[3 * v + c] = zi;
          acc += (Acc)rd[3 * lane + c] * (Acc)zi;
        }
      }
      __syncwarp();
      continue;
    }
    if (!mbar_wait(bar, phase)) {
      if (lane == 0) atomicOr(status, ST_WAIT_TIMEOUT);
      mbar_wait(bar, phase);  // the copy may still land: bounded second wait, then stop
      break;
    }
    phase ^= 1;
    Acc zz[3];
    const int T = (m + 31) >> 5;
    if (T == 3)
      tiles_apply<3, Acc, TS>(buf, rd, yd, zz, lane);
    else if (T == 2)
      tiles_apply<2, Acc, TS>(buf, rd, yd, zz, lane);
    else
      tiles_apply<1, Acc, TS>(buf, rd, yd, zz, lane);
    const Acc sc = fac_scale ? (Acc)fac_scale[d] : (Acc)1;
#pragma unroll
    for (int J = 0; J < 3; ++J) {
      const int i = 32 * J + lane;
      if (i < m) {
        const float zi = (float)(zz[J] * sc * sc);
        z[3 * dom_verts[vs + i / 3] + i % 3] = zi;
        acc += (Acc)rd[i] * (Acc)zi;
      }
    }
    __syncwarp();  // every lane is done with buf before the next copy overwrites it
  }
  if (with_dot == 1) grid_dot_commit<Acc>(dot, acc);
}

// Coarse level of the two-level apply, one warp per coarse domain: restriction
// rc = sum of r over each coarse node's vertices (linsolve.rs:648-655), the domain's
// z1 = W1^T (W1 rc) from its FP32 tiles, written as the coarse correction ec.
__global__ void __launch_bounds__(32) k_coarse_apply(
    const uint32_t* __restrict__ cdom_start, const uint32_t* __restrict__ cdom_nodes,
    const uint32_t* __restrict__ dom_start, const uint32_t* __restrict__ dom_verts,
    const uint64_t* __restrict__ cfac_off, const float* __restrict__ cfac, const float* __restrict__ r,
    float* __restrict__ ec, uint32_t ncdom, const PcgScalars* done) {
  __shared__ __align__(16) float buf[6 * TILE_FLOATS];
  __shared__ float rd[96];
  __shared__ double yd[96];
  if (done && done->done) return;
  const int lane = threadIdx.x;
  for (uint32_t d1 = blockIdx.x; d1 < ncdom; d1 += gridDim.x) {
    const uint32_t n0 = cdom_start[d1], mn = cdom_start[d1 + 1] - n0;
    const int m = 3 * (int)mn;
    const uint64_t off = cfac_off[d1];
    const int nfl = (int)(cfac_off[d1 + 1] - off);
    for (int e = lane; e < nfl; e += 32) buf[e] = cfac[off + e];
    for (uint32_t a = 0; a < mn; ++a) {
      const uint32_t g = cdom_nodes[n0 + a];
      double s0 = 0, s1 = 0, s2 = 0;
      for (uint32_t p = dom_start[g] + lane; p < dom_start[g + 1]; p += 32) {
        const uint32_t v = dom_verts[p];
        s0 += (double)r[3 * v];
        s1 += (double)r[3 * v + 1];
        s2 += (double)r[3 * v + 2];
      }
      s0 = warp_sum(s0);
      s1 = warp_sum(s1);
      s2 = warp_sum(s2);
      if (lane == 0) {
        rd[3 * a] = (float)s0;
        rd[3 * a + 1] = (float)s1;
        rd[3 * a + 2] = (float)s2;
      }
    }
    for (int i = m + lane; i < 96; i += 32) rd[i] = 0.f;
    __syncwarp();
    double zz[3];
    const int T = (m + 31) >> 5;
    if (T == 3)
      tiles_apply<3, double, float>(buf, rd, yd, zz, lane);
    else if (T == 2)
      tiles_apply<2, double, float>(buf, rd, yd, zz, lane);
    else
      tiles_apply<1, double, float>(buf, rd, yd, zz, lane);
#pragma unroll
    for (int J = 0; J < 3; ++J) {
      const int i = 32 * J + lane;
      if (i < m) ec[3 * cdom_nodes[n0 + i / 3] + i % 3] = (float)zz[J];
    }
    __syncwarp();
  }
}

// z += w * ec[coarse node of the vertex] (the weighted prolongation, linsolve.rs:657-665),
// with the fused r.z of the PCG.
template <class Acc>
__global__ void k_prolong(const float* __restrict__ r, float* __restrict__ z, const float* __restrict__ ec,
                          const uint32_t* __restrict__ dom_of, uint32_t nb, float w, DotSink d, int with_dot) {
  if (with_dot && d.sc->done) return;
  Acc acc = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nb; v += gridDim.x * blockDim.x) {
    const uint32_t g = dom_of[v];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float zc = fmaf(w, ec[3 * g + c], z[3 * v + c]);
      z[3 * v + c] = zc;
      acc += (Acc)r[3 * v + c] * (Acc)zc;
    }
  }
  if (with_dot) grid_dot_commit<Acc>(d, acc);
}

// Shared-memory opt-in for the largest domain (32 vertices, m = 96), set once outside any
// stream capture.
int schwarz_configure() {
  static bool done = false;
  if (done) return MGUSO_OK;
  size_t fsm = sizeof(double) * (96 * 97 + 2 * 96);
  MG_CUDA(cudaFuncSetAttribute(k_schwarz_factor<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
  MG_CUDA(cudaFuncSetAttribute(k_schwarz_factor<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
  MG_CUDA(cudaFuncSetAttribute(k_coarse_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
  const int asm32 = (int)(128 + (size_t)APPLY_WARPS * apply_slice_bytes<float>());
  const int asm16 = (int)(128 + (size_t)APPLY_WARPS * apply_slice_bytes<__half>());
  MG_CUDA(cudaFuncSetAttribute(k_schwarz_apply<APPLY_WARPS, double, float>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, asm32));
  MG_CUDA(cudaFuncSetAttribute(k_schwarz_apply<APPLY_WARPS, float, float>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, asm32));
  MG_CUDA(cudaFuncSetAttribute(k_schwarz_apply<APPLY_WARPS, double, __half>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, asm16));
  MG_CUDA(cudaFuncSetAttribute(k_schwarz_apply<APPLY_WARPS, float, __half>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, asm16));
  done = true;
  return MGUSO_OK;
}

int schwarz_apply(mguso_schwarz* s, const float* r, float* z, cudaStream_t st, const DotSink* dot) {
  DotSink d{};
  // two levels: the level-0 apply skips after convergence but leaves the r.z to the
  // prolongation, which completes z
  int with_dot = dot ? (s->levels == 2 ? 2 : 1) : 0;
  if (dot) d = *dot;
  bool mixed = dot && dot->mixed;
  if (s->max_m > 96) {
    set_error("Schwarz domain larger than 32 vertices");
    return MGUSO_ERR_UNSUPPORTED;
  }
  const bool h = s->half;
  size_t smem = 128 + (size_t)APPLY_WARPS * (h ? apply_slice_bytes<__half>() : apply_slice_bytes<float>());
  // resident CTAs per SM as shared memory allows (2 with FP32 tiles, 4 with FP16), grid-stride
  uint32_t grid = std::min<uint32_t>(ceil_div(s->ndom, APPLY_WARPS), (h ? 4u : 2u) * (uint32_t)s->a->ctx->sm_count);
  void* fn = h ? (mixed ? (void*)k_schwarz_apply<APPLY_WARPS, double, __half>
                        : (void*)k_schwarz_apply<APPLY_WARPS, float, __half>)
               : (mixed ? (void*)k_schwarz_apply<APPLY_WARPS, double, float>
                        : (void*)k_schwarz_apply<APPLY_WARPS, float, float>);
  const uint32_t* a0 = s->dom_start.p;
  const uint32_t* a1 = s->dom_verts.p;
  const uint64_t* a2 = s->fac_off.p;
  const void* a3 = h ? (const void*)s->fac_h.p : (const void*)s->fac.p;
  const float* a4 = h ? s->fac_scale.p : nullptr;
  uint32_t nd = s->ndom;
  uint32_t* stp = s->status.p;
  const uint8_t* a5 = s->dom_diag.p;
  const float* a6 = s->vfac.p;
  void* args[] = {(void*)&a0, (void*)&a1, (void*)&a2, (void*)&a3, (void*)&a4, (void*)&r, (void*)&z,
                  (void*)&nd, (void*)&stp, (void*)&d, (void*)&with_dot, (void*)&a5, (void*)&a6};
  if (grid == 0) return MGUSO_OK;
  MG_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(32 * APPLY_WARPS), args, smem, st));
  if (s->levels != 2 || s->ncdom == 0) return MGUSO_OK;
  const uint32_t cgrid = std::min<uint32_t>(s->ncdom, 16u * (uint32_t)s->a->ctx->sm_count);
  k_coarse_apply<<<cgrid, 32, 0, st>>>(s->cdom_start.p, s->cdom_nodes.p, s->dom_start.p, s->dom_verts.p,
                                       s->cfac_off.p, s->cfac.p, r, s->ec.p, s->ncdom, dot ? dot->sc : nullptr);
  const uint32_t nb = s->a->nb;
  const uint32_t pgrid = std::max<uint32_t>(1, std::min<uint32_t>(ceil_div(nb, 256), 8u * (uint32_t)s->a->ctx->sm_count));
  const int wd = dot ? 1 : 0;
  if (mixed)
    k_prolong<double><<<pgrid, 256, 0, st>>>(r, z, s->ec.p, s->dom_of.p, nb, s->weight, d, wd);
  else
    k_prolong<float><<<pgrid, 256, 0, st>>>(r, z, s->ec.p, s->dom_of.p, nb, s->weight, d, wd);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// ---------------------------------------------------------------------------------------
// Block Jacobi (linsolve.rs:294-315): per-vertex 3x3 inverse in f64, stored as 9 floats;
// a singular block (|det| < 1e-20) falls back to 1/diagonal (1 where the diagonal is 0).
// ---------------------------------------------------------------------------------------
__global__ void k_bj_factor(const uint32_t* __restrict__ row_ptr, const uint32_t* __restrict__ col,
                            const float* __restrict__ val, uint32_t nb, float* __restrict__ inv) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nb) return;
  double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t k = row_ptr[v]; k < row_ptr[v + 1]; ++k)
    if (col[k] == v)
      for (int e = 0; e < 9; ++e) m[e] = (double)val[9 * (size_t)k + e];
  double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
               m[2] * (m[3] * m[7] - m[4] * m[6]);
  double o[9];
  if (fabs(det) < 1e-20) {
    for (int e = 0; e < 9; ++e) o[e] = 0.0;
    for (int i = 0; i < 3; ++i) o[4 * i] = m[4 * i] != 0.0 ? 1.0 / m[4 * i] : 1.0;
  } else {
    double id = 1.0 / det;
    o[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    o[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    o[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    o[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    o[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    o[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    o[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    o[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    o[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  }
  for (int e = 0; e < 9; ++e) inv[9 * (size_t)v + e] = (float)o[e];
}

int blockjacobi_factor(mguso_bsr* a, float* inv, cudaStream_t s) {
  if (a->nb == 0) return MGUSO_OK;
  k_bj_factor<<<ceil_div(a->nb, 128), 128, 0, s>>>(a->row_ptr.p, a->col.p, a->val.p, a->nb, inv);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

}  // namespace mg
