// LBVH broad phase on sm_100a: Morton codes (30-bit u32 / 63-bit u64), a onesweep LSD
// radix sort of (key, payload) pairs, the Karras tree, a single-pass atomic-climb refit,
// and a traversal that emits every (query, triangle) pair whose boxes overlap.
//
// Reference pipeline (engine-gpu/src/{morton,radix,karras,bvh_aabb,bvh_traverse}.rs and
// the shaders of the same names): 30-bit codes only, an 8-bit LSD radix sort limited to
// 65 536 keys with a serial per-block scatter, level-by-level AABB passes, and one stack
// per thread. The results this file must reproduce bit-for-bit are the CPU oracles
// morton_codes_cpu (morton.rs:50-63; centroid = (a+b+c)/3, no FMA contraction), the
// stable sort permutation, karras_tree_cpu (karras.rs:24-88) and propagate_aabb_cpu
// (bvh_aabb.rs:28-56); the pair SET is `all(qlo <= bhi) && all(blo <= qhi)` against leaf
// boxes (bvh_traverse.wgsl:64-92).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "lbvh.cuh"

namespace mg {

// ---------------------------------------------------------------------------------------
// Morton codes
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b ^ 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u ^ 0x80000000u) : ~u);
}

__device__ __forceinline__ float centroid_c(const float* __restrict__ pos, const uint32_t* t, int c) {
  float a = pos[3 * t[0] + c], b = pos[3 * t[1] + c], d = pos[3 * t[2] + c];
  return __fdiv_rn(__fadd_rn(__fadd_rn(a, b), d), 3.0f);
}

__global__ void k_centroid_bounds(const float* __restrict__ pos, const uint32_t* __restrict__ tris, uint32_t nt,
                                  uint32_t* __restrict__ ord /*6: lo.xyz as ord (min), hi.xyz (max)*/) {
  uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0, 0, 0};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    uint32_t tv[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
    for (int c = 0; c < 3; ++c) {
      uint32_t o = f2ord(centroid_c(pos, tv, c));
      lo[c] = min(lo[c], o);
      hi[c] = max(hi[c], o);
    }
  }
  for (int c = 0; c < 3; ++c) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = min(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = max(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int c = 0; c < 3; ++c) {
      atomicMin(&ord[c], lo[c]);
      atomicMax(&ord[3 + c], hi[c]);
    }
  }
}

// params: lo.xyz, inv.xyz (centroid_bounds, morton.rs:30-47)
__global__ void k_bounds_finish(const uint32_t* __restrict__ ord, float* __restrict__ params) {
  if (threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      float lo = ord2f(ord[c]), hi = ord2f(ord[3 + c]);
      float ext = __fsub_rn(hi, lo);
      params[c] = lo;
      params[3 + c] = ext > 0.0f ? __fdiv_rn(1.0f, ext) : 0.0f;
    }
  }
}

__device__ __forceinline__ float clampf_nan(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
  uint32_t x = v & 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}
__device__ __forceinline__ uint64_t expand21(uint64_t v) {
  uint64_t x = v & 0x1fffffull;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

template <class K>
__device__ __forceinline__ K morton_of(float nx, float ny, float nz);
template <>
__device__ __forceinline__ uint32_t morton_of<uint32_t>(float nx, float ny, float nz) {
  auto q = [](float v) {
    return __float2uint_rz(clampf_nan(__fmul_rn(clampf_nan(v, 0.0f, 1.0f), 1023.0f), 0.0f, 1023.0f));
  };
  return expand10(q(nx)) * 4u + expand10(q(ny)) * 2u + expand10(q(nz));
}
template <>
__device__ __forceinline__ uint64_t morton_of<uint64_t>(float nx, float ny, float nz) {
  auto q = [](float v) {
    return (uint64_t)__float2uint_rz(clampf_nan(__fmul_rn(clampf_nan(v, 0.0f, 1.0f), 2097151.0f), 0.0f, 2097151.0f));
  };
  return expand21(q(nx)) * 4ull + expand21(q(ny)) * 2ull + expand21(q(nz));
}

template <class K>
__global__ void k_morton(const float* __restrict__ pos, const uint32_t* __restrict__ tris, uint32_t nt,
                         const float* __restrict__ params, K* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  uint32_t tv[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  float n[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) n[c] = __fmul_rn(__fsub_rn(centroid_c(pos, tv, c), params[c]), params[3 + c]);
  keys[t] = morton_of<K>(n[0], n[1], n[2]);
  vals[t] = t;
}

// Morton codes of points (query ordering): same normalisation with the given params.
__global__ void k_morton_points(const float* __restrict__ pts, uint32_t np, const float* __restrict__ params,
                                uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float n[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) n[c] = __fmul_rn(__fsub_rn(pts[3 * i + c], params[c]), params[3 + c]);
  keys[i] = morton_of<uint32_t>(n[0], n[1], n[2]);
  vals[i] = i;
}

// ---------------------------------------------------------------------------------------
// Onesweep radix sort (stable LSD, 8-bit digits, decoupled look-back across tiles)
// ---------------------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 8;
constexpr uint32_t RS_TILE = RS_THREADS * RS_ITEMS;  // 2048 keys per tile
constexpr uint32_t FLAG_AGG = 1u << 30, FLAG_PRE = 2u << 30, VAL_MASK = (1u << 30) - 1;

template <class K>
__global__ void k_rs_hist(const K* __restrict__ keys, uint32_t n, int passes, uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[8 * 256];
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    K k = keys[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&sh[p * 256 + (uint32_t)((k >> (8 * p)) & 0xff)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// exclusive scan of each pass's 256 counts (one CTA of 256 threads per pass)
__global__ void k_rs_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ ofs) {
  __shared__ uint32_t s[256];
  int p = blockIdx.x, d = threadIdx.x;
  uint32_t v = hist[p * 256 + d];
  s[d] = v;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    uint32_t t = d >= o ? s[d - o] : 0;
    __syncthreads();
    s[d] += t;
    __syncthreads();
  }
  ofs[p * 256 + d] = s[d] - v;
}

template <class K>
__global__ void __launch_bounds__(RS_THREADS) k_onesweep(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                         K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                         uint32_t n, int shift, const uint32_t* __restrict__ gofs,
                                                         uint32_t* status, uint32_t* tile_counter, uint32_t* err,
                                                         const uint32_t* __restrict__ phist) {
  // phist (the pass's digit histogram, or null): when every key has the same digit the pass
  // keeps the order, and each CTA only copies its tile (the same decision in every CTA, so
  // no look-back is started); the host then never reads the histogram back
  if (phist && phist[(uint32_t)((kin[0] >> shift) & 0xff)] == n) {
    const uint32_t b0 = blockIdx.x * RS_TILE, b1 = min(b0 + RS_TILE, n);
    for (uint32_t j = b0 + threadIdx.x; j < b1; j += RS_THREADS) {
      kout[j] = kin[j];
      vout[j] = vin[j];
    }
    return;
  }
  __shared__ uint32_t whist[RS_WARPS][256];
  __shared__ uint32_t tile_excl[256], g_pref[256];
  __shared__ K skeys[RS_TILE];
  __shared__ uint32_t svals[RS_TILE];
  __shared__ uint32_t s_tile;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (int d = lane; d < 256; d += 32) whist[w][d] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t base = tile * RS_TILE;
  const uint32_t tile_n = min(RS_TILE, n - base);
  K key[RS_ITEMS];
  uint32_t val[RS_ITEMS], rank[RS_ITEMS];
  const uint32_t wbase = base + (uint32_t)w * RS_ITEMS * 32;
#pragma unroll
  for (int i = 0; i < RS_ITEMS; ++i) {
    uint32_t idx = wbase + i * 32 + lane;
    bool valid = idx < n;
    key[i] = valid ? kin[idx] : (K)0;
    val[i] = valid ? vin[idx] : 0u;
    uint32_t d = valid ? (uint32_t)((key[i] >> shift) & 0xff) : 0x100u + lane;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    int leader = __ffs(peers) - 1;
    uint32_t before = __popc(peers & ((1u << lane) - 1u));
    uint32_t old = 0;
    if (valid && lane == leader) {
      old = whist[w][d];
      whist[w][d] = old + __popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader);
    rank[i] = old + before;
    __syncwarp();
  }
  __syncthreads();
  // per digit: offsets of each warp, tile count, look-back for the global prefix
  {
    const int d = tid;
    uint32_t run = 0;
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      uint32_t c = whist[ww][d];
      whist[ww][d] = run;
      run += c;
    }
    volatile uint32_t* st = status;
    st[(size_t)tile * 256 + d] = FLAG_AGG | run;
    uint32_t excl = 0;
    int64_t j = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (j >= 0) {
      uint32_t v = st[(size_t)j * 256 + d];
      uint32_t flag = v & ~VAL_MASK;
      if (flag == 0) {
        if (++spins > (1u << 26)) {
          atomicOr(err, ST_WAIT_TIMEOUT);
          break;
        }
        continue;
      }
      excl += v & VAL_MASK;
      if (flag == FLAG_PRE) break;
      --j;
    }
    __threadfence();
    st[(size_t)tile * 256 + d] = FLAG_PRE | (excl + run);
    g_pref[d] = gofs[d] + excl;
    tile_excl[d] = run;  // scanned below
  }
  __syncthreads();
  // exclusive scan of the tile's digit counts (256 entries, one per thread)
  {
    const int d = tid;
    uint32_t v = tile_excl[d];
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    __shared__ uint32_t wsum[RS_WARPS];
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    uint32_t wofs = 0;
    for (int ww = 0; ww < w; ++ww) wofs += wsum[ww];
    __syncthreads();
    tile_excl[d] = wofs + incl - v;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < RS_ITEMS; ++i) {
    uint32_t idx = wbase + i * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)((key[i] >> shift) & 0xff);
      uint32_t p = tile_excl[d] + whist[w][d] + rank[i];
      skeys[p] = key[i];
      svals[p] = val[i];
    }
  }
  __syncthreads();
  for (uint32_t j = tid; j < tile_n; j += RS_THREADS) {
    K k = skeys[j];
    uint32_t d = (uint32_t)((k >> shift) & 0xff);
    uint32_t o = g_pref[d] + (j - tile_excl[d]);
    kout[o] = k;
    vout[o] = svals[j];
  }
}

// ---------------------------------------------------------------------------------------
// Karras tree (karras.rs:24-88), with parent links for the refit
// ---------------------------------------------------------------------------------------
template <class K>
__device__ __forceinline__ int kdelta(const K* __restrict__ keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  K x = keys[i] ^ keys[j];
  constexpr int W = 8 * sizeof(K);
  if (x == 0) return W + __clz((uint32_t)i ^ (uint32_t)j);
  if constexpr (sizeof(K) == 8)
    return __clzll((long long)x);
  else
    return __clz((int)x);
}

template <class K>
__global__ void k_karras(const K* __restrict__ keys, uint32_t nn, uint32_t* __restrict__ left,
                         uint32_t* __restrict__ right, uint32_t* __restrict__ parent_int,
                         uint32_t* __restrict__ parent_leaf) {
  const int n = (int)nn;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1) < 0) ? -1 : 1;
  int dmin = kdelta(keys, n, i, i - d);
  int lmax = 2;
  while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int first = min(i, j), last = max(i, j);
  int nd = kdelta(keys, n, first, last);
  int split = first, step = last - first;
  for (;;) {
    step = (step + 1) / 2;
    int ns = split + step;
    if (ns < last && kdelta(keys, n, first, ns) > nd) split = ns;
    if (step <= 1) break;
  }
  int g = split;
  uint32_t lc = (first == g) ? ((uint32_t)g | LEAF_BIT) : (uint32_t)g;
  uint32_t rc = (last == g + 1) ? ((uint32_t)(g + 1) | LEAF_BIT) : (uint32_t)(g + 1);
  left[i] = lc;
  right[i] = rc;
  if (lc & LEAF_BIT)
    parent_leaf[lc & ~LEAF_BIT] = (uint32_t)i;
  else
    parent_int[lc] = (uint32_t)i;
  if (rc & LEAF_BIT)
    parent_leaf[rc & ~LEAF_BIT] = (uint32_t)i;
  else
    parent_int[rc] = (uint32_t)i;
  if (i == 0) parent_int[0] = NO_PARENT;
}

// ---------------------------------------------------------------------------------------
// Boxes: leaf boxes in sorted order, then one climb per leaf (second arrival merges).
// Boxes are stored as two float4 (lo.xyz, -, hi.xyz, -).
// ---------------------------------------------------------------------------------------
__global__ void k_leaf_boxes(const float* __restrict__ pos, const uint32_t* __restrict__ tris,
                             const uint32_t* __restrict__ perm, uint32_t nt, float4* __restrict__ leaf) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  uint32_t t = perm[i];
  float lo[3], hi[3];
  for (int c = 0; c < 3; ++c) {
    float a = pos[3 * tris[3 * t] + c], b = pos[3 * tris[3 * t + 1] + c], d = pos[3 * tris[3 * t + 2] + c];
    lo[c] = fminf(fminf(a, b), d);
    hi[c] = fmaxf(fmaxf(a, b), d);
  }
  leaf[2 * i] = make_float4(lo[0], lo[1], lo[2], 0.f);
  leaf[2 * i + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

// Displacement boxes: per leaf, the AABB of the primitive's vertices' displacements dx.
__global__ void k_leaf_disp_boxes(const float* __restrict__ dx, const uint32_t* __restrict__ tris,
                                  const uint32_t* __restrict__ perm, uint32_t nt, float4* __restrict__ leaf) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  uint32_t t = perm[i];
  const uint32_t v0 = tris[3 * t], v1 = tris[3 * t + 1], v2 = tris[3 * t + 2];
  float lo[3], hi[3];
  for (int c = 0; c < 3; ++c) {
    float a = dx[3 * v0 + c], b = dx[3 * v1 + c], d = dx[3 * v2 + c];
    lo[c] = fminf(fminf(a, b), d);
    hi[c] = fmaxf(fmaxf(a, b), d);
  }
  leaf[2 * i] = make_float4(lo[0], lo[1], lo[2], 0.f);
  leaf[2 * i + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

__device__ __forceinline__ void child_box(uint32_t c, const float4* leaf, const float4* node, float4& lo, float4& hi) {
  const float4* src = (c & LEAF_BIT) ? leaf + 2 * (c & ~LEAF_BIT) : node + 2 * c;
  lo = __ldcg(src);
  hi = __ldcg(src + 1);
}

// cb (4 float4 per internal node; may be null) receives each node's two children's boxes as
// read.
__global__ void k_refit(const uint32_t* __restrict__ parent_leaf, const uint32_t* __restrict__ parent_int,
                        const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                        const float4* __restrict__ leaf, float4* node, float4* __restrict__ cb, uint32_t* flags,
                        uint32_t nt) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt || nt < 2) return;
  uint32_t p = parent_leaf[i];
  uint32_t guard = 0;
  while (p != NO_PARENT && guard++ < 64u * 1024u) {
    __threadfence();
    if (atomicAdd(&flags[p], 1u) == 0u) return;
    __threadfence();
    float4 a0, a1, b0, b1;
    child_box(left[p], leaf, node, a0, a1);
    child_box(right[p], leaf, node, b0, b1);
    float4 lo = make_float4(fminf(a0.x, b0.x), fminf(a0.y, b0.y), fminf(a0.z, b0.z), 0.f);
    float4 hi = make_float4(fmaxf(a1.x, b1.x), fmaxf(a1.y, b1.y), fmaxf(a1.z, b1.z), 0.f);
    __stcg(node + 2 * p, lo);
    __stcg(node + 2 * p + 1, hi);
    if (cb) {
      float4* c4 = cb + 4 * (size_t)p;
      c4[0] = a0;
      c4[1] = a1;
      c4[2] = b0;
      c4[3] = b1;
    }
    p = parent_int[p];
  }
}

// ---------------------------------------------------------------------------------------
// Traversal: one query box per thread, queries visited in Morton order (qorder) so that a
// warp walks neighbouring queries down the same subtrees. Children are tested from the
// parent; overlapping internal children are pushed on a 64-deep stack.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ bool overlap(const float4& qlo, const float4& qhi, const float4& blo, const float4& bhi) {
  return qlo.x <= bhi.x && qlo.y <= bhi.y && qlo.z <= bhi.z && blo.x <= qhi.x && blo.y <= qhi.y && blo.z <= qhi.z;
}

__global__ void k_point_boxes(const float* __restrict__ pts, uint32_t np, float pad, float4* __restrict__ qbox) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
  qbox[2 * i] = make_float4(__fsub_rn(x, pad), __fsub_rn(y, pad), __fsub_rn(z, pad), 0.f);
  qbox[2 * i + 1] = make_float4(__fadd_rn(x, pad), __fadd_rn(y, pad), __fadd_rn(z, pad), 0.f);
}

__global__ void __launch_bounds__(128) k_traverse(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                                                  const float4* __restrict__ node, const float4* __restrict__ leaf,
                                                  const uint32_t* __restrict__ prim, uint32_t nt,
                                                  const float4* __restrict__ qbox, const uint32_t* __restrict__ qorder,
                                                  uint32_t nq, uint32_t* __restrict__ pairs, uint64_t cap,
                                                  unsigned long long* __restrict__ count, uint32_t* __restrict__ status) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nq || nt == 0) return;
  uint32_t q = qorder ? qorder[k] : k;
  const float4 qlo = qbox[2 * q], qhi = qbox[2 * q + 1];
  auto emit = [&](uint32_t lf) {
    unsigned long long at = atomicAdd(count, 1ull);
    if (at < cap) {
      pairs[2 * at] = q;
      pairs[2 * at + 1] = prim[lf];
    } else {
      atomicOr(status, ST_PAIR_OVERFLOW);
    }
  };
  if (nt == 1) {
    if (overlap(qlo, qhi, leaf[0], leaf[1])) emit(0);
    return;
  }
  uint32_t stack[64];
  int sp = 0;
  uint32_t cur = 0;  // root internal node
  // the root itself is tested first, as the reference does
  if (!overlap(qlo, qhi, __ldg(node), __ldg(node + 1))) return;
  for (;;) {
    uint32_t ch[2] = {__ldg(left + cur), __ldg(right + cur)};
    uint32_t next = NO_PARENT;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uint32_t x = ch[c];
      const float4* b = (x & LEAF_BIT) ? leaf + 2 * (x & ~LEAF_BIT) : node + 2 * x;
      float4 blo = __ldg(b), bhi = __ldg(b + 1);
      if (!overlap(qlo, qhi, blo, bhi)) continue;
      if (x & LEAF_BIT) {
        emit(x & ~LEAF_BIT);
      } else if (next == NO_PARENT) {
        next = x;
      } else if (sp < 64) {
        stack[sp++] = x;
      } else {
        atomicOr(status, ST_STACK_OVERFLOW);
      }
    }
    if (next != NO_PARENT) {
      cur = next;
    } else if (sp > 0) {
      cur = stack[--sp];
    } else {
      break;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------------------
template <class K>
static int sort_impl(Lbvh* b, K* keys, uint32_t* vals, uint32_t n, int key_bits, cudaStream_t s) {
  if (n <= 1) return MGUSO_OK;
  int passes = (key_bits + 7) / 8;
  MG_TRY(b->rs_hist.reserve(8 * 256));
  MG_TRY(b->rs_ofs.reserve(8 * 256));
  uint32_t ntiles = ceil_div(n, RS_TILE);
  MG_TRY(b->rs_status.grow((size_t)ntiles * 256));
  MG_TRY(b->rs_counter.reserve(8));
  MG_TRY(b->rs_tmpk.grow((size_t)n * sizeof(K)));
  MG_TRY(b->rs_tmpv.grow(n));
  MG_CUDA(cudaMemsetAsync(b->rs_hist.p, 0, 4 * 8 * 256, s));
  int sms = device_sm_count();
  k_rs_hist<K><<<std::min<uint32_t>(ceil_div(n, 256), sms * 8), 256, 0, s>>>(keys, n, passes, b->rs_hist.p);
  k_rs_scan<<<passes, 256, 0, s>>>(b->rs_hist.p, b->rs_ofs.p);
  MG_CUDA(cudaGetLastError());
  // every pass is launched; a pass whose digit is the same for every key finds that out on
  // the device and only copies, so the sort needs no readback
  K* kA = keys;
  uint32_t* vA = vals;
  K* kB = (K*)b->rs_tmpk.p;
  uint32_t* vB = b->rs_tmpv.p;
  for (int p = 0; p < passes; ++p) {
    MG_CUDA(cudaMemsetAsync(b->rs_status.p, 0, 4 * (size_t)ntiles * 256, s));
    MG_CUDA(cudaMemsetAsync(b->rs_counter.p, 0, 4, s));
    k_onesweep<K><<<ntiles, RS_THREADS, 0, s>>>(kA, vA, kB, vB, n, 8 * p, b->rs_ofs.p + p * 256, b->rs_status.p,
                                               b->rs_counter.p, b->err_sink ? b->err_sink : b->status.p,
                                               b->rs_hist.p + p * 256);
    MG_CUDA(cudaGetLastError());
    std::swap(kA, kB);
    std::swap(vA, vB);
  }
  if (kA != keys) {
    MG_CUDA(cudaMemcpyAsync(keys, kA, sizeof(K) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    MG_CUDA(cudaMemcpyAsync(vals, vA, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  }
  return MGUSO_OK;
}

int radix_sort_pairs(Lbvh* b, void* keys, uint32_t* vals, uint32_t n, int key_bits, cudaStream_t s) {
  if (key_bits <= 32) return sort_impl<uint32_t>(b, (uint32_t*)keys, vals, n, key_bits, s);
  return sort_impl<uint64_t>(b, (uint64_t*)keys, vals, n, key_bits, s);
}

// the centroid-bounds accumulator's start (ordered bits): the three minima at their highest
// value, the three maxima at their lowest
__global__ void k_ord_init(uint32_t* __restrict__ ord) {
  if (threadIdx.x < 6) ord[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
}

template <class K>
static int build_impl(Lbvh* b, const float* pos, const uint32_t* tris, uint32_t nt, int key_bits, cudaStream_t s) {
  b->shaped = false;
  b->nt = nt;
  b->key_bits = key_bits;
  MG_TRY(b->keys.reserve((size_t)std::max<uint32_t>(nt, 1) * sizeof(K)));
  MG_TRY(b->perm.reserve(std::max<uint32_t>(nt, 1)));
  MG_TRY(b->left.reserve(std::max<uint32_t>(nt, 2)));
  MG_TRY(b->right.reserve(std::max<uint32_t>(nt, 2)));
  MG_TRY(b->parent_int.reserve(std::max<uint32_t>(nt, 2)));
  MG_TRY(b->parent_leaf.reserve(std::max<uint32_t>(nt, 1)));
  MG_TRY(b->leaf.reserve(2 * (size_t)std::max<uint32_t>(nt, 1)));
  MG_TRY(b->node.reserve(2 * (size_t)std::max<uint32_t>(nt, 2)));
  if (b->child_boxes) MG_TRY(b->cbox.reserve(4 * (size_t)std::max<uint32_t>(nt, 2)));
  MG_TRY(b->flags.reserve(std::max<uint32_t>(nt, 2)));
  MG_TRY(b->params.reserve(8));
  MG_TRY(b->ord.reserve(8));
  MG_TRY(b->status.reserve(4));
  if (nt == 0) return MGUSO_OK;
  k_ord_init<<<1, 32, 0, s>>>(b->ord.p);
  int sms = device_sm_count();
  k_centroid_bounds<<<std::min<uint32_t>(ceil_div(nt, 256), sms * 8), 256, 0, s>>>(pos, tris, nt, b->ord.p);
  k_bounds_finish<<<1, 32, 0, s>>>(b->ord.p, b->params.p);
  K* keys = (K*)b->keys.p;
  k_morton<K><<<ceil_div(nt, 256), 256, 0, s>>>(pos, tris, nt, b->params.p, keys, b->perm.p);
  MG_CUDA(cudaGetLastError());
  if (b->ev_on) cudaEventRecord(b->ev[1], s);
  MG_TRY(sort_impl<K>(b, keys, b->perm.p, nt, key_bits, s));
  if (b->ev_on) cudaEventRecord(b->ev[2], s);
  if (nt > 1) {
    k_karras<K><<<ceil_div(nt - 1, 256), 256, 0, s>>>(keys, nt, b->left.p, b->right.p, b->parent_int.p,
                                                     b->parent_leaf.p);
  }
  if (b->ev_on) cudaEventRecord(b->ev[3], s);
  k_leaf_boxes<<<ceil_div(nt, 256), 256, 0, s>>>(pos, tris, b->perm.p, nt, (float4*)b->leaf.p);
  if (nt > 1) {
    MG_CUDA(cudaMemsetAsync(b->flags.p, 0, 4 * (size_t)(nt - 1), s));
    k_refit<<<ceil_div(nt, 256), 256, 0, s>>>(b->parent_leaf.p, b->parent_int.p, b->left.p, b->right.p,
                                             (const float4*)b->leaf.p, (float4*)b->node.p,
                                             b->child_boxes ? b->cbox.p : nullptr, b->flags.p, nt);
  }
  MG_CUDA(cudaGetLastError());
  if (b->ev_on) cudaEventRecord(b->ev[4], s);
  b->shaped = true;
  return MGUSO_OK;
}

int lbvh_refit_disp(Lbvh* b, const float* dx, const uint32_t* tris, cudaStream_t s) {
  const uint32_t nt = b->nt;
  MG_TRY(b->dleaf.reserve(2 * (size_t)std::max<uint32_t>(nt, 1)));
  MG_TRY(b->dnode.reserve(2 * (size_t)std::max<uint32_t>(nt, 2)));
  if (b->child_boxes) MG_TRY(b->dcbox.reserve(4 * (size_t)std::max<uint32_t>(nt, 2)));
  if (nt == 0) return MGUSO_OK;
  k_leaf_disp_boxes<<<ceil_div(nt, 256), 256, 0, s>>>(dx, tris, b->perm.p, nt, b->dleaf.p);
  if (nt > 1) {
    MG_CUDA(cudaMemsetAsync(b->flags.p, 0, 4 * (size_t)(nt - 1), s));
    k_refit<<<ceil_div(nt, 256), 256, 0, s>>>(b->parent_leaf.p, b->parent_int.p, b->left.p, b->right.p, b->dleaf.p,
                                             b->dnode.p, b->child_boxes ? b->dcbox.p : nullptr, b->flags.p, nt);
  }
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int lbvh_refit_pos(Lbvh* b, const float* pos, const uint32_t* tris, cudaStream_t s) {
  const uint32_t nt = b->nt;
  MG_CHECK_ARG(b->shaped, "LBVH refit before a complete build");
  if (nt == 0) return MGUSO_OK;
  // sized by the last build already (these only check, unless that build stopped early)
  MG_TRY(b->leaf.reserve(2 * (size_t)nt));
  MG_TRY(b->node.reserve(2 * (size_t)std::max<uint32_t>(nt, 2)));
  if (b->child_boxes) MG_TRY(b->cbox.reserve(4 * (size_t)std::max<uint32_t>(nt, 2)));
  MG_TRY(b->flags.reserve(std::max<uint32_t>(nt, 2)));
  k_leaf_boxes<<<ceil_div(nt, 256), 256, 0, s>>>(pos, tris, b->perm.p, nt, (float4*)b->leaf.p);
  if (nt > 1) {
    MG_CUDA(cudaMemsetAsync(b->flags.p, 0, 4 * (size_t)(nt - 1), s));
    k_refit<<<ceil_div(nt, 256), 256, 0, s>>>(b->parent_leaf.p, b->parent_int.p, b->left.p, b->right.p,
                                             (const float4*)b->leaf.p, (float4*)b->node.p,
                                             b->child_boxes ? b->cbox.p : nullptr, b->flags.p, nt);
  }
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int lbvh_build(Lbvh* b, const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, int key_bits,
               cudaStream_t s) {
  (void)nv;
  MG_CHECK_ARG(key_bits == 30 || key_bits == 63, "key_bits must be 30 or 63");
  MG_TRY(b->status.reserve(4));
  if (b->ev_on) cudaEventRecord(b->ev[0], s);
  if (key_bits == 30) return build_impl<uint32_t>(b, pos, tris, nt, key_bits, s);
  return build_impl<uint64_t>(b, pos, tris, nt, key_bits, s);
}

int lbvh_query_boxes(Lbvh* b, const float4* qbox, const uint32_t* qorder, uint32_t nq, uint32_t* pairs, uint64_t cap,
                     unsigned long long* count, cudaStream_t s) {
  if (nq == 0 || b->nt == 0) return MGUSO_OK;
  k_traverse<<<ceil_div(nq, 128), 128, 0, s>>>(b->left.p, b->right.p, (const float4*)b->node.p,
                                               (const float4*)b->leaf.p, b->perm.p, b->nt, qbox, qorder, nq, pairs,
                                               cap, count, b->status.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

int lbvh_query_points(Lbvh* b, const float* pts, uint32_t np, float dhat, uint32_t* pairs, uint64_t cap,
                      unsigned long long* count, bool morton_order, cudaStream_t s) {
  MG_TRY(b->qbox.reserve(2 * (size_t)std::max<uint32_t>(np, 1)));
  MG_TRY(b->qkeys.reserve(std::max<uint32_t>(np, 1)));
  MG_TRY(b->qorder.reserve(std::max<uint32_t>(np, 1)));
  if (np == 0) return MGUSO_OK;
  k_point_boxes<<<ceil_div(np, 256), 256, 0, s>>>(pts, np, dhat, (float4*)b->qbox.p);
  const uint32_t* order = nullptr;
  if (morton_order && b->nt > 0) {
    k_morton_points<<<ceil_div(np, 256), 256, 0, s>>>(pts, np, b->params.p, b->qkeys.p, b->qorder.p);
    MG_TRY(sort_impl<uint32_t>(b, b->qkeys.p, b->qorder.p, np, 30, s));
    order = b->qorder.p;
  }
  MG_CUDA(cudaGetLastError());
  if (b->ev_on) cudaEventRecord(b->ev[5], s);
  MG_TRY(lbvh_query_boxes(b, (const float4*)b->qbox.p, order, np, pairs, cap, count, s));
  if (b->ev_on) cudaEventRecord(b->ev[6], s);
  return MGUSO_OK;
}

// ---------------------------------------------------------------------------------------
// Allocation-free pair sort. Some callers may not allocate device memory after start-up:
// a host engine that hands all of the GPU's memory to its own pool when it starts, or a
// per-frame path where cudaMalloc's implicit device-wide synchronisation would stall the
// other streams. mguso_radix_sort_pairs_noalloc runs the same onesweep passes as
// radix_sort_pairs, with its temporaries in one fixed file-scope device array instead of
// buffers that grow on demand.
//
// Differences from radix_sort_pairs: every digit pass runs the full scatter (radix_sort_pairs
// turns a pass whose digit is the same for every key into a tile copy, found on the device;
// such a pass is the identity for a stable sort, so the output is the same), and the call
// waits for the sort to finish so it can report a look-back timeout from the scratch's
// error word.
// ---------------------------------------------------------------------------------------
constexpr uint32_t NOALLOC_MAX_PAIRS = 1u << 18;  // 262 144 pairs
constexpr size_t NA_TMPK = 0;                                         // u64 keys, ping-pong
constexpr size_t NA_TMPV = NA_TMPK + 8 * (size_t)NOALLOC_MAX_PAIRS;   // u32 payloads
constexpr size_t NA_STATUS = NA_TMPV + 4 * (size_t)NOALLOC_MAX_PAIRS; // look-back flags
constexpr size_t NA_HIST = NA_STATUS + 4 * 256 * (size_t)(NOALLOC_MAX_PAIRS / RS_TILE);
constexpr size_t NA_OFS = NA_HIST + 4 * 8 * 256;
constexpr size_t NA_MISC = NA_OFS + 4 * 8 * 256;  // [0] tile counter, [1] error word
constexpr size_t NA_BYTES = NA_MISC + 256;         // 3.2 MiB per device
static_assert(NOALLOC_MAX_PAIRS % RS_TILE == 0, "scratch holds whole tiles");

// Every device that loads the library holds this array until the process exits. Host code
// must not pass the symbol itself to a kernel: its device address comes from
// cudaGetSymbolAddress, taken once per device below.
static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_ptr[NA_MAX_DEVICES] = {};

// Device address of the scratch array on the current device (looked up on first use).
static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  MG_CUDA(cudaGetDevice(&dev));
  MG_CHECK_ARG(dev >= 0 && dev < NA_MAX_DEVICES, "device index beyond the allocation-free sort's table");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress(sort scratch): ") + cudaGetErrorString(e));
      return MGUSO_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = (unsigned char*)p;
  }
  *out = g_noalloc_ptr[dev];
  return MGUSO_OK;
}

template <class K>
static int noalloc_sort(unsigned char* sc, K* keys, uint32_t* vals, uint32_t n, int key_bits, cudaStream_t s) {
  const int passes = (key_bits + 7) / 8;
  const uint32_t ntiles = ceil_div(n, RS_TILE);
  uint32_t* hist = (uint32_t*)(sc + NA_HIST);
  uint32_t* ofs = (uint32_t*)(sc + NA_OFS);
  uint32_t* status = (uint32_t*)(sc + NA_STATUS);
  uint32_t* counter = (uint32_t*)(sc + NA_MISC);
  uint32_t* err = counter + 1;
  // the array keeps the previous call's contents: clear what the passes accumulate into
  MG_CUDA(cudaMemsetAsync(hist, 0, 4 * 8 * 256, s));
  MG_CUDA(cudaMemsetAsync(err, 0, 4, s));
  const int sms = device_sm_count();
  k_rs_hist<K><<<std::min<uint32_t>(ceil_div(n, 256), sms * 8), 256, 0, s>>>(keys, n, passes, hist);
  k_rs_scan<<<passes, 256, 0, s>>>(hist, ofs);
  MG_CUDA(cudaGetLastError());
  K* kA = keys;
  uint32_t* vA = vals;
  K* kB = (K*)(sc + NA_TMPK);
  uint32_t* vB = (uint32_t*)(sc + NA_TMPV);
  for (int p = 0; p < passes; ++p) {
    MG_CUDA(cudaMemsetAsync(status, 0, 4 * (size_t)ntiles * 256, s));
    MG_CUDA(cudaMemsetAsync(counter, 0, 4, s));
    k_onesweep<K><<<ntiles, RS_THREADS, 0, s>>>(kA, vA, kB, vB, n, 8 * p, ofs + p * 256, status, counter, err,
                                               nullptr);
    MG_CUDA(cudaGetLastError());
    std::swap(kA, kB);
    std::swap(vA, vB);
  }
  if (kA != keys) {
    MG_CUDA(cudaMemcpyAsync(keys, kA, sizeof(K) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    MG_CUDA(cudaMemcpyAsync(vals, vA, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  }
  uint32_t h_err = 0;
  MG_CUDA(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, s));
  MG_CUDA(cudaStreamSynchronize(s));
  if (h_err & ST_WAIT_TIMEOUT) {
    set_error("allocation-free sort: a decoupled look-back wait timed out");
    return MGUSO_ERR_TIMEOUT;
  }
  return MGUSO_OK;
}

}  // namespace mg

extern "C" int mguso_radix_sort_pairs_noalloc(void* keys, uint32_t* vals, uint32_t n, int key_bits, void* stream) {
  using namespace mg;
  MG_CHECK_ARG(key_bits >= 1 && key_bits <= 64, "key_bits must be in [1, 64]");
  if (n > NOALLOC_MAX_PAIRS) {
    set_error("mguso_radix_sort_pairs_noalloc: n = " + std::to_string(n) +
              " exceeds its fixed scratch limit of 262144 pairs; use mguso_radix_sort_pairs");
    return MGUSO_ERR_INVALID_ARG;
  }
  MG_CHECK_ARG(n == 0 || (keys && vals), "null argument");
  unsigned char* sc = nullptr;
  MG_TRY(noalloc_scratch(&sc));
  if (n <= 1) return MGUSO_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (key_bits <= 32) return noalloc_sort<uint32_t>(sc, (uint32_t*)keys, vals, n, key_bits, s);
  return noalloc_sort<uint64_t>(sc, (uint64_t*)keys, vals, n, key_bits, s);
}
