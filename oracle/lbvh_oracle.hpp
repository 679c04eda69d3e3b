// CPU oracle (TEST INFRASTRUCTURE ONLY) for the LBVH broad phase: Morton codes, a stable
// LSD radix sort of (key, payload) pairs, the Karras tree, bottom-up AABB propagation and
// the traversal's candidate-pair predicate.
//
// Follows core-engine/crates/engine-gpu/src/morton.rs:11-63 (30-bit codes),
// radix.rs:112-352 (stable LSD sort semantics), karras.rs:24-88 (tree),
// bvh_aabb.rs:13-56 (exact min/max node boxes) and shaders/bvh_traverse.wgsl:64-92
// (query box [p - dhat, p + dhat] against leaf boxes, `all(qlo <= bhi) && all(blo <= qhi)`).
//
// No reference exists for 63-bit codes: they follow the same quantisation with
// 21 bits per axis (`(clamp(n,0,1) * (2^21-1)) as u32`, x in the most significant bit of
// each triple), and the Karras tie-break extends to 64 + clz32(i ^ j). Parity of those two
// is therefore unpinned; everything else is pinned by the reference's own tests
// (morton.rs:273, radix.rs:361-417, karras.rs:313-333, bvh_aabb.rs:381,
// bvh_traverse.rs:287).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace mo {

inline uint32_t expand_bits10(uint32_t v) {
  uint32_t x = v & 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

inline uint64_t expand_bits21(uint64_t v) {
  uint64_t x = v & 0x1fffffull;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// Rust's `f32 as u32` saturates and maps NaN to 0.
inline uint32_t f32_as_u32(float v) {
  if (!(v > 0.0f)) return 0u;
  if (v >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)v;
}

inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// morton_code_cpu (morton.rs:21-24).
inline uint32_t morton30(float nx, float ny, float nz) {
  auto q = [](float v) { return f32_as_u32(clampf(clampf(v, 0.0f, 1.0f) * 1023.0f, 0.0f, 1023.0f)); };
  return expand_bits10(q(nx)) * 4u + expand_bits10(q(ny)) * 2u + expand_bits10(q(nz));
}

inline uint64_t morton63(float nx, float ny, float nz) {
  const float S = 2097151.0f;  // 2^21 - 1
  auto q = [&](float v) { return (uint64_t)f32_as_u32(clampf(clampf(v, 0.0f, 1.0f) * S, 0.0f, S)); };
  return expand_bits21(q(nx)) * 4ull + expand_bits21(q(ny)) * 2ull + expand_bits21(q(nz));
}

// centroid_bounds (morton.rs:30-47): centroid = (a + b + c) / 3 per component.
inline void centroid_bounds(const float* pos, const uint32_t* tris, size_t nt, float lo[3], float inv[3]) {
  float hi[3];
  for (int c = 0; c < 3; ++c) {
    lo[c] = INFINITY;
    hi[c] = -INFINITY;
  }
  for (size_t t = 0; t < nt; ++t) {
    const float* a = pos + 3 * tris[3 * t];
    const float* b = pos + 3 * tris[3 * t + 1];
    const float* d = pos + 3 * tris[3 * t + 2];
    for (int c = 0; c < 3; ++c) {
      float ctr = (a[c] + b[c] + d[c]) / 3.0f;
      lo[c] = std::min(lo[c], ctr);
      hi[c] = std::max(hi[c], ctr);
    }
  }
  for (int c = 0; c < 3; ++c) {
    float ext = hi[c] - lo[c];
    inv[c] = ext > 0.0f ? 1.0f / ext : 0.0f;
  }
}

// morton_codes_cpu (morton.rs:50-63); `bits` is 30 or 63.
template <class K>
inline std::vector<K> morton_codes(const float* pos, const uint32_t* tris, size_t nt, int bits) {
  float lo[3], inv[3];
  centroid_bounds(pos, tris, nt, lo, inv);
  std::vector<K> out(nt);
  for (size_t t = 0; t < nt; ++t) {
    const float* a = pos + 3 * tris[3 * t];
    const float* b = pos + 3 * tris[3 * t + 1];
    const float* d = pos + 3 * tris[3 * t + 2];
    float n[3];
    for (int c = 0; c < 3; ++c) {
      float ctr = (a[c] + b[c] + d[c]) / 3.0f;
      n[c] = (ctr - lo[c]) * inv[c];
    }
    if (bits == 30)
      out[t] = (K)morton30(n[0], n[1], n[2]);
    else
      out[t] = (K)morton63(n[0], n[1], n[2]);
  }
  return out;
}

// Stable sort of (key, payload) by key: the permutation an LSD radix sort produces
// (radix.rs:112-352; radix.rs:382-417 pins stability).
template <class K>
inline void stable_sort_pairs(std::vector<K>& keys, std::vector<uint32_t>& vals) {
  std::vector<uint32_t> idx(keys.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (uint32_t)i;
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
  std::vector<K> k2(keys.size());
  std::vector<uint32_t> v2(vals.size());
  for (size_t i = 0; i < idx.size(); ++i) {
    k2[i] = keys[idx[i]];
    v2[i] = vals[idx[i]];
  }
  keys.swap(k2);
  vals.swap(v2);
}

constexpr uint32_t LEAF = 0x80000000u;

inline int clz32(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }
inline int clz64(uint64_t x) { return x == 0 ? 64 : __builtin_clzll(x); }
template <class K> inline int clzk(K x);
template <> inline int clzk<uint32_t>(uint32_t x) { return clz32(x); }
template <> inline int clzk<uint64_t>(uint64_t x) { return clz64(x); }

// karras_tree_cpu (karras.rs:24-88); the tie-break adds the key width.
template <class K>
inline void karras_tree(const K* codes, size_t n, uint32_t* left, uint32_t* right) {
  const int W = (int)(8 * sizeof(K));
  auto delta = [&](int i, int j) -> int {
    if (j < 0 || j >= (int)n) return -1;
    K x = codes[i] ^ codes[j];
    if (x == 0) return W + clz32((uint32_t)i ^ (uint32_t)j);
    return clzk<K>(x);
  };
  int m = n > 0 ? (int)n - 1 : 0;
  for (int i = 0; i < m; ++i) {
    int d = (delta(i, i + 1) - delta(i, i - 1) < 0) ? -1 : 1;
    int delta_min = delta(i, i - d);
    int l_max = 2;
    while (delta(i, i + l_max * d) > delta_min) l_max *= 2;
    int l = 0;
    int t = l_max / 2;
    while (t >= 1) {
      if (delta(i, i + (l + t) * d) > delta_min) l += t;
      t /= 2;
    }
    int j = i + l * d;
    int first = std::min(i, j), last = std::max(i, j);
    int node_delta = delta(first, last);
    int split = first;
    int step = last - first;
    for (;;) {
      step = (step + 1) / 2;
      int ns = split + step;
      if (ns < last && delta(first, ns) > node_delta) split = ns;
      if (step <= 1) break;
    }
    int gamma = split;
    left[i] = (first == gamma) ? ((uint32_t)gamma | LEAF) : (uint32_t)gamma;
    right[i] = (last == gamma + 1) ? ((uint32_t)(gamma + 1) | LEAF) : (uint32_t)(gamma + 1);
  }
}

// propagate_aabb_cpu (bvh_aabb.rs:28-56), iterative post-order. Boxes are [lo.xyz, hi.xyz].
inline void propagate_aabb(const uint32_t* left, const uint32_t* right, const float* leaf, size_t n,
                           float* node) {
  if (n < 2) return;
  // children before parents: an explicit stack of (node, visited).
  std::vector<std::pair<uint32_t, bool>> st;
  st.push_back({0u, false});
  auto box_of = [&](uint32_t c) -> const float* {
    return (c & LEAF) ? leaf + 6 * (c & ~LEAF) : node + 6 * c;
  };
  while (!st.empty()) {
    auto [i, visited] = st.back();
    st.pop_back();
    if (!visited) {
      st.push_back({i, true});
      if (!(right[i] & LEAF)) st.push_back({right[i], false});
      if (!(left[i] & LEAF)) st.push_back({left[i], false});
    } else {
      const float* a = box_of(left[i]);
      const float* b = box_of(right[i]);
      float* o = node + 6 * i;
      for (int c = 0; c < 3; ++c) {
        o[c] = std::min(a[c], b[c]);
        o[3 + c] = std::max(a[3 + c], b[3 + c]);
      }
    }
  }
}

// Leaf boxes in sorted order: leaf i wraps triangle prim[i] (bvh_traverse.rs:316-328).
inline std::vector<float> leaf_boxes(const float* pos, const uint32_t* tris, const uint32_t* prim, size_t nt) {
  std::vector<float> out(6 * nt);
  for (size_t i = 0; i < nt; ++i) {
    const uint32_t* t = tris + 3 * prim[i];
    for (int c = 0; c < 3; ++c) {
      float a = pos[3 * t[0] + c], b = pos[3 * t[1] + c], d = pos[3 * t[2] + c];
      out[6 * i + c] = std::min(std::min(a, b), d);
      out[6 * i + 3 + c] = std::max(std::max(a, b), d);
    }
  }
  return out;
}

inline bool overlaps(const float q[6], const float* b) {
  return q[0] <= b[3] && q[1] <= b[4] && q[2] <= b[5] && b[0] <= q[3] && b[1] <= q[4] && b[2] <= q[5];
}

// The traversal's emitted pair SET (bvh_traverse.wgsl:64-92): (v, prim[leaf]) for every leaf
// whose box overlaps [p_v - dhat, p_v + dhat]. Node boxes are exact unions, so the set does
// not depend on the tree's shape; it is computed here by a depth-first walk of the oracle's
// own tree and returned sorted by (v, tri).
inline std::vector<std::pair<uint32_t, uint32_t>> traverse_pairs(const uint32_t* left, const uint32_t* right,
                                                                 const float* node, const float* leaf,
                                                                 const uint32_t* prim, size_t nt,
                                                                 const float* pos, size_t nv, float dhat) {
  std::vector<std::pair<uint32_t, uint32_t>> out;
  if (nt == 0) return out;
  std::vector<uint32_t> st;
  for (size_t v = 0; v < nv; ++v) {
    float q[6];
    for (int c = 0; c < 3; ++c) {
      q[c] = pos[3 * v + c] - dhat;
      q[3 + c] = pos[3 * v + c] + dhat;
    }
    size_t first = out.size();
    if (nt == 1) {
      if (overlaps(q, leaf)) out.push_back({(uint32_t)v, prim[0]});
      continue;
    }
    st.clear();
    st.push_back(0u);
    while (!st.empty()) {
      uint32_t nd = st.back();
      st.pop_back();
      if (nd & LEAF) {
        uint32_t lf = nd & ~LEAF;
        if (overlaps(q, leaf + 6 * lf)) out.push_back({(uint32_t)v, prim[lf]});
      } else if (overlaps(q, node + 6 * nd)) {
        st.push_back(left[nd]);
        st.push_back(right[nd]);
      }
    }
    std::sort(out.begin() + first, out.end());
  }
  return out;
}

}  // namespace mo
