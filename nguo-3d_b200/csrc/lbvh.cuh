// LBVH state behind the mguso_lbvh handle.
#pragma once
#include "internal.cuh"

namespace mg {

constexpr uint32_t LEAF_BIT = 0x80000000u;  // karras.rs:14
constexpr uint32_t NO_PARENT = 0xffffffffu;

struct Lbvh {
  mguso_ctx* ctx = nullptr;
  uint32_t nt = 0;
  int key_bits = 30;
  DevBuf<unsigned char> keys;       // nt keys (u32 or u64), sorted after build
  DevBuf<uint32_t> perm;            // sorted leaf -> triangle
  DevBuf<uint32_t> left, right;     // nt - 1 internal nodes
  DevBuf<uint32_t> parent_int, parent_leaf;
  DevBuf<float4> leaf, node;        // 2 float4 per box (lo, hi)
  DevBuf<float4> cleaf, cnode;      // boxes inflated per primitive (CCD pruning), same tree
  DevBuf<uint32_t> flags;
  DevBuf<float> params;             // centroid lo.xyz, inv.xyz
  DevBuf<uint32_t> ord;
  DevBuf<uint32_t> status;
  // radix-sort scratch
  DevBuf<uint32_t> rs_hist, rs_ofs, rs_status, rs_counter, rs_tmpv;
  DevBuf<unsigned char> rs_tmpk;
  int last_sort_passes = 0;
  // query scratch
  DevBuf<float4> qbox;
  DevBuf<uint32_t> qkeys, qorder;
  // optional per-stage timing events: 0 start, 1 morton, 2 sort, 3 karras, 4 refit,
  // 5 query prep, 6 traversal
  bool ev_on = false;
  cudaEvent_t ev[7] = {};
};

int radix_sort_pairs(Lbvh* b, void* keys, uint32_t* vals, uint32_t n, int key_bits, cudaStream_t s);
int lbvh_build(Lbvh* b, const float* pos, uint32_t nv, const uint32_t* tris, uint32_t nt, int key_bits,
               cudaStream_t s);
// Refits the built tree with every leaf box grown by the largest radius rv[] of its
// primitive's vertices (tris as passed to lbvh_build), into cleaf/cnode.
int lbvh_refit_inflated(Lbvh* b, const float* pos, const uint32_t* tris, const float* rv, cudaStream_t s);
int lbvh_query_boxes(Lbvh* b, const float4* qbox, const uint32_t* qorder, uint32_t nq, uint32_t* pairs, uint64_t cap,
                     unsigned long long* count, cudaStream_t s);
int lbvh_query_points(Lbvh* b, const float* pts, uint32_t np, float dhat, uint32_t* pairs, uint64_t cap,
                      unsigned long long* count, bool morton_order, cudaStream_t s);

}  // namespace mg

struct mguso_lbvh {
  mg::Lbvh b;
  mg::DevBuf<unsigned long long> count;
  mg::DevBuf<float> hpos;
  mg::DevBuf<uint32_t> htris, hpairs;
};

namespace mg {

// Visits every leaf whose box overlaps [qlo, qhi] (the predicate of
// bvh_traverse.wgsl:64-92), calling f(leaf_primitive). 64-entry stack; returns false on
// stack overflow.
template <class F>
__device__ __forceinline__ bool lbvh_visit(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                                           const float4* __restrict__ node, const float4* __restrict__ leaf,
                                           const uint32_t* __restrict__ prim, uint32_t nt, float4 qlo, float4 qhi,
                                           F&& f) {
  auto ov = [&](const float4& lo, const float4& hi) {
    return qlo.x <= hi.x && qlo.y <= hi.y && qlo.z <= hi.z && lo.x <= qhi.x && lo.y <= qhi.y && lo.z <= qhi.z;
  };
  if (nt == 0) return true;
  if (nt == 1) {
    if (ov(leaf[0], leaf[1])) f(prim[0]);
    return true;
  }
  if (!ov(__ldg(node), __ldg(node + 1))) return true;
  uint32_t stack[64];
  int sp = 0;
  uint32_t cur = 0;
  bool ok = true;
  for (;;) {
    uint32_t ch[2] = {__ldg(left + cur), __ldg(right + cur)};
    uint32_t next = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uint32_t x = ch[c];
      const float4* b = (x & 0x80000000u) ? leaf + 2 * (x & 0x7fffffffu) : node + 2 * x;
      if (!ov(__ldg(b), __ldg(b + 1))) continue;
      if (x & 0x80000000u) {
        f(prim[x & 0x7fffffffu]);
      } else if (next == 0xffffffffu) {
        next = x;
      } else if (sp < 64) {
        stack[sp++] = x;
      } else {
        ok = false;
      }
    }
    if (next != 0xffffffffu) {
      cur = next;
    } else if (sp > 0) {
      cur = stack[--sp];
    } else {
      break;
    }
  }
  return ok;
}

// As lbvh_visit, but a subtree is entered only if query box 1 overlaps its box in (node,
// leaf) AND query box 2 overlaps its box in (node2, leaf2): two conservative tests over the
// same tree, intersected.
template <class F>
__device__ __forceinline__ bool lbvh_visit2(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                                            const float4* __restrict__ node, const float4* __restrict__ leaf,
                                            const float4* __restrict__ node2, const float4* __restrict__ leaf2,
                                            const uint32_t* __restrict__ prim, uint32_t nt, float4 q1lo, float4 q1hi,
                                            float4 q2lo, float4 q2hi, F&& f) {
  auto ov = [](const float4& qlo, const float4& qhi, const float4& lo, const float4& hi) {
    return qlo.x <= hi.x && qlo.y <= hi.y && qlo.z <= hi.z && lo.x <= qhi.x && lo.y <= qhi.y && lo.z <= qhi.z;
  };
  auto both = [&](const float4* b1, const float4* b2) {
    return ov(q1lo, q1hi, __ldg(b1), __ldg(b1 + 1)) && ov(q2lo, q2hi, __ldg(b2), __ldg(b2 + 1));
  };
  if (nt == 0) return true;
  if (nt == 1) {
    if (both(leaf, leaf2)) f(prim[0]);
    return true;
  }
  if (!both(node, node2)) return true;
  uint32_t stack[64];
  int sp = 0;
  uint32_t cur = 0;
  bool ok = true;
  for (;;) {
    uint32_t ch[2] = {__ldg(left + cur), __ldg(right + cur)};
    uint32_t next = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      uint32_t x = ch[c];
      const bool lf = (x & 0x80000000u) != 0;
      const uint32_t i = x & 0x7fffffffu;
      if (!(lf ? both(leaf + 2 * i, leaf2 + 2 * i) : both(node + 2 * i, node2 + 2 * i))) continue;
      if (lf) {
        f(prim[i]);
      } else if (next == 0xffffffffu) {
        next = x;
      } else if (sp < 64) {
        stack[sp++] = x;
      } else {
        ok = false;
      }
    }
    if (next != 0xffffffffu) {
      cur = next;
    } else if (sp > 0) {
      cur = stack[--sp];
    } else {
      break;
    }
  }
  return ok;
}

}  // namespace mg
