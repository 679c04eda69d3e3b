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
  bool shaped = false;              // the last build enqueued its whole shape (refits may follow)
  DevBuf<unsigned char> keys;       // nt keys (u32 or u64), sorted after build
  DevBuf<uint32_t> perm;            // sorted leaf -> triangle
  DevBuf<uint32_t> left, right;     // nt - 1 internal nodes
  DevBuf<uint32_t> parent_int, parent_leaf;
  DevBuf<float4> leaf, node;        // 2 float4 per box (lo, hi)
  DevBuf<float4> dleaf, dnode;      // displacement boxes of the same tree (CCD pruning)
  // per internal node, its two children's boxes side by side (left lo, hi, right lo, hi), so
  // that a walk reads a node's child indices and their boxes in one round of loads; kept only
  // when child_boxes is set (the scene's trees, whose walks read them)
  DevBuf<float4> cbox, dcbox;
  bool child_boxes = true;
  DevBuf<uint32_t> flags;
  DevBuf<float> params;             // centroid lo.xyz, inv.xyz
  DevBuf<uint32_t> ord;
  DevBuf<uint32_t> status;
  uint32_t* err_sink = nullptr;     // when set, the sort's wait-timeout bit goes here instead of status
  // radix-sort scratch
  DevBuf<uint32_t> rs_hist, rs_ofs, rs_status, rs_counter, rs_tmpv;
  DevBuf<unsigned char> rs_tmpk;
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
// Leaf and node boxes at pos over the tree's existing shape (keys, permutation and children
// from the last lbvh_build, which must have had the same primitives; MGUSO_ERR_INVALID_ARG
// when that build did not complete): the boxes are exact
// unions again, so every overlap query returns the same leaves as after a rebuild at pos,
// only the shape fits pos less tightly.
int lbvh_refit_pos(Lbvh* b, const float* pos, const uint32_t* tris, cudaStream_t s);
// Displacement boxes (AABB of dx over each primitive's vertices, refitted up the tree) into
// dleaf/dnode, for the CCD's pruning test.
int lbvh_refit_disp(Lbvh* b, const float* dx, const uint32_t* tris, cudaStream_t s);
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

// Resumable walk over the leaves whose boxes overlap [qlo, qhi] (the predicate of
// lbvh_visit): start() and each step() hand back at most two leaf primitives, so a warp's
// lanes can advance their walks in lockstep and pool the leaves they reach. 64-entry stack;
// ok turns false on overflow.
struct BoxWalk {
  const uint32_t *left, *right, *prim;
  const float4 *node, *leaf, *cbox;
  uint32_t nt;
  float4 qlo, qhi;
  uint32_t stack[64];
  int sp;
  uint32_t cur;
  bool ok;

  __device__ __forceinline__ bool over(const float4& lo, const float4& hi) const {
    return qlo.x <= hi.x && qlo.y <= hi.y && qlo.z <= hi.z && lo.x <= qhi.x && lo.y <= qhi.y && lo.z <= qhi.z;
  }
  __device__ __forceinline__ bool enter(const float4* pb) const { return over(__ldg(pb), __ldg(pb + 1)); }
  __device__ __forceinline__ int start(bool& done, uint32_t out[2]) {
    sp = 0;
    cur = 0;
    ok = true;
    done = true;
    if (nt == 0) return 0;
    if (nt == 1) {
      if (enter(leaf)) {
        out[0] = prim[0];
        return 1;
      }
      return 0;
    }
    done = !enter(node);
    return 0;
  }
  __device__ __forceinline__ int step(bool& done, uint32_t out[2]) {
    int n = 0;
    const uint32_t ch[2] = {__ldg(left + cur), __ldg(right + cur)};
    const float4* cb = cbox + 4 * (size_t)cur;
    const bool in[2] = {over(__ldg(cb), __ldg(cb + 1)), over(__ldg(cb + 2), __ldg(cb + 3))};
    uint32_t next = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const uint32_t x = ch[c];
      const bool lf = (x & 0x80000000u) != 0;
      const uint32_t i = x & 0x7fffffffu;
      if (!in[c]) continue;
      if (lf) {
        out[n++] = prim[i];
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
      done = true;
    }
    return n;
  }
};

// CCD traversal (ccd_max_step's broad phase, implicit.rs:1690-1947, with exact pruning).
// A subtree is entered when the search box overlaps its position box (node, leaf) and its
// pairs with the query are not all settled by accd_toi's first test (contact.rs:378-437),
// which returns max_t = 1.25 whenever 1.25 u_max < 0.98 d0 (u_max: the largest relative
// displacement of the pair's four points; d0: their distance). Over a subtree, with the
// query's displacements inside the ball (cq, rq) and the subtree's inside its displacement
// box D (dnode, dleaf), the pairs' relative displacements are bounded by 2 rq (within the
// query), the diagonal of D (within a primitive) and rq + farthest(cq, D) (across), so
// u_max <= max(2 rq, diag D, rq + farthest(cq, D)); and d0 >= the distance between the
// query's box (qlo, qhi) and the subtree's position box. The subtree is skipped when
// 1.3 u_bound < 0.98 distance (4% margin over 1.25 for rounding).
//
// The walk is resumable: start() and each step() hand back at most two leaf primitives, so
// the lanes of a warp can advance their walks in lockstep and pool the leaves they reach
// (the root solves then run on full warps). 64-entry stack; ok turns false on overflow.
struct CcdWalk {
  const uint32_t *left, *right, *prim;
  const float4 *node, *leaf, *dnode, *dleaf, *cbox, *dcbox;
  uint32_t nt;
  float4 slo, shi, qlo, qhi;
  float3 cq;
  float rq;
  uint32_t stack[64];
  int sp;
  uint32_t cur;
  bool ok;

  __device__ __forceinline__ bool enter(const float4* pb, const float4* db) const {
    return enter_box(__ldg(pb), __ldg(pb + 1), db);
  }
  // the test of enter() with the position box given (db: the displacement box, read only
  // when the pruning bound is needed)
  __device__ __forceinline__ bool enter_box(const float4 lo, const float4 hi, const float4* db) const {
    if (!(slo.x <= hi.x && slo.y <= hi.y && slo.z <= hi.z && lo.x <= shi.x && lo.y <= shi.y && lo.z <= shi.z))
      return false;
    const float gx = fmaxf(fmaxf(qlo.x - hi.x, lo.x - qhi.x), 0.f);
    const float gy = fmaxf(fmaxf(qlo.y - hi.y, lo.y - qhi.y), 0.f);
    const float gz = fmaxf(fmaxf(qlo.z - hi.z, lo.z - qhi.z), 0.f);
    const float gap2 = gx * gx + gy * gy + gz * gz;
    if (gap2 == 0.f) return true;
    const float4 dlo = __ldg(db), dhi = __ldg(db + 1);
    const float fx = fmaxf(fabsf(cq.x - dlo.x), fabsf(cq.x - dhi.x));
    const float fy = fmaxf(fabsf(cq.y - dlo.y), fabsf(cq.y - dhi.y));
    const float fz = fmaxf(fabsf(cq.z - dlo.z), fabsf(cq.z - dhi.z));
    const float ex = dhi.x - dlo.x, ey = dhi.y - dlo.y, ez = dhi.z - dlo.z;
    const float u = fmaxf(fmaxf(2.f * rq, sqrtf(ex * ex + ey * ey + ez * ez)), rq + sqrtf(fx * fx + fy * fy + fz * fz));
    return !(1.3f * u < 0.98f * sqrtf(gap2));
  }
  // Begins the walk; returns the number of leaves written to out (the single leaf of a
  // one-primitive tree) and sets done when nothing is left to visit.
  __device__ __forceinline__ int start(bool& done, uint32_t out[2]) {
    sp = 0;
    cur = 0;
    ok = true;
    done = true;
    if (nt == 0) return 0;
    if (nt == 1) {
      if (enter(leaf, dleaf)) {
        out[0] = prim[0];
        return 1;
      }
      return 0;
    }
    done = !enter(node, dnode);
    return 0;
  }
  // Visits the children of the current node: entered leaves go to out (returned count),
  // an entered inner child becomes the next node (the second is stacked).
  __device__ __forceinline__ int step(bool& done, uint32_t out[2]) {
    int n = 0;
    const uint32_t ch[2] = {__ldg(left + cur), __ldg(right + cur)};
    const float4* cb = cbox + 4 * (size_t)cur;
    const float4* db = dcbox + 4 * (size_t)cur;
    const bool in[2] = {enter_box(__ldg(cb), __ldg(cb + 1), db), enter_box(__ldg(cb + 2), __ldg(cb + 3), db + 2)};
    uint32_t next = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const uint32_t x = ch[c];
      const bool lf = (x & 0x80000000u) != 0;
      const uint32_t i = x & 0x7fffffffu;
      if (!in[c]) continue;
      if (lf) {
        out[n++] = prim[i];
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
      done = true;
    }
    return n;
  }
};

}  // namespace mg
