// Self contact on the GPU: LBVH candidates, static-collider sides, the active stencil set
// and the CCD step filter.
//
// Reference: self_collision_stencils (implicit.rs:678-753), collider_sides
// (implicit.rs:1431-1475) and ccd_max_step (implicit.rs:1690-1947), whose broad phase is a
// uniform hash grid (broadphase.rs:263-526). Here candidates come from two LBVHs built over
// the current positions (triangles, and edges as degenerate triangles), with the exact box
// predicate the grid over-approximates: a vertex against a triangle's box grown by the
// search radius, an edge's box grown by it against another edge's box. Every stencil the
// grid finds within its activation gap is found here (the gap test is exact), with the
// same 1-ring exclusion, movability filter and shared-vertex rule. Stencils are sorted by
// (kind, primitive, primitive) to reproduce the reference's sorted, deduplicated order.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "elements.cuh"
#include "scene.cuh"

namespace mg {

__device__ __forceinline__ bool excluded(const uint32_t* ex_ptr, const uint32_t* ex_list, uint32_t v, uint32_t a,
                                         uint32_t b, uint32_t c) {
  for (uint32_t k = ex_ptr[v]; k < ex_ptr[v + 1]; ++k) {
    uint32_t e = ex_list[k];
    if (e == a || e == b || e == c) return true;
  }
  return false;
}

struct BvhView {
  const uint32_t *left, *right, *prim;
  const float4 *node, *leaf;
  uint32_t n;
  const float4 *dnode, *dleaf;  // displacement boxes of the same tree (CCD only)
  const float4 *cbox, *dcbox;   // children's position and displacement boxes per inner node
};

static BvhView view(const Lbvh& b) {
  return BvhView{b.left.p, b.right.p, b.perm.p, (const float4*)b.node.p, (const float4*)b.leaf.p, b.nt,
                 (const float4*)b.dnode.p, (const float4*)b.dleaf.p, (const float4*)b.cbox.p,
                 (const float4*)b.dcbox.p};
}

// One tree per instance over that instance's primitives (a query only meets its own
// instance); base[k] turns a tree's local primitive index into the scene's.
struct BvhSet {
  BvhView t[PCG_MAX_INST];
  uint32_t base[PCG_MAX_INST];
};

static BvhSet view_set(const std::vector<std::unique_ptr<Lbvh>>& b, const std::vector<uint32_t>& base) {
  BvhSet s{};
  for (size_t k = 0; k < b.size(); ++k) {
    s.t[k] = view(*b[k]);
    s.base[k] = base[k];
  }
  return s;
}

template <class F>
__device__ __forceinline__ bool visit(const BvhSet& bs, uint32_t k, float4 lo, float4 hi, F&& f) {
  const BvhView& bv = bs.t[k];
  const uint32_t base = bs.base[k];
  return lbvh_visit(bv.left, bv.right, bv.node, bv.leaf, bv.prim, bv.n, lo, hi,
                    [&](uint32_t local) { f(base + local); });
}

__device__ __forceinline__ void point_box(const float* x, uint32_t v, float pad, float4& lo, float4& hi) {
  float a = x[3 * v], b = x[3 * v + 1], c = x[3 * v + 2];
  lo = make_float4(__fsub_rn(a, pad), __fsub_rn(b, pad), __fsub_rn(c, pad), 0.f);
  hi = make_float4(__fadd_rn(a, pad), __fadd_rn(b, pad), __fadd_rn(c, pad), 0.f);
}

__device__ __forceinline__ void edge_box(const float* x, uint32_t a, uint32_t b, float pad, float4& lo, float4& hi) {
  float l[3], h[3];
  for (int c = 0; c < 3; ++c) {
    float p = x[3 * a + c], q = x[3 * b + c];
    l[c] = __fsub_rn(fminf(p, q), pad);
    h[c] = __fadd_rn(fmaxf(p, q), pad);
  }
  lo = make_float4(l[0], l[1], l[2], 0.f);
  hi = make_float4(h[0], h[1], h[2], 0.f);
}

// Side streams: the work enqueued on them after aux_fork runs after everything on s.st so
// far, and s.st's work after aux_join runs after all of theirs.
static constexpr int N_AUX = 4;
static int aux_fork(Scene& s) {
  if (s.aux.empty()) {
    s.aux.resize(N_AUX);
    s.aux_ev.resize(N_AUX);
    for (int i = 0; i < N_AUX; ++i) {
      MG_CUDA(cudaStreamCreateWithFlags(&s.aux[i], cudaStreamNonBlocking));
      MG_CUDA(cudaEventCreateWithFlags(&s.aux_ev[i], cudaEventDisableTiming));
    }
    MG_CUDA(cudaEventCreateWithFlags(&s.fork_ev, cudaEventDisableTiming));
  }
  MG_CUDA(cudaEventRecord(s.fork_ev, s.st));
  for (int i = 0; i < N_AUX; ++i) MG_CUDA(cudaStreamWaitEvent(s.aux[i], s.fork_ev, 0));
  return MGUSO_OK;
}
static int aux_join(Scene& s) {
  for (int i = 0; i < N_AUX; ++i) {
    MG_CUDA(cudaEventRecord(s.aux_ev[i], s.aux[i]));
    MG_CUDA(cudaStreamWaitEvent(s.st, s.aux_ev[i], 0));
  }
  return MGUSO_OK;
}

// The instances' triangle and edge LBVHs at x, built concurrently on the side streams (each
// tree has its own scratch). With refit, a tree keeps the shape of its last build and gets
// its boxes at x (leaf boxes and one climb instead of bounds, keys, sort, Karras and climb):
// the traversals' leaf sets are defined by box overlap with exact node unions, so they are
// the same for any shape over the same primitives, and within a step the shape built at its
// first iterate stays a close fit.
int build_bvhs(Scene& s, const float* x, bool refit) {
  MG_TRY(aux_fork(s));
  int rc = MGUSO_OK;
  for (uint32_t k = 0; k < s.ninst && rc == MGUSO_OK; ++k) {
    if (!((s.iter_active >> k) & 1u)) continue;  // an instance the batch no longer iterates
    const uint32_t t0 = s.inst_tri[k], e0 = s.inst_edge[k];
    const uint32_t nt = s.inst_tri[k + 1] - t0, ne = s.inst_edge[k + 1] - e0;
    Lbvh* tb = s.tri_bvh[k].get();
    Lbvh* eb = s.edge_bvh[k].get();
    const uint32_t* tt = s.tris.p + 3 * (size_t)t0;
    const uint32_t* et = s.edge_tris.p + 3 * (size_t)e0;
    cudaStream_t ts = s.aux[(2 * k) % N_AUX], es = s.aux[(2 * k + 1) % N_AUX];
    rc = (refit && tb->shaped && tb->nt == nt) ? lbvh_refit_pos(tb, x, tt, ts) : lbvh_build(tb, x, s.nv, tt, nt, 30, ts);
    if (rc == MGUSO_OK)
      rc = (refit && eb->shaped && eb->nt == ne) ? lbvh_refit_pos(eb, x, et, es) : lbvh_build(eb, x, s.nv, et, ne, 30, es);
  }
  MG_TRY(aux_join(s));
  return rc;
}

// ---- self intersection (has_self_intersection, implicit.rs:618-650) ------------------
// edge_triangle_intersect (contact.rs:324-352) in FP32, in the reference's operation order
// (this file is compiled without FMA contraction): the segment crosses the triangle's plane
// strictly and the crossing point's barycentric coordinates are inside or on the boundary.
__device__ __forceinline__ bool edge_triangle_intersect_f(V3<float> e0, V3<float> e1, V3<float> v0, V3<float> v1,
                                                          V3<float> v2) {
  const V3<float> d1 = v1 - v0, d2 = v2 - v0, a0 = e0 - v0, a1 = e1 - v0;
  const V3<float> n = d1.cross(d2);
  const float s1 = a0.dot(n), s2 = a1.dot(n);
  if (!(s1 * s2 < 0.f)) return false;
  const float t = s1 / (s1 - s2);
  const V3<float> r = a0 * (1.f - t) + a1 * t;
  const float a = d1.dot(d1), b = d1.dot(d2), c = d2.dot(d2);
  const float det = a * c - b * b;
  if (det == 0.f) return false;
  const float p = d1.dot(r), q = d2.dot(r);
  const float u = (c * p - b * q) / det, v = (a * q - b * p) / det;
  return u >= 0.f && v >= 0.f && u + v <= 1.f;
}

// Every mesh edge against the triangles whose boxes overlap its own box (every piercing
// pair is among them): pairs with a movable vertex that share no vertex, counted per
// instance into red[RED_STRIDE k + 14].
__global__ void k_self_intersect(BvhSet bv, const uint8_t* __restrict__ vinst, const float* __restrict__ x,
                                 const uint32_t* __restrict__ edges, const uint32_t* __restrict__ tris,
                                 const float* __restrict__ im, uint32_t ne, unsigned int* __restrict__ red,
                                 uint32_t* status) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ne) return;
  const uint32_t e0 = edges[2 * j], e1 = edges[2 * j + 1];
  float4 lo, hi;
  edge_box(x, e0, e1, 0.f, lo, hi);
  const bool emov = im[e0] > 0.f || im[e1] > 0.f;
  const V3<float> p0 = ld3<float>(x, e0), p1 = ld3<float>(x, e1);
  unsigned int hits = 0;
  const bool ok = visit(bv, vinst[e0], lo, hi, [&](uint32_t t) {
    const uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
    if (!emov && !(im[a] > 0.f || im[b] > 0.f || im[c] > 0.f)) return;
    if (e0 == a || e0 == b || e0 == c || e1 == a || e1 == b || e1 == c) return;
    if (edge_triangle_intersect_f(p0, p1, ld3<float>(x, a), ld3<float>(x, b), ld3<float>(x, c))) ++hits;
  });
  if (!ok) atomicOr(status, ST_STACK_OVERFLOW);
  if (hits) atomicAdd(red + RED_STRIDE * vinst[e0] + 14, hits);
}

// Piercing (edge, triangle) pairs of every instance at the scene's positions x, counted into
// red[RED_STRIDE k + 14] (which the caller zeroes); rebuilds the triangle BVHs at x.
int self_intersections(Scene& s, bool refit) {
  if (s.n_edge == 0) return MGUSO_OK;
  MG_TRY(aux_fork(s));
  int rc = MGUSO_OK;
  for (uint32_t k = 0; k < s.ninst && rc == MGUSO_OK; ++k) {
    const uint32_t t0 = s.inst_tri[k], nt = s.inst_tri[k + 1] - t0;
    Lbvh* tb = s.tri_bvh[k].get();
    const uint32_t* tt = s.tris.p + 3 * (size_t)t0;
    rc = (refit && tb->shaped && tb->nt == nt) ? lbvh_refit_pos(tb, s.x.p, tt, s.aux[k % N_AUX])
                                 : lbvh_build(tb, s.x.p, s.nv, tt, nt, 30, s.aux[k % N_AUX]);
  }
  MG_TRY(aux_join(s));
  MG_TRY(rc);
  BvhSet tv = view_set(s.tri_bvh, s.inst_tri);
  k_self_intersect<<<ceil_div(s.n_edge, 128), 128, 0, s.st>>>(tv, s.vinst.p, s.x.p, s.edges.p, s.tris.p, s.inv_mass.p,
                                                             s.n_edge, s.red.p, s.status.p);
  MG_CUDA(cudaGetLastError());
  return MGUSO_OK;
}

// ---- collider sides ------------------------------------------------------------------
// best (d2 bits, triangle) per non-static vertex over collider triangles within dhat; ties
// go to the lowest triangle index, which is the first one the reference's triangle-major
// visit reaches.
__global__ void k_side_best(BvhSet bv, const uint8_t* __restrict__ vinst, const float* __restrict__ x, const uint32_t* __restrict__ tris,
                            const uint8_t* __restrict__ ctri, const uint8_t* __restrict__ svert,
                            const float* __restrict__ im, const uint32_t* __restrict__ ex_ptr,
                            const uint32_t* __restrict__ ex_list, uint32_t nv, float dhat,
                            unsigned long long* __restrict__ best, uint32_t* __restrict__ status, uint32_t active) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv || !((active >> vinst[v]) & 1u)) return;
  unsigned long long b = ~0ull;
  if (!svert[v] && im[v] > 0.f) {
    float4 lo, hi;
    point_box(x, v, dhat, lo, hi);
    V3<float> p = ld3<float>(x, v);
    bool ok = visit(bv, vinst[v], lo, hi, [&](uint32_t t) {
      if (!ctri[t]) return;
      uint32_t a = tris[3 * t], bb = tris[3 * t + 1], c = tris[3 * t + 2];
      if (excluded(ex_ptr, ex_list, v, a, bb, c)) return;
      float w[3];
      V3<float> q = closest_point_bary(p, ld3<float>(x, a), ld3<float>(x, bb), ld3<float>(x, c), w);
      float d2 = (p - q).length_squared();
      unsigned long long k = ((unsigned long long)__float_as_uint(d2) << 32) | t;
      if (k < b) b = k;
    });
    if (!ok) atomicOr(status, ST_STACK_OVERFLOW);
  }
  best[v] = b;
}

__device__ __forceinline__ float side_of(uint32_t v, const unsigned long long* best, const float* x,
                                         const uint32_t* tris, const float* pn, float dhat) {
  unsigned long long b = best[v];
  if (b == ~0ull) return 1.f;
  float d2 = __uint_as_float((uint32_t)(b >> 32));
  if (d2 >= dhat * dhat) return 1.f;
  uint32_t t = (uint32_t)b;
  uint32_t ia = tris[3 * t], ib = tris[3 * t + 1], ic = tris[3 * t + 2];
  V3<float> a = ld3<float>(x, ia), bb = ld3<float>(x, ib), c = ld3<float>(x, ic), p = ld3<float>(x, v);
  float l[3];
  V3<float> q = closest_point_bary(p, a, bb, c, l);
  V3<float> e = p - q;
  V3<float> pnv[3] = {ld3<float>(pn, ia), ld3<float>(pn, ib), ld3<float>(pn, ic)};
  V3<float> n = surface_normal_at(l, (bb - a).cross(c - a).normalize_or_zero(), pnv);
  return e.dot(n) < 0.f ? -1.f : 1.f;
}

// ---- stencils ------------------------------------------------------------------------------
__device__ __forceinline__ void emit_stencil(Stencil* out, unsigned long long* keys, uint32_t* ids,
                                             unsigned long long* counter, uint32_t cap, uint32_t* status,
                                             uint32_t kind, uint32_t pa, uint32_t pb, const uint32_t idx[4], double d,
                                             double ghat, const double g[12]) {
  unsigned long long at = atomicAdd(counter, 1ull);
  if (at >= cap) {
    atomicOr(status, ST_CAPACITY);
    return;
  }
  Stencil& S = out[at];
  for (int k = 0; k < 4; ++k) S.idx[k] = idx[k];
  S.kind = kind;
  S.pad = 0;
  S.d = d;
  S.ghat = ghat;
  for (int k = 0; k < 12; ++k) S.g[k] = g[k];
  keys[at] = ((unsigned long long)kind << 62) | ((unsigned long long)pa << 31) | pb;
  ids[at] = (uint32_t)at;
}

// ---- warp-pooled narrow phase ---------------------------------------------------------------
// Each lane walks its query's tree (BoxWalk, CcdWalk) and pushes the leaves it reaches, as
// (query, primitive) pairs, onto its warp's queue in shared memory; whenever 32 are queued the
// whole warp takes them, one per lane, through the remaining filters and the narrow phase
// (distances, accd_toi). The walks stay per lane, but the narrow phase (the bulk of the work)
// runs on full warps instead of on the few lanes whose walk happens to sit on a leaf. Its
// results are order-free: stencils are sorted by their pair key afterwards, CCD results are
// per (instance, pass) minima and sums.
constexpr int WQ_WARPS = 4;   // 128-thread blocks
constexpr int WQ_QCAP = 96;   // < 32 left over + 2 leaves per lane and step

__device__ __forceinline__ void wq_push(uint2* q, int& n, bool has, uint2 e) {
  const unsigned m = __ballot_sync(0xffffffffu, has);
  if (has) q[n + __popc(m & ((1u << (threadIdx.x & 31)) - 1u))] = e;
  n += __popc(m);
}

// Takes batches of up to 32 queued pairs while at least min_n are queued (n is warp-uniform).
template <class F>
__device__ __forceinline__ void wq_take(uint2* q, int& n, int min_n, F&& solve) {
  const int lane = (int)(threadIdx.x & 31);
  __syncwarp();
  while (n >= min_n && n > 0) {
    const int take = n < 32 ? n : 32;
    const bool has = lane < take;
    const uint2 e = has ? q[n - take + lane] : make_uint2(0u, 0u);
    __syncwarp();
    n -= take;
    if (has) solve(e);
  }
}

template <class R>
__device__ __forceinline__ R vt_distance(const float* x, const uint32_t idx[4], bool collider, bool inside, R g[12]) {
  V3<R> gg[4];
  R d = point_tri_distance_grad<R>(ld3<R>(x, idx[0]), ld3<R>(x, idx[1]), ld3<R>(x, idx[2]), ld3<R>(x, idx[3]),
                                   collider && inside, gg);
  for (int a = 0; a < 4; ++a)
    for (int c = 0; c < 3; ++c) g[3 * a + c] = gg[a][c];
  return d;
}

template <class R>
__device__ __forceinline__ R ee_distance(const float* x, const uint32_t idx[4], R g[12]) {
  V3<R> gg[4];
  R d = segment_segment_distance_grad<R>(ld3<R>(x, idx[0]), ld3<R>(x, idx[1]), ld3<R>(x, idx[2]), ld3<R>(x, idx[3]),
                                         gg);
  for (int a = 0; a < 4; ++a)
    for (int c = 0; c < 3; ++c) g[3 * a + c] = gg[a][c];
  return d;
}

// Vertex-triangle pairs: lane v walks the triangles near vertex v; the distances run pooled
// per warp. A static collider triangle needs v's side of the collider, which depends on v
// alone (side_of), so the lane that takes the pair evaluates it.
__global__ void __launch_bounds__(WQ_WARPS * 32) k_vt_stencils(
    BvhSet bv, const uint8_t* __restrict__ vinst, const float* __restrict__ x, const uint32_t* __restrict__ tris,
    const uint8_t* __restrict__ ctri, const float* __restrict__ im, const uint32_t* __restrict__ ex_ptr,
    const uint32_t* __restrict__ ex_list, const unsigned long long* __restrict__ best, const float* __restrict__ pn,
    int has_static, uint32_t nv, float dhat, int mixed, Stencil* out, unsigned long long* keys, uint32_t* ids,
    unsigned long long* counter, uint32_t cap, uint32_t* status, uint32_t active) {
  __shared__ uint2 qbuf[WQ_WARPS][WQ_QCAP];
  uint2* q = qbuf[threadIdx.x >> 5];
  int qn = 0;
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t base = 0;
  bool done = true;
  BoxWalk walk;
  walk.ok = true;
  uint32_t outp[2];
  int nout = 0;
  if (v < nv) {
    const uint32_t k = vinst[v];
    if ((active >> k) & 1u) {
      const BvhView& tv = bv.t[k];
      base = bv.base[k];
      walk.left = tv.left;
      walk.right = tv.right;
      walk.prim = tv.prim;
      walk.node = tv.node;
      walk.leaf = tv.leaf;
      walk.cbox = tv.cbox;
      walk.nt = tv.n;
      point_box(x, v, dhat, walk.qlo, walk.qhi);
      nout = walk.start(done, outp);
    }
  }
  auto solve = [&](uint2 e) {
    const uint32_t qv = e.x, t = e.y;
    const uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
    if (!(im[qv] > 0.f || im[a] > 0.f || im[b] > 0.f || im[c] > 0.f)) return;
    if (excluded(ex_ptr, ex_list, qv, a, b, c)) return;
    uint32_t idx[4] = {qv, a, b, c};
    const bool collider = has_static && ctri[t];
    const bool inside = collider && side_of(qv, best, x, tris, pn, dhat) < 0.f;
    double g[12];
    float gf[12];
    float df = vt_distance<float>(x, idx, collider, inside, gf);
    double d = df;
    for (int cc = 0; cc < 12; ++cc) g[cc] = gf[cc];
    if (mixed && df < 10.f * dhat) d = vt_distance<double>(x, idx, collider, inside, g);
    if (!(d < (double)dhat)) return;
    emit_stencil(out, keys, ids, counter, cap, status, 0, qv, t, idx, d, dhat, g);
  };
  for (;;) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const bool leaf = c < nout;
      wq_push(q, qn, leaf, make_uint2(v, leaf ? base + outp[c] : 0u));
    }
    wq_take(q, qn, 32, solve);
    if (!__any_sync(0xffffffffu, !done)) break;
    nout = done ? 0 : walk.step(done, outp);
  }
  wq_take(q, qn, 1, solve);
  if (!walk.ok) atomicOr(status, ST_STACK_OVERFLOW);
}

// Edge-edge pairs: lane t (edge t) takes the pairs (t, p) with p > t, the lower-indexed edge
// first in the stencil and its key, so each pair is seen once. An edge in its instance's static
// tail (every edge from there on has both vertices pinned) has no partner above it that can
// move, and skips its walk. The distances run pooled per warp.
__global__ void __launch_bounds__(WQ_WARPS * 32) k_ee_stencils(
    BvhSet bv, const uint8_t* __restrict__ vinst, const float* __restrict__ x, const uint32_t* __restrict__ edges,
    const uint32_t* __restrict__ ee_tail, const float* __restrict__ im, uint32_t ne, float search, float dhat,
    int mixed, Stencil* out, unsigned long long* keys, uint32_t* ids, unsigned long long* counter, uint32_t cap,
    uint32_t* status, uint32_t active) {
  __shared__ uint2 qbuf[WQ_WARPS][WQ_QCAP];
  uint2* q = qbuf[threadIdx.x >> 5];
  int qn = 0;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t base = 0;
  bool done = true;
  BoxWalk walk;
  walk.ok = true;
  uint32_t outp[2];
  int nout = 0;
  if (t < ne) {
    const uint32_t b0 = edges[2 * t], b1 = edges[2 * t + 1];
    const uint32_t k = vinst[b0];
    if (t < ee_tail[k] && ((active >> k) & 1u)) {
      const BvhView& tv = bv.t[k];
      base = bv.base[k];
      walk.left = tv.left;
      walk.right = tv.right;
      walk.prim = tv.prim;
      walk.node = tv.node;
      walk.leaf = tv.leaf;
      walk.cbox = tv.cbox;
      walk.nt = tv.n;
      edge_box(x, b0, b1, search, walk.qlo, walk.qhi);
      nout = walk.start(done, outp);
    }
  }
  auto solve = [&](uint2 e) {
    const uint32_t qt = e.x, p = e.y;
    const uint32_t b0 = edges[2 * qt], b1 = edges[2 * qt + 1], a0 = edges[2 * p], a1 = edges[2 * p + 1];
    if (!(im[b0] > 0.f || im[b1] > 0.f || im[a0] > 0.f || im[a1] > 0.f)) return;
    if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) return;
    uint32_t idx[4] = {b0, b1, a0, a1};
    double g[12];
    float gf[12];
    float df = ee_distance<float>(x, idx, gf);
    double d = df;
    for (int c = 0; c < 12; ++c) g[c] = gf[c];
    if (mixed && df < 10.f * dhat) d = ee_distance<double>(x, idx, g);
    double ghat = (double)(0.5f * (dhat + dhat));
    if (!(d < ghat)) return;
    emit_stencil(out, keys, ids, counter, cap, status, 1, qt, p, idx, d, ghat, g);
  };
  for (;;) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const bool leaf = c < nout;
      const uint32_t p = leaf ? base + outp[c] : 0u;
      wq_push(q, qn, leaf && p > t, make_uint2(t, p));
    }
    wq_take(q, qn, 32, solve);
    if (!__any_sync(0xffffffffu, !done)) break;
    nout = done ? 0 : walk.step(done, outp);
  }
  wq_take(q, qn, 1, solve);
  if (!walk.ok) atomicOr(status, ST_STACK_OVERFLOW);
}

__global__ void k_permute_stencils(const Stencil* __restrict__ in, const uint32_t* __restrict__ ids, uint32_t n,
                                   Stencil* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[ids[i]];
}

int collect_stencils(Scene& s, uint32_t* nst_out) {
  cudaStream_t st = s.st;
  const float dhat = s.p.contact_dhat;
  const BvhSet tv = view_set(s.tri_bvh, s.inst_tri), ev = view_set(s.edge_bvh, s.inst_edge);
  if (s.has_static) {
    k_side_best<<<ceil_div(s.nv, 128), 128, 0, st>>>(tv, s.vinst.p, s.x.p, s.tris.p, s.collider_tri.p, s.static_vert.p,
                                                   s.inv_mass.p, s.ex_ptr.p, s.ex_list.p, s.nv, dhat, s.side_best.p,
                                                   s.status.p, s.iter_active);
  }
  for (int attempt = 0; attempt < 4; ++attempt) {
    MG_TRY(s.stencils.reserve(s.cap_stencils));
    MG_TRY(s.stencils_sorted.reserve(s.cap_stencils));
    MG_TRY(s.st_keys.reserve(s.cap_stencils));
    MG_TRY(s.st_ids.reserve(s.cap_stencils));
    MG_CUDA(cudaMemsetAsync(s.counters.p, 0, 8 * 8, st));
    // the two kinds run concurrently on side streams (they share the output through its
    // atomic counter; the stencils are put in key order below)
    MG_TRY(aux_fork(s));
    k_vt_stencils<<<ceil_div(s.nv, 128), 128, 0, s.aux[0]>>>(
        tv, s.vinst.p, s.x.p, s.tris.p, s.collider_tri.p, s.inv_mass.p, s.ex_ptr.p, s.ex_list.p, s.side_best.p,
        s.collider_pn.p, s.has_static ? 1 : 0, s.nv, dhat, s.mixed ? 1 : 0, s.stencils.p, s.st_keys.p, s.st_ids.p,
        s.counters.p, s.cap_stencils, s.status.p, s.iter_active);
    if (s.n_edge)
      k_ee_stencils<<<ceil_div(s.n_edge, 128), 128, 0, s.aux[1]>>>(
          ev, s.vinst.p, s.x.p, s.edges.p, s.ee_tail.p, s.inv_mass.p, s.n_edge, dhat, dhat, s.mixed ? 1 : 0,
          s.stencils.p, s.st_keys.p, s.st_ids.p, s.counters.p, s.cap_stencils, s.status.p, s.iter_active);
    MG_CUDA(cudaGetLastError());
    MG_TRY(aux_join(s));
    unsigned long long cnt = 0;
    MG_CUDA(cudaMemcpyAsync(&cnt, s.counters.p, 8, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    if (cnt <= s.cap_stencils) {
      uint32_t n = (uint32_t)cnt;
      if (n > 1) MG_TRY(radix_sort_pairs(&s.sorter, s.st_keys.p, s.st_ids.p, n, 64, st));
      if (n) k_permute_stencils<<<ceil_div(n, 128), 128, 0, st>>>(s.stencils.p, s.st_ids.p, n, s.stencils_sorted.p);
      MG_CUDA(cudaGetLastError());
      *nst_out = n;
      return MGUSO_OK;
    }
    s.cap_stencils = (uint32_t)std::min<unsigned long long>(2 * cnt + 1024, 1ull << 28);
    MG_CUDA(cudaMemsetAsync(s.status.p, 0, 4, st));  // clear the capacity flag and retry
  }
  set_error("stencil buffer growth did not converge");
  return MGUSO_ERR_PAIR_OVERFLOW;
}

// ---- CCD -----------------------------------------------------------------------------------
__device__ __forceinline__ void atomic_min_pos(unsigned int* addr, float v) {
  atomicMin(addr, __float_as_uint(fmaxf(v, 0.f)));
}

// per-instance maximum of |dx_v| into out[RED_STRIDE * instance]
__global__ void k_max_norm(const float* __restrict__ dx, const uint8_t* __restrict__ vinst, uint32_t nv,
                           unsigned int* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const float m = ld3<float>(dx, i).length();
    if (m > 0.f) atomicMax(out + RED_STRIDE * vinst[i], __float_as_uint(m));
  }
}

// analytic colliders: keep >= 20% of the current gap (implicit.rs:1795-1818)
__global__ void k_ccd_colliders(const uint32_t* __restrict__ free_verts, uint32_t n_free, const uint8_t* __restrict__ vinst,
                                const float* __restrict__ x, const float* __restrict__ dx, const float* __restrict__ cols,
                                uint32_t ncol, unsigned int* __restrict__ red) {
  uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_free) return;
  uint32_t i = free_verts[f];
  V3<float> xi = ld3<float>(x, i), di = ld3<float>(dx, i);
  const float GAP = 0.2f;
  float t = 1.f;
  for (uint32_t c = 0; c < ncol; ++c) {
    const float* cc = cols + 8 * c;
    V3<float> a(cc[1], cc[2], cc[3]);
    float d0;
    V3<float> n;
    if (cc[0] == 0.f) {
      n = V3<float>(cc[4], cc[5], cc[6]);
      d0 = (xi - a).dot(n);
    } else {
      V3<float> v = xi - a;
      float l = v.length();
      if (l < 1e-9f) {
        d0 = -cc[7];
      } else {
        d0 = l - cc[7];
        n = v / l;
      }
    }
    if (d0 <= 0.f) continue;
    if (cc[0] == 0.f) {
      float rate = di.dot(n);
      if (rate < 0.f) t = fminf(t, (GAP - 1.0f) * d0 / rate);
    } else {
      float l = di.length();
      if (l > 1e-12f) t = fminf(t, (1.0f - GAP) * d0 / l);
    }
  }
  if (t < 1.f) atomic_min_pos(red + RED_STRIDE * vinst[i] + 1, t);
}

// static pins: the radius interpolated linearly over the extended horizon 1.25 dx, clamped
// to land on the pin's ghat sphere (implicit.rs:1755-1789)
__global__ void k_ccd_pins(const uint32_t* __restrict__ pin_vert, uint32_t n_pin, const uint8_t* __restrict__ pin_kin,
                           const float* __restrict__ pin_target, const float* __restrict__ pin_ghat,
                           const float* __restrict__ im, const uint8_t* __restrict__ vinst, const float* __restrict__ x,
                           const float* __restrict__ dx, unsigned int* __restrict__ red) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_pin || pin_kin[p]) return;
  const uint32_t i = pin_vert[p];
  if (!(im[i] > 0.f)) return;
  const float LS_MAX_T = 1.25f;
  const V3<float> tg = ld3<float>(pin_target, p);
  const float gh = pin_ghat[p];
  const float r0 = (ld3<float>(x, i) - tg).length();
  if (r0 >= gh) return;
  const float r1 = (ld3<float>(x, i) + ld3<float>(dx, i) * LS_MAX_T - tg).length();
  if (r1 > gh) {
    const float denom = r1 - r0;
    if (denom != 0.f) {
      const float t = LS_MAX_T * (gh - r0) / denom;
      if (t < 1.f) atomic_min_pos(red + RED_STRIDE * vinst[i] + 1, fmaxf(t, 0.f));
    }
  }
}

// Strain-limit line search (implicit.rs:1709-1753): per face, bisect the step fraction on
// max(sigma(x + t dx) - 1) < limit over [0, 1.25] until the bisection window stops
// shrinking (at most 64 halvings); a face already inside its limit at 1.25 does not limit.
__global__ void k_ccd_sl(uint32_t n, const uint32_t* __restrict__ fv, const float* __restrict__ fdm,
                         const float* __restrict__ flim, const uint8_t* __restrict__ vinst,
                         const float* __restrict__ x, const float* __restrict__ dx, unsigned int* __restrict__ red) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  const float LS_MAX_T = 1.25f;
  const M2<float> dm{fdm[4 * f], fdm[4 * f + 1], fdm[4 * f + 2], fdm[4 * f + 3]};
  const float limit = flim[f];
  V3<float> x0[3], d0[3];
  for (int a = 0; a < 3; ++a) {
    x0[a] = ld3<float>(x, fv[3 * f + a]);
    d0[a] = ld3<float>(dx, fv[3 * f + a]);
  }
  auto at = [&](float frac) {
    V3<float> p[3] = {x0[0] + d0[0] * frac, x0[1] + d0[1] * frac, x0[2] + d0[2] * frac};
    return max_stretch_excess<float>(p, dm);
  };
  if (at(LS_MAX_T) < limit) return;
  float lo = 0.f, hi = LS_MAX_T, window = hi - lo;
  for (int it = 0; it < 64; ++it) {
    const float mid = 0.5f * (lo + hi);
    if (at(mid) - limit < 0.f)
      lo = mid;
    else
      hi = mid;
    const float w = hi - lo;
    if (w == window) break;
    window = w;
  }
  if (lo < 1.f) atomic_min_pos(red + RED_STRIDE * vinst[fv[3 * f]] + 1, lo);
}

// CCD candidate pruning: a pair whose accd_toi (contact.rs:378-437) would return max_t at
// its first test cannot lower the step fraction, and traversal skips whole subtrees of such
// pairs (CcdWalk) from the primitives' displacement boxes, refitted per CCD call.

// Per-instance CCD passes of one launch: up to CCD_CHUNK consecutive search radii of the
// widening schedule (ascending). The traversal uses the largest; each candidate pair's ACCD
// result then counts for every pass whose search box reaches it (the box test of that pass
// alone), so one launch yields each pass's step fraction and cap count exactly as separate
// passes would. Instances whose fraction an earlier launch settled are skipped.
constexpr int CCD_CHUNK = 6;
struct CcdPass {
  float search[PCG_MAX_INST][CCD_CHUNK];
  uint32_t npass[PCG_MAX_INST];
  uint32_t todo;  // bit k: instance k
};

// per (instance, pass) accumulators: [0] step fraction (float bits, atomic min), [1] caps
__device__ __forceinline__ unsigned int* ccd_slot(unsigned int* acc, uint32_t k, int i) {
  return acc + 2 * (CCD_CHUNK * k + i);
}

// The first pass (index into the chunk) whose query box overlaps the primitive's box
// [plo, phi]; the query box of pass i is built as the traversal builds its own.
__device__ __forceinline__ int first_pass_point(const CcdPass& cp, uint32_t k, const float* x, uint32_t v,
                                                const float plo[3], const float phi[3]) {
  const int n = (int)cp.npass[k];
  for (int i = 0; i < n; ++i) {
    float4 lo, hi;
    point_box(x, v, cp.search[k][i], lo, hi);
    if (lo.x <= phi[0] && lo.y <= phi[1] && lo.z <= phi[2] && plo[0] <= hi.x && plo[1] <= hi.y && plo[2] <= hi.z)
      return i;
  }
  return n;
}
__device__ __forceinline__ int first_pass_edge(const CcdPass& cp, uint32_t k, const float* x, uint32_t a,
                                               uint32_t b, const float plo[3], const float phi[3]) {
  const int n = (int)cp.npass[k];
  for (int i = 0; i < n; ++i) {
    float4 lo, hi;
    edge_box(x, a, b, cp.search[k][i], lo, hi);
    if (lo.x <= phi[0] && lo.y <= phi[1] && lo.z <= phi[2] && plo[0] <= hi.x && plo[1] <= hi.y && plo[2] <= hi.z)
      return i;
  }
  return n;
}

// A lane's step fractions and cap counts per pass for one instance at a time, flushed to the
// per (instance, pass) accumulators when the instance changes and at the end.
struct CcdAcc {
  uint32_t k;
  float t[CCD_CHUNK];
  uint32_t cap[CCD_CHUNK];
  uint32_t solves;
  __device__ __forceinline__ void reset(uint32_t kk) {
    k = kk;
    solves = 0;
#pragma unroll
    for (int i = 0; i < CCD_CHUNK; ++i) {
      t[i] = 1.f;
      cap[i] = 0;
    }
  }
  __device__ __forceinline__ void flush(const CcdPass& cp, unsigned int* acc, unsigned int* red, int solve_slot) {
    if (k == 0xffffffffu) return;
    const int np = (int)cp.npass[k];
#pragma unroll
    for (int i = 0; i < CCD_CHUNK; ++i) {
      if (i < np && t[i] < 1.f) atomic_min_pos(ccd_slot(acc, k, i), t[i]);
      if (i < np && cap[i]) atomicAdd(ccd_slot(acc, k, i) + 1, cap[i]);
    }
    if (solves) atomicAdd(red + RED_STRIDE * k + solve_slot, solves);
  }
  __device__ __forceinline__ void add(uint32_t kk, int i0, float tt, bool capped, const CcdPass& cp,
                                      unsigned int* acc, unsigned int* red, int solve_slot) {
    if (kk != k) {
      flush(cp, acc, red, solve_slot);
      reset(kk);
    }
    ++solves;
#pragma unroll
    for (int i = 0; i < CCD_CHUNK; ++i)
      if (i >= i0) {
        t[i] = fminf(t[i], tt);
        cap[i] += capped ? 1u : 0u;
      }
  }
};

__device__ __forceinline__ void walk_init(CcdWalk& w, const BvhSet& bs, uint32_t k, float4 lo, float4 hi, float4 qlo,
                                          float4 qhi, float3 cq, float rq) {
  const BvhView& bv = bs.t[k];
  w.left = bv.left;
  w.right = bv.right;
  w.prim = bv.prim;
  w.node = bv.node;
  w.leaf = bv.leaf;
  w.dnode = bv.dnode;
  w.dleaf = bv.dleaf;
  w.cbox = bv.cbox;
  w.dcbox = bv.dcbox;
  w.nt = bv.n;
  w.slo = lo;
  w.shi = hi;
  w.qlo = qlo;
  w.qhi = qhi;
  w.cq = cq;
  w.rq = rq;
}

// Vertex-triangle passes: lane v walks the triangles near vertex v.
template <class R>
__global__ void __launch_bounds__(WQ_WARPS * 32, 4) k_ccd_vt(
    BvhSet bv, const CcdPass* __restrict__ cpp, const uint8_t* __restrict__ vinst, const float* __restrict__ x,
    const float* __restrict__ dx, const uint32_t* __restrict__ tris, const uint8_t* __restrict__ ctri,
    const float* __restrict__ im, const uint32_t* __restrict__ ex_ptr, const uint32_t* __restrict__ ex_list,
    const unsigned long long* __restrict__ best, const float* __restrict__ pn, int has_static, uint32_t nv, float dhat,
    uint32_t max_iter, unsigned int* __restrict__ red, unsigned int* __restrict__ acc, uint32_t* __restrict__ status) {
  __shared__ uint2 qbuf[WQ_WARPS][WQ_QCAP];
  uint2* q = qbuf[threadIdx.x >> 5];
  int qn = 0;
  const CcdPass& cp = *cpp;
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t k = 0xffffffffu, base = 0, nleaf = 0;
  bool done = true;
  float side = 2.f;
  CcdWalk walk;
  walk.ok = true;
  uint32_t out[2];
  int nout = 0;
  if (v < nv) {
    const uint32_t kv = vinst[v];
    if ((cp.todo >> kv) & 1u) {
      k = kv;
      base = bv.base[k];
      float4 lo, hi, qlo, qhi;
      point_box(x, v, cp.search[k][cp.npass[k] - 1], lo, hi);
      point_box(x, v, 0.f, qlo, qhi);
      walk_init(walk, bv, k, lo, hi, qlo, qhi, make_float3(dx[3 * v], dx[3 * v + 1], dx[3 * v + 2]), 0.f);
      nout = walk.start(done, out);
    }
  }
  CcdAcc a;
  a.reset(0xffffffffu);
  auto solve = [&](uint2 e) {
    const uint32_t qv = e.x, t = e.y, kq = vinst[qv];
    const uint32_t ta = tris[3 * t], tb = tris[3 * t + 1], tc = tris[3 * t + 2];
    if (!(im[qv] > 0.f || im[ta] > 0.f || im[tb] > 0.f || im[tc] > 0.f)) return;
    if (excluded(ex_ptr, ex_list, qv, ta, tb, tc)) return;
    float plo[3], phi[3];
    for (int c = 0; c < 3; ++c) {
      const float pa = x[3 * ta + c], pb = x[3 * tb + c], pc = x[3 * tc + c];
      plo[c] = fminf(fminf(pa, pb), pc);
      phi[c] = fmaxf(fmaxf(pa, pb), pc);
    }
    const int i0 = first_pass_point(cp, kq, x, qv, plo, phi);
    if (i0 >= (int)cp.npass[kq]) return;
    const uint32_t idx[4] = {qv, ta, tb, tc};
    V3<R> x0[4], dd[4];
    for (int c = 0; c < 4; ++c) {
      x0[c] = ld3<R>(x, idx[c]);
      dd[c] = ld3<R>(dx, idx[c]);
    }
    bool capped = false;
    const R toi = accd_toi<R>(x0, dd, R(0), R(1.25), R(0.01), max_iter, 0, &capped);
    a.add(kq, i0, (float)(toi / R(1.25)), capped, cp, acc, red, 6);
  };
  for (;;) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      bool has = c < nout;
      const uint32_t t = has ? base + out[c] : 0u;
      if (has) {
        ++nleaf;
        // a collider triangle only counts on the vertex's outer side (lazily, once per vertex)
        if (has_static && ctri[t]) {
          if (side == 2.f) side = side_of(v, best, x, tris, pn, dhat);
          if (side < 0.f) has = false;
        }
      }
      wq_push(q, qn, has, make_uint2(v, t));
    }
    wq_take(q, qn, 32, solve);
    if (!__any_sync(0xffffffffu, !done)) break;
    nout = done ? 0 : walk.step(done, out);
  }
  wq_take(q, qn, 1, solve);
  a.flush(cp, acc, red, 6);
  if (!walk.ok) atomicOr(status, ST_STACK_OVERFLOW);
  if (nleaf) atomicAdd(red + RED_STRIDE * k + 5, nleaf);
}

// Edge-edge passes. As k_ee_stencils: lane j takes the pairs (j, i) with i > j (the
// lower-indexed edge first), and an edge of its instance's static tail skips its walk.
template <class R>
__global__ void __launch_bounds__(WQ_WARPS * 32, 4) k_ccd_ee(
    BvhSet bv, const CcdPass* __restrict__ cpp, const uint8_t* __restrict__ vinst, const float* __restrict__ x,
    const float* __restrict__ dx, const uint32_t* __restrict__ edges, const uint32_t* __restrict__ ee_tail,
    const float* __restrict__ im, uint32_t ne, uint32_t max_iter, unsigned int* __restrict__ red,
    unsigned int* __restrict__ acc, uint32_t* __restrict__ status) {
  __shared__ uint2 qbuf[WQ_WARPS][WQ_QCAP];
  uint2* q = qbuf[threadIdx.x >> 5];
  int qn = 0;
  const CcdPass& cp = *cpp;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t k = 0xffffffffu, base = 0, nleaf = 0;
  bool done = true;
  CcdWalk walk;
  walk.ok = true;
  uint32_t out[2];
  int nout = 0;
  if (j < ne) {
    const uint32_t b0 = edges[2 * j], b1 = edges[2 * j + 1];
    const uint32_t kj = vinst[b0];
    if (((cp.todo >> kj) & 1u) && j < ee_tail[kj]) {
      k = kj;
      base = bv.base[k];
      float4 lo, hi, qlo, qhi;
      edge_box(x, b0, b1, cp.search[k][cp.npass[k] - 1], lo, hi);
      edge_box(x, b0, b1, 0.f, qlo, qhi);
      // the query edge's displacements lie in the ball around their midpoint
      const float3 d0 = make_float3(dx[3 * b0], dx[3 * b0 + 1], dx[3 * b0 + 2]);
      const float3 d1 = make_float3(dx[3 * b1], dx[3 * b1 + 1], dx[3 * b1 + 2]);
      const float3 cq = make_float3(0.5f * (d0.x + d1.x), 0.5f * (d0.y + d1.y), 0.5f * (d0.z + d1.z));
      const float ex = d1.x - d0.x, ey = d1.y - d0.y, ez = d1.z - d0.z;
      const float rq = 0.5f * sqrtf(ex * ex + ey * ey + ez * ez) * 1.0001f;
      walk_init(walk, bv, k, lo, hi, qlo, qhi, cq, rq);
      nout = walk.start(done, out);
    }
  }
  CcdAcc a;
  a.reset(0xffffffffu);
  auto solve = [&](uint2 e) {
    const uint32_t qj = e.x, i = e.y;
    const uint32_t b0 = edges[2 * qj], b1 = edges[2 * qj + 1], a0 = edges[2 * i], a1 = edges[2 * i + 1];
    const uint32_t kq = vinst[b0];
    if (!(im[b0] > 0.f || im[b1] > 0.f || im[a0] > 0.f || im[a1] > 0.f)) return;
    if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) return;
    float plo[3], phi[3];
    for (int c = 0; c < 3; ++c) {
      const float pa = x[3 * a0 + c], pb = x[3 * a1 + c];
      plo[c] = fminf(pa, pb);
      phi[c] = fmaxf(pa, pb);
    }
    const int i0 = first_pass_edge(cp, kq, x, b0, b1, plo, phi);
    if (i0 >= (int)cp.npass[kq]) return;
    const uint32_t idx[4] = {b0, b1, a0, a1};
    V3<R> x0[4], dd[4];
    for (int c = 0; c < 4; ++c) {
      x0[c] = ld3<R>(x, idx[c]);
      dd[c] = ld3<R>(dx, idx[c]);
    }
    bool capped = false;
    const R toi = accd_toi<R>(x0, dd, R(0), R(1.25), R(0.01), max_iter, 1, &capped);
    a.add(kq, i0, (float)(toi / R(1.25)), capped, cp, acc, red, 8);
  };
  for (;;) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const bool leaf = c < nout;
      const uint32_t i = leaf ? base + out[c] : 0u;
      nleaf += leaf ? 1u : 0u;
      wq_push(q, qn, leaf && i > j, make_uint2(j, i));
    }
    wq_take(q, qn, 32, solve);
    if (!__any_sync(0xffffffffu, !done)) break;
    nout = done ? 0 : walk.step(done, out);
  }
  wq_take(q, qn, 1, solve);
  a.flush(cp, acc, red, 8);
  if (!walk.ok) atomicOr(status, ST_STACK_OVERFLOW);
  if (nleaf) atomicAdd(red + RED_STRIDE * k + 7, nleaf);
}

// ccd_max_step (implicit.rs:1690-1947) without strain limiting, per instance. The
// search direction is s.dx; per instance k, red[RED_STRIDE k + 0] = max |dx|, + 1 collider t,
// + 2 self t, + 3 caps. Instances outside `active` get t = 1 and no work. Each instance runs
// the reference's widening-radius schedule on its own displacement and edge length; a pass
// covers every instance that still needs one.
// ---- the CCD schedule on the device -----------------------------------------------------
// The widening search of ccd_max_step (implicit.rs:1829-1947) per instance: the first launch
// runs the schedule's first radius alone, each later one up to CCD_CHUNK further radii
// (allowed, 4 allowed, ... up to the instance's largest displacement, and no further than the
// first radius that the previous launch's fraction already settles: the traversal runs at the
// chunk's largest radius, so a chunk that overshot it would only search a larger box for a
// result the sequential schedule never looks at); an instance is settled by the first radius
// whose step fraction keeps every move inside it, or by the full radius.
// Plan, traversals and settle run as the body of a conditional while node, so the host never
// waits on the schedule; CcdState holds it all.
struct CcdState {
  CcdPass cp;  // the current launch's radii
  float sched[PCG_MAX_INST][CCD_CHUNK];
  float allowed[PCG_MAX_INST], max_disp[PCG_MAX_INST], half_len[PCG_MAX_INST];
  // the radius from which on a pass is sure to settle: t_i md <= r_i holds once r_i >= t md
  // for the fraction t of any smaller radius, since t_i only falls as the radius grows
  float reach[PCG_MAX_INST];
  float t[PCG_MAX_INST];  // step fraction per instance (0 for inactive ones)
  uint32_t caps[PCG_MAX_INST];
  uint32_t launch, todo;
};

__global__ void k_red_init(unsigned int* __restrict__ red, uint32_t K) {
  const uint32_t i = threadIdx.x;
  if (i >= RED_STRIDE * K) return;
  const uint32_t q = i % RED_STRIDE;
  red[i] = (q == 1 || q == 2) ? __float_as_uint(1.f) : 0u;
}

// Per instance: the step fraction the colliders, pins and strain limits allow (red + 1), the
// largest displacement (red + 0) and the first allowed radius; todo = the instances whose
// self contact is still to be checked.
__global__ void k_ccd_start(CcdState* __restrict__ cs, const unsigned int* __restrict__ red, uint32_t K,
                            uint32_t active, int self) {
  const uint32_t k = threadIdx.x;
  if (k < PCG_MAX_INST) {
    const bool on = k < K && ((active >> k) & 1u);
    const float md = k < K ? __uint_as_float(red[RED_STRIDE * k]) : 0.f;
    cs->max_disp[k] = md;
    cs->t[k] = on ? __uint_as_float(red[RED_STRIDE * k + 1]) : 0.f;
    cs->caps[k] = 0;
    cs->allowed[k] = fmaxf(fminf(cs->half_len[k], md), 1.0e-9f);
    cs->reach[k] = md;
  }
  if (k == 0) {
    cs->launch = 0;
    cs->todo = self ? active : 0u;
  }
}

// This launch's radii per undecided instance, and fresh accumulators.
__global__ void k_ccd_plan(CcdState* __restrict__ cs, unsigned int* __restrict__ acc, float fixed) {
  const uint32_t k = threadIdx.x;
  if (k < PCG_MAX_INST * CCD_CHUNK) {
    acc[2 * k] = __float_as_uint(1.f);
    acc[2 * k + 1] = 0u;
  }
  if (k >= PCG_MAX_INST) return;
  if (k == 0) cs->cp.todo = cs->todo;
  if (!((cs->todo >> k) & 1u)) {
    cs->cp.npass[k] = 0;
    return;
  }
  const float md = cs->max_disp[k];
  float a = cs->allowed[k];
  uint32_t n = 0;
  for (;;) {
    cs->sched[k][n] = a;
    cs->cp.search[k][n] = fixed + 2.0f * a;
    ++n;
    if (cs->launch == 0 || n == (uint32_t)CCD_CHUNK || a >= md || a >= cs->reach[k]) break;
    a = fminf(a * 4.0f, md);
  }
  cs->cp.npass[k] = n;
}

// Settles every instance whose launch decided it, widens the others, and sets the loop's
// condition: go on while an instance is undecided, for at most 64 launches.
__global__ void k_ccd_settle(CcdState* __restrict__ cs, const unsigned int* __restrict__ acc,
                             cudaGraphConditionalHandle h, int cond) {
  __shared__ uint32_t settled_mask;
  const uint32_t k = threadIdx.x;
  if (k == 0) settled_mask = 0;
  __syncthreads();
  if (k < PCG_MAX_INST && ((cs->cp.todo >> k) & 1u)) {
    const uint32_t np = cs->cp.npass[k];
    const float md = cs->max_disp[k];
    bool settled = false;
    for (uint32_t i = 0; i < np && !settled; ++i) {
      const bool full = cs->sched[k][i] >= md;
      const float t_self = __uint_as_float(acc[2 * (CCD_CHUNK * k + i)]);
      if (full || t_self * md <= cs->sched[k][i]) {
        cs->caps[k] = acc[2 * (CCD_CHUNK * k + i) + 1];
        cs->t[k] = fminf(cs->t[k], t_self);
        settled = true;
      }
    }
    if (settled) {
      atomicOr(&settled_mask, 1u << k);
    } else {
      cs->allowed[k] = fminf(cs->sched[k][np - 1] * 4.0f, md);
      cs->reach[k] = fminf(cs->reach[k], __uint_as_float(acc[2 * (CCD_CHUNK * k + np - 1)]) * md);
    }
  }
  __syncthreads();
  if (k == 0) {
    cs->todo &= ~settled_mask;
    cs->launch += 1;
    if (cond) cudaGraphSetConditional(h, (cs->todo && cs->launch < 64) ? 1u : 0u);
  }
}

__global__ void k_ccd_clamp(CcdState* __restrict__ cs) {
  const uint32_t k = threadIdx.x;
  if (k < PCG_MAX_INST) cs->t[k] = fminf(fmaxf(cs->t[k], 0.f), 1.f);
}

// One launch of the self-contact schedule: plan, then the two traversals (settle follows).
static void ccd_body(Scene& s, const BvhSet& tv, const BvhSet& ev, CcdState* cs) {
  cudaStream_t st = s.st;
  const float dhat = s.p.contact_dhat;
  const float fixed = dhat;  // max_edge_gap() + 2 * max_edge_offset() for face edges
  const uint32_t iters = std::max<uint32_t>(s.p.ccd_max_iter, 1);
  const CcdPass* cpp = &cs->cp;
  k_ccd_plan<<<1, PCG_MAX_INST * CCD_CHUNK, 0, st>>>(cs, s.ccd_acc.p, fixed);
  if (s.mixed) {
    k_ccd_vt<double><<<ceil_div(s.nv, 128), 128, 0, st>>>(
        tv, cpp, s.vinst.p, s.x.p, s.dx.p, s.tris.p, s.collider_tri.p, s.inv_mass.p, s.ex_ptr.p, s.ex_list.p,
        s.side_best.p, s.collider_pn.p, s.has_static ? 1 : 0, s.nv, dhat, iters, s.red.p, s.ccd_acc.p, s.status.p);
    if (s.n_edge)
      k_ccd_ee<double><<<ceil_div(s.n_edge, 128), 128, 0, st>>>(ev, cpp, s.vinst.p, s.x.p, s.dx.p, s.edges.p,
                                                               s.ee_tail.p, s.inv_mass.p, s.n_edge, iters, s.red.p, s.ccd_acc.p,
                                                               s.status.p);
  } else {
    k_ccd_vt<float><<<ceil_div(s.nv, 128), 128, 0, st>>>(
        tv, cpp, s.vinst.p, s.x.p, s.dx.p, s.tris.p, s.collider_tri.p, s.inv_mass.p, s.ex_ptr.p, s.ex_list.p,
        s.side_best.p, s.collider_pn.p, s.has_static ? 1 : 0, s.nv, dhat, iters, s.red.p, s.ccd_acc.p, s.status.p);
    if (s.n_edge)
      k_ccd_ee<float><<<ceil_div(s.n_edge, 128), 128, 0, st>>>(ev, cpp, s.vinst.p, s.x.p, s.dx.p, s.edges.p,
                                                              s.ee_tail.p, s.inv_mass.p, s.n_edge, iters, s.red.p, s.ccd_acc.p,
                                                              s.status.p);
  }
}

// The self-contact schedule's graph: one conditional while node around plan, the two
// traversals and settle. Rebuilt when a by-value argument changes.
static int ccd_graph(Scene& s, const BvhSet& tv, const BvhSet& ev, CcdState* cs) {
  cudaStream_t st = s.st;
  const uint32_t iters = std::max<uint32_t>(s.p.ccd_max_iter, 1);
  std::vector<unsigned char> key(2 * sizeof(BvhSet) + 8 * sizeof(void*) + 16);
  unsigned char* q = key.data();
  auto put = [&](const void* p, size_t n) {
    std::memcpy(q, p, n);
    q += n;
  };
  put(&tv, sizeof(BvhSet));
  put(&ev, sizeof(BvhSet));
  const void* ptrs[8] = {s.x.p, s.dx.p, s.tris.p, s.edges.p, s.ccd_acc.p, s.red.p, s.side_best.p, cs};
  put(ptrs, sizeof(ptrs));
  const uint32_t misc[4] = {s.nv, s.n_edge, iters, s.mixed ? 1u : 0u};
  put(misc, sizeof(misc));
  if (s.ccd_exec && key == s.ccd_key) return MGUSO_OK;
  if (s.ccd_exec) cudaGraphExecDestroy(s.ccd_exec);
  s.ccd_exec = nullptr;
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
  ccd_body(s, tv, ev, cs);
  k_ccd_settle<<<1, 32, 0, st>>>(cs, s.ccd_acc.p, cond, 1);
  const cudaError_t le = cudaGetLastError();
  cudaGraph_t body = nullptr;
  e = cudaStreamEndCapture(st, &body);
  if (le != cudaSuccess || e != cudaSuccess) {
    cudaGraphDestroy(g);
    MG_CUDA(le);
    MG_CUDA(e);
  }
  const cudaError_t ie = cudaGraphInstantiate(&s.ccd_exec, g, 0);
  cudaGraphDestroy(g);
  MG_CUDA(ie);
  s.ccd_key = key;
  return MGUSO_OK;
}

// The step fraction along s.dx from s.x for every instance in `active` (ccd_max_step,
// implicit.rs:1690-1947): analytic colliders, static pins and strain-limit faces in single
// launches, then with self collision the widening schedule as one graph launch. Everything is
// enqueued on the scene's stream with no host wait; the results land in the device state
// (read by k_advance through ccd_t) and in a pinned copy that ccd_results reads once the
// stream has passed it.
int ccd_step(Scene& s, uint32_t active) {
  cudaStream_t st = s.st;
  const uint32_t K = s.ninst;
  MG_TRY(s.ccd_state.reserve(sizeof(CcdState)));
  MG_TRY(s.ccd_acc.reserve(2 * CCD_CHUNK * PCG_MAX_INST));
  MG_TRY(s.ccd_out.reserve(sizeof(CcdState)));
  CcdState* cs = (CcdState*)s.ccd_state.p;
  if (!s.ccd_half_set) {
    float hl[PCG_MAX_INST] = {};
    for (uint32_t k = 0; k < K; ++k) hl[k] = 0.5f * s.char_len[k];
    MG_CUDA(cudaMemcpyAsync(cs->half_len, hl, sizeof(hl), cudaMemcpyHostToDevice, st));
    s.ccd_half_set = true;
  }
  const bool self = s.p.self_collision != 0;
  k_red_init<<<1, RED_STRIDE * PCG_MAX_INST, 0, st>>>(s.red.p, K);
  if (s.n_col || self || s.n_static_pin || s.n_sl) {
    const int sms = s.ctx->sm_count;
    k_max_norm<<<std::min<uint32_t>(ceil_div(s.nv, 256), sms * 4), 256, 0, st>>>(s.dx.p, s.vinst.p, s.nv, s.red.p);
    if (s.n_col && s.n_free)
      k_ccd_colliders<<<ceil_div(s.n_free, 128), 128, 0, st>>>(s.free_verts.p, s.n_free, s.vinst.p, s.x.p, s.dx.p,
                                                             s.colliders.p, s.n_col, s.red.p);
    if (s.n_static_pin)
      k_ccd_pins<<<ceil_div(s.n_pin, 128), 128, 0, st>>>(s.pin_vert.p, s.n_pin, s.pin_kin.p, s.pin_target.p,
                                                        s.pin_ghat.p, s.inv_mass.p, s.vinst.p, s.x.p, s.dx.p, s.red.p);
    if (s.n_sl)
      k_ccd_sl<<<ceil_div(s.n_sl, 128), 128, 0, st>>>(s.n_sl, s.sl_v.p, s.sl_dm.p, s.sl_limit.p, s.vinst.p, s.x.p,
                                                     s.dx.p, s.red.p);
  }
  k_ccd_start<<<1, 32, 0, st>>>(cs, s.red.p, K, active, self ? 1 : 0);
  MG_CUDA(cudaGetLastError());
  if (self) {
    // the trees' displacement boxes (the trees were built at this iterate)
    MG_TRY(aux_fork(s));
    int rc = MGUSO_OK;
    for (uint32_t k = 0; k < K && rc == MGUSO_OK; ++k) {
      if (!((active >> k) & 1u)) continue;  // its self contact is not checked
      rc = lbvh_refit_disp(s.tri_bvh[k].get(), s.dx.p, s.tris.p + 3 * (size_t)s.inst_tri[k], s.aux[(2 * k) % N_AUX]);
      if (rc == MGUSO_OK)
        rc = lbvh_refit_disp(s.edge_bvh[k].get(), s.dx.p, s.edge_tris.p + 3 * (size_t)s.inst_edge[k],
                             s.aux[(2 * k + 1) % N_AUX]);
    }
    MG_TRY(aux_join(s));
    MG_TRY(rc);
    const BvhSet tv = view_set(s.tri_bvh, s.inst_tri), ev = view_set(s.edge_bvh, s.inst_edge);
    if (plain_launches()) {
      // the same launches driven by the host (for profilers)
      for (int launch = 0; launch < 64; ++launch) {
        ccd_body(s, tv, ev, cs);
        k_ccd_settle<<<1, 32, 0, st>>>(cs, s.ccd_acc.p, cudaGraphConditionalHandle{}, 0);
        MG_CUDA(cudaGetLastError());
        uint32_t todo = 0;
        MG_CUDA(cudaMemcpyAsync(&todo, &cs->todo, 4, cudaMemcpyDeviceToHost, st));
        MG_CUDA(cudaStreamSynchronize(st));
        if (!todo) break;
      }
    } else {
      MG_TRY(ccd_graph(s, tv, ev, cs));
      MG_CUDA(cudaGraphLaunch(s.ccd_exec, st));
    }
  }
  k_ccd_clamp<<<1, 32, 0, st>>>(cs);
  MG_CUDA(cudaGetLastError());
  MG_CUDA(cudaMemcpyAsync(s.ccd_out.p, cs, sizeof(CcdState), cudaMemcpyDeviceToHost, st));
  return MGUSO_OK;
}

const float* ccd_t(Scene& s) { return ((CcdState*)s.ccd_state.p)->t; }

uint32_t ccd_launches(Scene& s) { return ((const CcdState*)s.ccd_out.p)->launch; }

int ccd_results(Scene& s, float* t_out, uint32_t* cap_hits) {
  MG_CUDA(cudaStreamSynchronize(s.st));
  const CcdState* cs = (const CcdState*)s.ccd_out.p;
  for (uint32_t k = 0; k < s.ninst; ++k) {
    t_out[k] = cs->t[k];
    cap_hits[k] = cs->caps[k];
  }
  return MGUSO_OK;
}

}  // namespace mg
