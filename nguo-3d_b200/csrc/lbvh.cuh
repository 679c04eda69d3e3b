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
