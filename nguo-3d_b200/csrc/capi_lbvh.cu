// extern "C" entry points of the LBVH broad phase and the radix sort.
#include <cstring>

#include "lbvh.cuh"

using namespace mg;

extern "C" {

int mguso_lbvh_create(mguso_ctx* ctx, mguso_lbvh** out) {
  MG_CHECK_ARG(ctx && out, "null argument");
  MG_CUDA(cudaSetDevice(ctx->device));
  auto* b = new mguso_lbvh();
  b->b.ctx = ctx;
  b->b.child_boxes = false;  // its point and box queries walk node and leaf boxes only
  *out = b;
  return MGUSO_OK;
}

int mguso_lbvh_destroy(mguso_lbvh* b) {
  if (!b) return MGUSO_OK;
  for (auto& e : b->b.ev)
    if (e) cudaEventDestroy(e);
  delete b;
  return MGUSO_OK;
}

int mguso_lbvh_build(mguso_lbvh* b, const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt,
                     int key_bits, void* stream) {
  MG_CHECK_ARG(b && (nt == 0 || (positions && tris)), "null argument");
  MG_CHECK_ARG(nt < (1u << 30), "too many triangles (limit 2^30)");
  MG_TRY(b->b.status.reserve(4));
  MG_CUDA(cudaMemsetAsync(b->b.status.p, 0, 4, (cudaStream_t)stream));
  return lbvh_build(&b->b, positions, nv, tris, nt, key_bits, (cudaStream_t)stream);
}

int mguso_lbvh_query_points(mguso_lbvh* b, const float* points, uint32_t np, float dhat, uint32_t* pairs,
                            uint64_t cap, uint64_t* count, void* stream) {
  MG_CHECK_ARG(b && count && (np == 0 || points) && (cap == 0 || pairs), "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  MG_CUDA(cudaMemsetAsync(count, 0, 8, s));
  return lbvh_query_points(&b->b, points, np, dhat, pairs, cap, (unsigned long long*)count, true, s);
}

int mguso_lbvh_download(mguso_lbvh* b, uint64_t* keys, uint32_t* perm, uint32_t* left, uint32_t* right,
                        float* node_boxes) {
  MG_CHECK_ARG(b, "null lbvh");
  Lbvh& L = b->b;
  MG_CUDA(cudaDeviceSynchronize());
  uint32_t nt = L.nt;
  if (keys && nt) {
    if (L.key_bits == 30) {
      std::vector<uint32_t> k(nt);
      MG_CUDA(cudaMemcpy(k.data(), L.keys.p, 4 * (size_t)nt, cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i < nt; ++i) keys[i] = k[i];
    } else {
      MG_CUDA(cudaMemcpy(keys, L.keys.p, 8 * (size_t)nt, cudaMemcpyDeviceToHost));
    }
  }
  if (perm && nt) MG_CUDA(cudaMemcpy(perm, L.perm.p, 4 * (size_t)nt, cudaMemcpyDeviceToHost));
  if (nt > 1) {
    if (left) MG_CUDA(cudaMemcpy(left, L.left.p, 4 * (size_t)(nt - 1), cudaMemcpyDeviceToHost));
    if (right) MG_CUDA(cudaMemcpy(right, L.right.p, 4 * (size_t)(nt - 1), cudaMemcpyDeviceToHost));
    if (node_boxes) {
      std::vector<float4> nb(2 * (size_t)(nt - 1));
      MG_CUDA(cudaMemcpy(nb.data(), L.node.p, sizeof(float4) * nb.size(), cudaMemcpyDeviceToHost));
      for (uint32_t i = 0; i + 1 < nt; ++i) {
        const float4 &lo = nb[2 * i], &hi = nb[2 * i + 1];
        float* o = node_boxes + 6 * (size_t)i;
        o[0] = lo.x; o[1] = lo.y; o[2] = lo.z; o[3] = hi.x; o[4] = hi.y; o[5] = hi.z;
      }
    }
  }
  return MGUSO_OK;
}

int mguso_lbvh_status(mguso_lbvh* b) {
  MG_CHECK_ARG(b, "null lbvh");
  MG_CUDA(cudaStreamSynchronize(b->b.ctx->stream));
  MG_CUDA(cudaDeviceSynchronize());
  uint32_t st = 0;
  if (b->b.status.p) MG_CUDA(cudaMemcpy(&st, b->b.status.p, 4, cudaMemcpyDeviceToHost));
  if (st & ST_WAIT_TIMEOUT) {
    set_error("radix sort look-back wait timed out");
    return MGUSO_ERR_TIMEOUT;
  }
  if (st & ST_STACK_OVERFLOW) {
    set_error("LBVH traversal stack overflow (64 entries)");
    return MGUSO_ERR_BVH_STACK;
  }
  if (st & ST_PAIR_OVERFLOW) {
    set_error("pair buffer too small; *count holds the total");
    return MGUSO_ERR_PAIR_OVERFLOW;
  }
  return MGUSO_OK;
}

int mguso_lbvh_stage_times(mguso_lbvh* b, int enable, float* ms6) {
  MG_CHECK_ARG(b, "null lbvh");
  Lbvh& L = b->b;
  if (enable && !L.ev_on) {
    for (auto& e : L.ev) MG_CUDA(cudaEventCreate(&e));
    L.ev_on = true;
  }
  if (ms6 && L.ev_on) {
    MG_CUDA(cudaDeviceSynchronize());
    for (int i = 0; i < 6; ++i) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, L.ev[i], L.ev[i + 1]) != cudaSuccess) ms = -1.0f;
      ms6[i] = ms;
    }
    cudaGetLastError();
  }
  if (!enable) L.ev_on = false;
  return MGUSO_OK;
}

int mguso_lbvh_build_query(mguso_ctx* ctx, const float* positions, uint32_t nv, const uint32_t* tris, uint32_t nt,
                           int key_bits, float dhat, uint64_t* out_keys, uint32_t* out_perm, uint32_t* out_pairs,
                           uint64_t cap, uint64_t* count) {
  MG_CHECK_ARG(ctx && count && (nv == 0 || positions) && (nt == 0 || tris), "null argument");
  mguso_lbvh* b = nullptr;
  MG_TRY(mguso_lbvh_create(ctx, &b));
  std::unique_ptr<mguso_lbvh, int (*)(mguso_lbvh*)> guard(b, mguso_lbvh_destroy);
  cudaStream_t s = ctx->stream;
  MG_TRY(b->hpos.upload(positions, 3 * (size_t)nv, s));
  MG_TRY(b->htris.upload(tris, 3 * (size_t)nt, s));
  MG_TRY(b->count.reserve(1));
  MG_TRY(b->hpairs.reserve(2 * std::max<uint64_t>(cap, 1)));
  MG_TRY(mguso_lbvh_build(b, b->hpos.p, nv, b->htris.p, nt, key_bits, s));
  MG_TRY(mguso_lbvh_query_points(b, b->hpos.p, nv, dhat, b->hpairs.p, cap, (uint64_t*)b->count.p, s));
  MG_CUDA(cudaMemcpyAsync(count, b->count.p, 8, cudaMemcpyDeviceToHost, s));
  MG_CUDA(cudaStreamSynchronize(s));
  uint64_t got = std::min<uint64_t>(*count, cap);
  if (out_pairs && got) MG_CUDA(cudaMemcpy(out_pairs, b->hpairs.p, 8 * got, cudaMemcpyDeviceToHost));
  MG_TRY(mguso_lbvh_download(b, out_keys, out_perm, nullptr, nullptr, nullptr));
  return mguso_lbvh_status(b);
}

int mguso_radix_sort_pairs(mguso_ctx* ctx, void* keys, uint32_t* vals, uint32_t n, int key_bits, void* stream) {
  MG_CHECK_ARG(ctx && (n == 0 || (keys && vals)), "null argument");
  MG_CHECK_ARG(key_bits >= 1 && key_bits <= 64, "key_bits must be in [1, 64]");
  MG_CHECK_ARG(n < (1u << 30), "too many keys (limit 2^30)");
  if (!ctx->sort_scratch) {
    ctx->sort_scratch = new Lbvh();
    ctx->sort_scratch->ctx = ctx;
  }
  Lbvh* L = ctx->sort_scratch;
  MG_TRY(L->status.reserve(4));
  MG_CUDA(cudaMemsetAsync(L->status.p, 0, 4, (cudaStream_t)stream));
  return radix_sort_pairs(L, keys, vals, n, key_bits, (cudaStream_t)stream);
}

int mguso_radix_sort_status(mguso_ctx* ctx) {
  MG_CHECK_ARG(ctx, "null argument");
  if (!ctx->sort_scratch || !ctx->sort_scratch->status.p) return MGUSO_OK;
  MG_CUDA(cudaDeviceSynchronize());
  uint32_t st = 0;
  MG_CUDA(cudaMemcpy(&st, ctx->sort_scratch->status.p, 4, cudaMemcpyDeviceToHost));
  if (st & ST_WAIT_TIMEOUT) {
    set_error("radix sort look-back wait timed out");
    return MGUSO_ERR_TIMEOUT;
  }
  return MGUSO_OK;
}

}  // extern "C"
