// Operator-agnostic device PCG (see pcg.cu).
#pragma once
#include <functional>

#include "internal.cuh"

namespace mg {

using VecOp = std::function<int(const float* in, float* out, cudaStream_t, const DotSink*)>;

struct PcgOps {
  cudaStream_t stream = nullptr;
  bool mixed = true;
  int sms = 148;
  bool graphable = true;
  uint64_t key = 0;  // identifies the operator/buffers a cached graph was captured with
  VecOp spmv;        // out = A in, fused dot(in, out) into the sink
  VecOp precond;     // out = M^-1 in, fused dot(in, out) into the sink
};

int pcg_run(const PcgOps& ops, PcgWork& w, float tol, uint32_t max_iter, mguso_lin_stats* out);
int vec_grid(uint32_t n, int threads, int sms);
int pcg_vector_update(PcgWork& w, bool mixed, int sms, cudaStream_t st);
int bj_apply(const float* inv, const float* r, float* z, uint32_t nb, int sms, cudaStream_t st, const DotSink* d);

}  // namespace mg
