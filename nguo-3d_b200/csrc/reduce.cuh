// Deterministic grid-wide dot-product reduction with a fused "finish" step for the PCG
// scalars: per-CTA partials, summed in index order by the last CTA to arrive.
#pragma once
#include "internal.cuh"

namespace mg {

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums `v` over the CTA (fixed tree order); the result is valid in thread 0.
template <class T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T red[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T s = 0;
  if (w == 0) {
    int nw = (blockDim.x + 31) >> 5;
    s = lane < nw ? red[lane] : T(0);
    s = warp_sum(s);
  }
  return s;
}

__device__ __forceinline__ void finish_scalar(PcgScalars* sc, int fin, double sum) {
  switch (fin) {
    case FIN_STORE:
      sc->out = sum;
      break;
    case FIN_PAP: {
      sc->pap = sum;
      if (!(sum > 0.0)) {  // pAp <= 0 or NaN: the reference breaks out (linsolve.rs:386)
        sc->done = 1;
        sc->status |= ST_PCG_BREAKDOWN;
        sc->alpha = 0.0;
      } else {
        sc->alpha = sc->rz / sum;
      }
      break;
    }
    case FIN_RR: {
      sc->iters += 1;
      sc->residual = sqrt(sum) / sc->bnorm;
      if (sc->residual <= sc->tol || sc->iters >= sc->max_iter) sc->done = 1;
      break;
    }
    case FIN_RZ:
      sc->beta = sum / sc->rz;
      sc->rz = sum;
      break;
    case FIN_RZ0:
      sc->rz = sum;
      break;
    case FIN_BNORM:
      sc->bnorm = fmax(sqrt(sum), 1e-30);
      break;
    case FIN_RR0:
      sc->residual = sqrt(sum) / sc->bnorm;
      if (sc->residual <= sc->tol && false) sc->done = 1;
      break;
  }
}

// Called by every thread of every CTA of the grid with its private partial `v`.
template <class T>
__device__ __forceinline__ void grid_dot_commit(const DotSink& d, T v) {
  T s = block_sum<T>(v);
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    ((T*)d.partials)[blockIdx.x] = s;
    __threadfence();
    unsigned prev = atomicAdd(&d.sc->counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last && threadIdx.x < 32) {
    __threadfence();
    volatile T* part = (volatile T*)d.partials;
    T acc = 0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += 32) acc += part[i];
    acc = warp_sum(acc);
    if (threadIdx.x == 0) {
      finish_scalar(d.sc, d.finish, (double)acc);
      d.sc->counter = 0;
      __threadfence();
    }
  }
}

}  // namespace mg
