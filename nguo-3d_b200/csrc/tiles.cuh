// Schwarz factor storage shared by the standalone apply and the persistent PCG.
#pragma once
#include "internal.cuh"

namespace mg {

// W is stored per domain as its lower block-triangle of 32 x 32 tiles (I, J), J <= I, in
// the order (0,0), (1,0), (1,1), (2,0), (2,1), (2,2); element (r, c) of a tile lives at
// c * 32 + (r ^ c). Rows and columns past m are zero.
constexpr int TILE_FLOATS = 1024;
__host__ __device__ __forceinline__ int tile_index(int I, int J) { return I * (I + 1) / 2 + J; }
__host__ __device__ __forceinline__ int tile_offset(int r, int c) { return c * 32 + (r ^ c); }

// Per-warp shared slice of an apply: the domain's tiles (6 tiles of elements TS), the
// gathered residual (96 floats) and W r (96 values of the accumulation type, 768 bytes).
template <class TS>
__host__ __device__ constexpr uint32_t apply_slice_bytes() {
  return 6 * TILE_FLOATS * (uint32_t)sizeof(TS) + 96 * 4 + 96 * 8;
}
template <class TS>
__device__ __forceinline__ float tile_ld(const TS* t, int o) {
  return (float)t[o];
}
template <>
__device__ __forceinline__ float tile_ld<__half>(const __half* t, int o) {
  return __half2float(t[o]);
}

// One domain's z = W^T (W r) by one warp (see the apply kernel in schwarz.cu); tiles of
// element type TS (FP16 tiles give W / scale, so z comes out divided by scale^2).
template <int T, class Acc, class TS = float>
__device__ __forceinline__ void tiles_apply(const TS* __restrict__ w, const float* __restrict__ rd,
                                            Acc* __restrict__ yd, Acc (&z)[3], int lane) {
  const TS* t00 = w;
  const TS* t10 = w + 1 * TILE_FLOATS;
  const TS* t11 = w + 2 * TILE_FLOATS;
  const TS* t20 = w + 3 * TILE_FLOATS;
  const TS* t21 = w + 4 * TILE_FLOATS;
  const TS* t22 = w + 5 * TILE_FLOATS;
  Acc y0 = 0, y1 = 0, y2 = 0;
#pragma unroll 8
  for (int c = 0; c < 32; ++c) {
    const int o = tile_offset(lane, c);
    const Acc a0 = (Acc)rd[c];
    y0 += (Acc)tile_ld(t00, o) * a0;
    if (T > 1) {
      const Acc a1 = (Acc)rd[32 + c];
      y1 += (Acc)tile_ld(t10, o) * a0 + (Acc)tile_ld(t11, o) * a1;
      if (T > 2) {
        const Acc a2 = (Acc)rd[64 + c];
        y2 += (Acc)tile_ld(t20, o) * a0 + (Acc)tile_ld(t21, o) * a1 + (Acc)tile_ld(t22, o) * a2;
      }
    }
  }
  yd[lane] = y0;
  if (T > 1) yd[32 + lane] = y1;
  if (T > 2) yd[64 + lane] = y2;
  __syncwarp();
  Acc z0 = 0, z1 = 0, z2 = 0;
#pragma unroll 8
  for (int r = 0; r < 32; ++r) {
    const int o = tile_offset(r, lane);
    const Acc b0 = yd[r];
    z0 += (Acc)tile_ld(t00, o) * b0;
    if (T > 1) {
      const Acc b1 = yd[32 + r];
      z0 += (Acc)tile_ld(t10, o) * b1;
      z1 += (Acc)tile_ld(t11, o) * b1;
      if (T > 2) {
        const Acc b2 = yd[64 + r];
        z0 += (Acc)tile_ld(t20, o) * b2;
        z1 += (Acc)tile_ld(t21, o) * b2;
        z2 += (Acc)tile_ld(t22, o) * b2;
      }
    }
  }
  z[0] = z0;
  z[1] = z1;
  z[2] = z2;
}

// z = W_v^T (W_v r) for one vertex of a block-diagonal domain (W_v lower triangular, 6 floats
// w00 w10 w11 w20 w21 w22).
template <class Acc>
__device__ __forceinline__ void vertex_apply(const float* __restrict__ w6, const float* r3, Acc (&z)[3]) {
  const Acc w00 = w6[0], w10 = w6[1], w11 = w6[2], w20 = w6[3], w21 = w6[4], w22 = w6[5];
  const Acc r0 = r3[0], r1 = r3[1], r2 = r3[2];
  const Acc y0 = w00 * r0, y1 = w10 * r0 + w11 * r1, y2 = w20 * r0 + w21 * r1 + w22 * r2;
  z[0] = w00 * y0 + w10 * y1 + w20 * y2;
  z[1] = w11 * y1 + w21 * y2;
  z[2] = w22 * y2;
}

}  // namespace mg
