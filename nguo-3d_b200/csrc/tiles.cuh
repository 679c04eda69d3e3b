// Schwarz factor storage shared by the standalone apply and the persistent PCG.
#pragma once
#include "internal.cuh"

namespace mg {

// W is stored per domain as its lower block-triangle of 32 x 32 tiles (I, J), J <= I, in
// the order (0,0), (1,0), (1,1), (2,0), (2,1), (2,2), each tile column-major (column c at
// c * 32). FP32 tiles permute a column's elements: element (r, c) at c * 32 + (r ^ c), which
// keeps both scalar passes of the apply free of bank conflicts. FP16 tiles keep every
// aligned 8-element chunk of a column whole (16 bytes: one row of an ldmatrix load) and
// permute the chunks: chunk k of column c at position (k ^ (c >> 1)) & 3, so that the eight
// columns of an 8 x 8 ldmatrix load fall into distinct 16-byte bank groups. Rows and columns
// past m are zero.
constexpr int TILE_FLOATS = 1024;
__host__ __device__ __forceinline__ int tile_index(int I, int J) { return I * (I + 1) / 2 + J; }
template <class TS>
__host__ __device__ __forceinline__ int tile_off(int r, int c) {
  return c * 32 + (r ^ c);
}
template <>
__host__ __device__ __forceinline__ int tile_off<__half>(int r, int c) {
  return c * 32 + ((((r >> 3) ^ (c >> 1)) & 3) << 3) + (r & 7);
}
// The inverse: the (r, c) stored at offset o of a tile.
template <class TS>
__host__ __device__ __forceinline__ void tile_rc(int o, int& r, int& c) {
  c = o >> 5;
  r = (o & 31) ^ c;
}
template <>
__host__ __device__ __forceinline__ void tile_rc<__half>(int o, int& r, int& c) {
  c = o >> 5;
  r = (((((o & 31) >> 3) ^ (c >> 1)) & 3) << 3) + (o & 7);
}

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
    const int o = tile_off<TS>(lane, c);
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
    const int o = tile_off<TS>(r, lane);
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

// ---- one domain's apply on the tensor cores ----------------------------------------------
// z = W~^T (W~ r) for FP16 tiles W~ by one warp with mma.sync m16n8k16 (FP16 operands, FP32
// accumulation), over 16 x 16 blocks of the lower block-triangle. The vector operand is the
// B matrix's first three columns: a vector v scaled by a power of two 2^-e (|v| <= 1 after
// scaling, exactly) is split into v = h + m 2^-11 + l 2^-22 with h, m, l in FP16, so each
// product with an FP16 tile element is exact in FP32 and the three columns of the result add
// up to the FP32-accurate product (about 33 significant bits of v relative to its largest
// entry). Pass 1 forms y = W~ r with A = the W~ blocks (ldmatrix.trans from the column-major
// tiles), pass 2 z = W~^T y with A = their transposes (ldmatrix), y scaled and split again.
// rd: r (96 floats, zero past m); ys, zs: 96-float scratch; returns z for rows lane,
// lane + 32, lane + 64 (zero past m). The block order and every sum are fixed: deterministic.
__device__ __forceinline__ uint32_t tc_pack(__half lo, __half hi) {
  return (uint32_t)__half_as_ushort(lo) | ((uint32_t)__half_as_ushort(hi) << 16);
}
// term n (0, 1, 2; 3..7 zero) of the split of x (|x| <= 1)
__device__ __forceinline__ __half tc_term(float x, int n) {
  const __half h = __float2half_rn(x);
  if (n == 0) return h;
  const float r1 = x - __half2float(h);
  const __half mi = __float2half_rn(r1 * 2048.f);
  if (n == 1) return mi;
  if (n == 2) return __float2half_rn((r1 - __half2float(mi) * (1.f / 2048.f)) * 4194304.f);
  return __float2half_rn(0.f);
}
// the B fragment (two registers) of block kb of the scaled vector v: rows k = 16 kb + 2t,
// 2t + 1 (b0) and 2t + 8, 2t + 9 (b1), column n = g
__device__ __forceinline__ void tc_bfrag(const float* v, float inv, int kb, int lane, uint32_t& b0, uint32_t& b1) {
  const int g = lane >> 2, t = lane & 3, k = 16 * kb + 2 * t;
  b0 = tc_pack(tc_term(v[k] * inv, g), tc_term(v[k + 1] * inv, g));
  b1 = tc_pack(tc_term(v[k + 8] * inv, g), tc_term(v[k + 9] * inv, g));
}
__device__ __forceinline__ void tc_mma(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// the A fragment of 16-block (I, J) of W~ (trans = false: of its transpose)
template <bool TRANS>
__device__ __forceinline__ void tc_afrag(const __half* buf, int I, int J, int lane, uint32_t (&a)[4]) {
  const __half* base = buf + tile_index(I >> 1, J >> 1) * TILE_FLOATS;
  const int q = lane >> 3, j = lane & 7;
  // pass 1 (TRANS): matrix q covers A rows 8 (q & 1) and columns 8 (q >> 1); its memory rows
  // are W~ columns. Pass 2: A = the block's transpose, its rows are W~ columns.
  const int cq = TRANS ? (q >> 1) : (q & 1), rq = TRANS ? (q & 1) : (q >> 1);
  const int c = 16 * (J & 1) + 8 * cq + j;
  const int chunk = 2 * (I & 1) + rq;
  const uint32_t addr = smem_u32(base + c * 32 + (((chunk ^ (c >> 1)) & 3) << 3));
  if (TRANS)
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(addr));
  else
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(addr));
}
// the three split columns of a C fragment added up for rows g and g + 8 (valid in lanes with
// t = 0), times sc
__device__ __forceinline__ void tc_combine(const float (&c)[4], float sc, float& y0, float& y1) {
  const float n2a = __shfl_down_sync(0xffffffffu, c[0], 1);  // column 2 of row g (lane t = 1)
  const float n2b = __shfl_down_sync(0xffffffffu, c[2], 1);
  y0 = (c[0] + c[1] * (1.f / 2048.f) + n2a * (1.f / 4194304.f)) * sc;
  y1 = (c[2] + c[3] * (1.f / 2048.f) + n2b * (1.f / 4194304.f)) * sc;
}
__device__ __forceinline__ float tc_scale_exp(const float* v, int lane, float& sc) {
  float mx = fmaxf(fmaxf(fabsf(v[lane]), fabsf(v[lane + 32])), fabsf(v[lane + 64]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (!(mx > 1e-30f) || !isfinite(mx)) {  // a (near) zero vector: z = 0 (and no 2^-e overflow)
    sc = 0.f;
    return 0.f;
  }
  int e;
  frexpf(mx, &e);  // mx < 2^e
  sc = ldexpf(1.f, e);
  return ldexpf(1.f, -e);
}
__device__ __forceinline__ void tc_apply(const __half* __restrict__ buf, const float* __restrict__ rd,
                                         float* __restrict__ ys, float* __restrict__ zs, int m, float (&z)[3],
                                         int lane) {
  const int nb = (m + 15) >> 4, g = lane >> 2, t = lane & 3;
  float sr;
  const float ir = tc_scale_exp(rd, lane, sr);
  for (int i = lane; i < 96; i += 32) zs[i] = 0.f;
  if (sr == 0.f) {
    __syncwarp();
    z[0] = z[1] = z[2] = 0.f;
    return;
  }
  // pass 1: y = W~ r, block row I over blocks J <= I
  uint32_t b[6][2];
#pragma unroll
  for (int kb = 0; kb < 6; ++kb)
    if (kb < nb) tc_bfrag(rd, ir, kb, lane, b[kb][0], b[kb][1]);
  for (int I = 0; I < 6; ++I) {
    float y0 = 0.f, y1 = 0.f;
    if (I < nb) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int J = 0; J < 6; ++J)
        if (J <= I) {
          uint32_t a[4];
          tc_afrag<true>(buf, I, J, lane, a);
          tc_mma(c, a, b[J][0], b[J][1]);
        }
      tc_combine(c, sr, y0, y1);
    }
    if (t == 0) {
      ys[16 * I + g] = y0;
      ys[16 * I + g + 8] = y1;
    }
  }
  __syncwarp();
  // pass 2: z = W~^T y, block column J over blocks I >= J
  float sy;
  const float iy = tc_scale_exp(ys, lane, sy);
  if (sy != 0.f) {
#pragma unroll
    for (int kb = 0; kb < 6; ++kb)
      if (kb < nb) tc_bfrag(ys, iy, kb, lane, b[kb][0], b[kb][1]);
    for (int J = 0; J < nb; ++J) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int I = 0; I < 6; ++I)
        if (I >= J && I < nb) {
          uint32_t a[4];
          tc_afrag<false>(buf, I, J, lane, a);
          tc_mma(c, a, b[I][0], b[I][1]);
        }
      float z0, z1;
      tc_combine(c, sy, z0, z1);
      if (t == 0) {
        zs[16 * J + g] = z0;
        zs[16 * J + g + 8] = z1;
      }
    }
  }
  __syncwarp();
  z[0] = zs[lane];
  z[1] = zs[lane + 32];
  z[2] = zs[lane + 64];
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
