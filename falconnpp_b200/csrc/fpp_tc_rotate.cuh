// fpp_tc_rotate.cuh — HD3 rotation of a 256-point vector on the tensor cores,
// for the batched form's low-precision modes (the FP32 modes keep the
// bit-exact FWHT of fpp_device.cuh).
//
// The unnormalised FWHT of size 256 in the reference's (Sylvester) order is
// H256 = H16 (x) H16: with the vector as a 16 x 16 matrix X (x[16a + b] =
// X[a][b]), FWHT(x) = H16 X H16.  One warp computes one rotation round as two
// mma.sync m16n8k16 products with FP16 operands and FP32 accumulation:
//   W = H16 * B   (B = the round's input in B-fragment layout, two n-tiles)
//   Y = W * H16   (W's accumulator fragment is directly the A fragment)
// and Y's accumulator fragment, read as a B fragment, is the next round's
// input transposed (B[k][n] = Y[n][k]); so round 2 works on the transposed
// view and round 3 on the normal view again.  The sign flips of a round are
// XOR masks on the packed halves, taken from flip words arranged per view
// (round 2's words hold the transposed 16 x 16 bit matrix; built with the
// index).
//
// Lane (g, c) = (lane / 4, lane % 4) holds B elements (k, n) = (2c, 2c + 1,
// 2c + 8, 2c + 9) x (n = 8t + g) for n-tiles t = 0, 1; in the normal view
// their vector positions are 32c + 8t + g (+16, +128, +144).  The query is
// scaled by a power of two so that every intermediate stays below 4096 in
// magnitude (FP16 range); the scale is common to all tables of a query, so
// comparisons between them are unaffected.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fpp {

// d = A * B with a zero accumulator (no registers to clear beforehand)
__device__ __forceinline__ void mma_f16_m16n8k16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%10,%10,%10,%10};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(0.0f));
}

__device__ __forceinline__ uint32_t pack_f16x2(float lo, float hi) {
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// +-1 of H16[i][j] = (-1)^popc(i & j) as two packed halves
__device__ __forceinline__ uint32_t h16_pair(int i0, int j0, int i1, int j1) {
  const uint32_t lo = (__popc(i0 & j0) & 1) ? 0xBC00u : 0x3C00u;
  const uint32_t hi = (__popc(i1 & j1) & 1) ? 0xBC00u : 0x3C00u;
  return lo | (hi << 16);
}

// the lane's constant fragments of H16: as the A operand, and as the B
// operand of n-tiles 0 and 1
struct H16Frags {
  uint32_t a[4];
  uint32_t b[2][2];
  __device__ explicit H16Frags(int lane) {
    const int g = lane >> 2, c = lane & 3;
    a[0] = h16_pair(g, 2 * c, g, 2 * c + 1);
    a[1] = h16_pair(g + 8, 2 * c, g + 8, 2 * c + 1);
    a[2] = h16_pair(g, 2 * c + 8, g, 2 * c + 9);
    a[3] = h16_pair(g + 8, 2 * c + 8, g + 8, 2 * c + 9);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      b[t][0] = h16_pair(2 * c, 8 * t + g, 2 * c + 1, 8 * t + g);
      b[t][1] = h16_pair(2 * c + 8, 8 * t + g, 2 * c + 9, 8 * t + g);
    }
  }
};

// the scaled query as the lane's round-1 B registers (normal view)
__device__ __forceinline__ void tc_query_frags(const float* q, float scale, int lane, uint32_t (&qb)[2][2]) {
  const int g = lane >> 2, c = lane & 3;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int p = 32 * c + 8 * t + g;
    qb[t][0] = pack_f16x2(q[p] * scale, q[p + 16] * scale);
    qb[t][1] = pack_f16x2(q[p + 128] * scale, q[p + 144] * scale);
  }
}

// Three rounds (sign flip, FWHT-256) of the lane's fragments starting from
// qb, for NI (table, layer) items at once (independent chains, interleaved);
// tw[i] = the 3 x 8 flip words of item i in per-view order.  For each item,
// the best cross-polytope coordinate among positions < D: its value
// sgn(y)*y (low 9 mantissa bits cleared), and its bucket code (position |
// (y < 0) << log2D), equal values to the smaller position; the same on every
// lane.
template <int NI>
__device__ __forceinline__ void tc_rotate_top1(const uint32_t (&qb)[2][2], const uint32_t* const (&tw)[NI],
                                               const H16Frags& h, int lane, int D, int log2D, float (&best_v)[NI],
                                               int (&best_code)[NI]) {
  const int g = lane >> 2, c = lane & 3;
  uint32_t b[NI][2][2];
  uint32_t wl[NI][3], wh[NI][3];
#pragma unroll
  for (int i = 0; i < NI; ++i) {
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      b[i][t][0] = qb[t][0];
      b[i][t][1] = qb[t][1];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      wl[i][r] = __ldg(tw[i] + r * 8 + c);
      wh[i][r] = __ldg(tw[i] + r * 8 + c + 4);
    }
  }
  float y[NI][2][4];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    // sign flips: bits s and s + 16 of words c and c + 4 (s = 8t + g) go to
    // the sign bits 15 and 31 of the packed pair
#pragma unroll
    for (int i = 0; i < NI; ++i)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int sh = 15 - (8 * t + g);
        b[i][t][0] ^= (wl[i][r] << sh) & 0x80008000u;
        b[i][t][1] ^= (wh[i][r] << sh) & 0x80008000u;
      }
    float w[NI][2][4];
#pragma unroll
    for (int i = 0; i < NI; ++i)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        mma_f16_m16n8k16(w[i][t], h.a, b[i][t][0], b[i][t][1]);
      }
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const uint32_t a[4] = {pack_f16x2(w[i][0][0], w[i][0][1]), pack_f16x2(w[i][0][2], w[i][0][3]),
                             pack_f16x2(w[i][1][0], w[i][1][1]), pack_f16x2(w[i][1][2], w[i][1][3])};
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        mma_f16_m16n8k16(y[i][t], a, h.b[t][0], h.b[t][1]);
      }
    }
    if (r < 2) {
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        b[i][0][0] = pack_f16x2(y[i][0][0], y[i][0][1]);
        b[i][0][1] = pack_f16x2(y[i][1][0], y[i][1][1]);
        b[i][1][0] = pack_f16x2(y[i][0][2], y[i][0][3]);
        b[i][1][1] = pack_f16x2(y[i][1][2], y[i][1][3]);
      }
    }
  }
  // y[i][t][e] is Y[g + 8 (e >> 1)][8t + 2c + (e & 1)], position 16 * row + col.
  // The best coordinate is the largest key
  //   (|y| with the low 9 bits cleared) << 0 | (255 - position) << 1 | sign,
  // one u32 maximum per lane and one warp reduction (redux.sync) per item:
  // magnitudes order as their bits, equal truncated magnitudes go to the
  // smaller position, and the sign bit never decides (positions differ).
  // Truncating 9 of 23 mantissa bits (relative 2^-14) stays far below the
  // FP16 operand rounding of the rotation itself (2^-11 per round).
  // Positions >= D take key 0, which every position < D beats (for D < 256
  // its position bits are >= 1 there).
  constexpr uint32_t kMagMask = 0x7FFFFE00u;
  const uint32_t pbase = 255u - (uint32_t)(16 * g + 2 * c);
  const uint32_t rlim = 256u - (uint32_t)D;  // 255 - position < rlim <=> position >= D
  uint32_t key[NI];
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    key[i] = 0u;
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t u = __float_as_uint(y[i][t][e]);
        const uint32_t rp = pbase - (uint32_t)(128 * (e >> 1) + 8 * t + (e & 1));  // 255 - position
        uint32_t kk = (u & kMagMask) | (rp << 1) | (u >> 31);
        if (rp < rlim) kk = 0u;
        key[i] = max(key[i], kk);
      }
  }
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const uint32_t kb = __reduce_max_sync(0xffffffffu, key[i]);
    const int pos = 255 - (int)((kb >> 1) & 255u);
    const uint32_t mag = kb & kMagMask;
    best_v[i] = __uint_as_float(mag);
    // sgn(): -0 counts as positive (FP16-product sums are 0 or >= 2^-24 in magnitude)
    best_code[i] = ((kb & 1u) && mag) ? (pos | (1 << log2D)) : pos;
  }
}

}  // namespace fpp
