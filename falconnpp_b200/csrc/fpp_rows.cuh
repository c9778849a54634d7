// fpp_rows.cuh — reranking of gathered candidate rows: 8 lanes per row, 4 rows
// per warp step, two steps in flight, in FP32, BF16 or FP8-E4M3 storage with
// FP32 accumulation.
//
// Dot-product order (all modes): rows are split into 16-byte chunks; virtual
// lane t (0..31) accumulates chunks t, t+32, ... element by element with
// fmaf; the 32 virtual-lane sums are combined by the xor butterfly
// 16, 8, 4, 2, 1.  Real lane j of a row's 8 lanes plays virtual lanes j, j+8,
// j+16, j+24 and performs the 16 and 8 levels in registers.  For FP32 rows
// this is exactly the order of the CPU oracle, so the FP32 scores are the
// reference-parity scores bit for bit.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fpp_heap.h"

namespace fpp {

enum RowMode : int { kRowsF32 = 0, kRowsBF16 = 1, kRowsFP8 = 2 };

template <int MODE>
struct RowFmt {
  static constexpr int EPC = MODE == kRowsF32 ? 4 : (MODE == kRowsBF16 ? 8 : 16);  // elements per 16 B
};

__device__ __forceinline__ void unpack_chunk_f32(const uint4& u, float* x) {
  x[0] = __uint_as_float(u.x);
  x[1] = __uint_as_float(u.y);
  x[2] = __uint_as_float(u.z);
  x[3] = __uint_as_float(u.w);
}

__device__ __forceinline__ void unpack_chunk_bf16(const uint4& u, float* x) {
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    x[2 * i] = __uint_as_float(w[i] << 16);
    x[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
  }
}

__device__ __forceinline__ void unpack_chunk_fp8(const uint4& u, float* x) {
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] & 0xffffu), __NV_E4M3);
    const __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] >> 16), __NV_E4M3);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&lo));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&hi));
    x[4 * i] = a.x;
    x[4 * i + 1] = a.y;
    x[4 * i + 2] = b.x;
    x[4 * i + 3] = b.y;
  }
}

template <int MODE>
__device__ __forceinline__ void unpack_chunk(const uint4& u, float* x) {
  if (MODE == kRowsF32)
    unpack_chunk_f32(u, x);
  else if (MODE == kRowsBF16)
    unpack_chunk_bf16(u, x);
  else
    unpack_chunk_fp8(u, x);
}

// Scores of rows ids[0..U) written to score[0..U) (float bits).  Called by
// all threads of the block; warps take 4 rows per step (one per 8-lane group),
// STEPS steps at a time (all their loads in flight together).  qs is the query in shared memory, zero-padded to
// nchunk * elements-per-chunk floats; row_bytes is the row stride in bytes
// (multiple of 16); nchunk the 16-byte chunks that hold the d elements; scale
// (FP8 only) the per-row factor; hist11, when given, counts the scores by the
// top 11 bits of their order-preserving key.
template <int MODE, int VI, int STEPS = 2>
__device__ __forceinline__ void rerank_rows(const uint32_t* ids, unsigned U, uint32_t* score, const float* qs,
                                            const unsigned char* rows, size_t row_bytes, int nchunk,
                                            const float* scale, int warp, int nwarps, int lane,
                                            uint32_t* hist11 = nullptr) {
  constexpr int EPC = RowFmt<MODE>::EPC;
  const int j = lane & 7;
  const int rsub = lane >> 3;  // which of the warp's 4 rows
  const unsigned stride = (unsigned)nwarps * 4 * STEPS;
  // the ids of the next step are loaded one step ahead, so a row load never
  // waits for the id load in front of it
  uint32_t nid[STEPS];
#pragma unroll
  for (int s = 0; s < STEPS; ++s) {
    const unsigned r = (unsigned)warp * 4 * STEPS + s * 4 + rsub;
    nid[s] = r < U ? ids[r] : 0u;
  }
  for (unsigned base = (unsigned)warp * 4 * STEPS; base < U; base += stride) {
    uint4 data[STEPS][4][VI];
    uint32_t rid[STEPS];
    bool live[STEPS];
#pragma unroll
    for (int s = 0; s < STEPS; ++s) {
      const unsigned r = base + s * 4 + rsub;
      live[s] = r < U;
      rid[s] = nid[s];
      const uint4* row = reinterpret_cast<const uint4*>(rows + (size_t)rid[s] * row_bytes);
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int i = 0; i < VI; ++i) {
          const int c = j + 8 * v + 32 * i;
          data[s][v][i] = (live[s] && c < nchunk) ? __ldg(row + c) : make_uint4(0u, 0u, 0u, 0u);
        }
    }
#pragma unroll
    for (int s = 0; s < STEPS; ++s) {
      const unsigned r = base + stride + s * 4 + rsub;
      nid[s] = r < U ? ids[r] : 0u;
    }
#pragma unroll
    for (int s = 0; s < STEPS; ++s) {
      float acc[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        float a = 0.0f;
#pragma unroll
        for (int i = 0; i < VI; ++i) {
          const int c = j + 8 * v + 32 * i;
          if (c < nchunk) {
            float x[EPC];
            unpack_chunk<MODE>(data[s][v][i], x);
            const float4* q4 = reinterpret_cast<const float4*>(qs + c * EPC);
#pragma unroll
            for (int e4 = 0; e4 < EPC / 4; ++e4) {
              const float4 qq = q4[e4];
              a = fmaf(qq.x, x[4 * e4 + 0], a);
              a = fmaf(qq.y, x[4 * e4 + 1], a);
              a = fmaf(qq.z, x[4 * e4 + 2], a);
              a = fmaf(qq.w, x[4 * e4 + 3], a);
            }
          }
        }
        acc[v] = a;
      }
      float t = __fadd_rn(__fadd_rn(acc[0], acc[2]), __fadd_rn(acc[1], acc[3]));
      t = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, 4));
      t = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, 2));
      t = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, 1));
      if (MODE == kRowsFP8) t = __fmul_rn(t, live[s] ? __ldg(scale + rid[s]) : 0.0f);
      if (j == 0 && live[s]) {
        score[base + s * 4 + rsub] = __float_as_uint(t);
        if (hist11) atomicAdd(hist11 + (ord_key_bits(__float_as_uint(t)) >> 21), 1u);
      }
    }
  }
}

}  // namespace fpp
