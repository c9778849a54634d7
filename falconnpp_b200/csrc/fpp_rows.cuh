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
constexpr uint32_t kNoRow = 0xffffffffu;

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

// bulk prefetch of `bytes` (a multiple of 16) at a 16-byte aligned global
// address into L2; no registers or shared memory are held while it is in flight
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes));
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
  // rows of the step after next are prefetched into L2 (lane i < 4 * STEPS
  // takes row i of that step); their ids are loaded one step before that
  const bool pf_lane = lane < 4 * STEPS;
  const uint32_t pf_bytes = (uint32_t)row_bytes;
  uint32_t pf_id = kNoRow;
  if (pf_lane) {
    const unsigned r = (unsigned)warp * 4 * STEPS + stride + lane;
    if (r < U) prefetch_l2(rows + (size_t)ids[r] * row_bytes, pf_bytes);
    const unsigned r2 = r + stride;
    pf_id = r2 < U ? ids[r2] : kNoRow;
  }
  for (unsigned base = (unsigned)warp * 4 * STEPS; base < U; base += stride) {
    if (pf_id != kNoRow) prefetch_l2(rows + (size_t)pf_id * row_bytes, pf_bytes);
    if (pf_lane) {
      const unsigned r3 = base + 3 * stride + lane;
      pf_id = r3 < U ? ids[r3] : kNoRow;
    }
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

// ---------------------------------------------------------------------------
// Tensor-core rerank of BF16 / FP8-E4M3 rows (the approximate first pass of
// the batched form; its scores only pick the shortlist that is re-scored in
// FP32 with the parity order above).
//
// A warp takes 16 rows at a time and computes D[16 x 8] = rows[16 x K] *
// B[K x 8] with mma.sync (m16n8k16 BF16 or m16n8k32 E4M3, FP32 accumulate).
// Column n of B holds part n of the query: BF16 hi and lo (q ~ hi + lo to 16
// mantissa bits), or three E4M3 terms of q / qscale; the other columns are 0,
// so the score of a row is the sum of its 8 accumulator columns.
//
// Lane (g, c) = (lane / 4, lane % 4) loads 16-byte chunk 4j + c of rows g and
// g + 8; the 16 bytes are its A registers for two k-steps.  The k positions
// of a fragment are a permutation of the dimensions, the same for A and B
// (B column g is loaded by lanes with group g from the same chunk of the
// query part), so the products pair row and query elements of the same
// dimension.  Loads are issued four chunks (eight 16-byte loads per lane) at
// a time; the ids of the warp's next tile are loaded one tile ahead.
__device__ __forceinline__ void mma_bf16_m16n8k16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                  uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void mma_e4m3_m16n8k32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                  uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k32.row.col.f32.e4m3.e4m3.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <int MODE>
struct QueryParts {
  static constexpr int NP = MODE == kRowsBF16 ? 2 : 3;   // B columns in use
  static constexpr int PC = MODE == kRowsBF16 ? 64 : 32; // 16-byte chunks per part (d <= 512)
  static constexpr int EPC = RowFmt<MODE>::EPC;
  static constexpr int kBytes = NP * PC * 16;
};

// the query parts of the tensor-core rerank, from the FP32 query qs (zero
// padded to 1024): BF16 hi = bf16(q), lo = bf16(q - hi); E4M3 terms of
// y = q / qscale: h = e4m3(y), m = e4m3(y - h), l = e4m3(y - h - m).  Called
// by all threads of the block; the caller synchronises before use.
template <int MODE>
__device__ __forceinline__ void fill_query_parts(const float* qs, float qscale, unsigned char* qx) {
  using P = QueryParts<MODE>;
  constexpr int per_part = P::PC * P::EPC;
  for (int e = threadIdx.x; e < per_part; e += blockDim.x) {
    const float x = qs[e];
    if (MODE == kRowsBF16) {
      const __nv_bfloat16 hi = __float2bfloat16_rn(x);
      const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
      reinterpret_cast<__nv_bfloat16*>(qx)[e] = hi;
      reinterpret_cast<__nv_bfloat16*>(qx)[per_part + e] = lo;
    } else {
      float y = x / qscale;
#pragma unroll
      for (int p = 0; p < P::NP; ++p) {
        const __nv_fp8_storage_t t = __nv_cvt_float_to_fp8(y, __NV_SATFINITE, __NV_E4M3);
        qx[p * per_part + e] = (unsigned char)t;
        const __half_raw hr = __nv_cvt_fp8_to_halfraw(t, __NV_E4M3);
        y = y - __half2float(*reinterpret_cast<const __half*>(&hr));
      }
    }
  }
}

template <int MODE>
__device__ __forceinline__ void rerank_rows_mma(const uint32_t* ids, unsigned U, uint32_t* score,
                                                const unsigned char* qx, const unsigned char* rows, size_t row_bytes,
                                                int nchunk, const float* scale, float qscale, int warp, int nwarps,
                                                int lane, uint32_t* hist11) {
  using P = QueryParts<MODE>;
  const int g = lane >> 2;
  const int c = lane & 3;
  const int JN = (nchunk + 3) >> 2;
  const unsigned ntiles = (U + 15u) >> 4;
  const uint4* qpart = reinterpret_cast<const uint4*>(qx) + (g < P::NP ? g : 0) * P::PC + c;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  unsigned tile = (unsigned)warp;
  const unsigned nw = (unsigned)nwarps;
  uint32_t nid0 = 0u, nid1 = 0u;
  if (tile < ntiles) {
    const unsigned r0 = tile * 16u + g;
    nid0 = r0 < U ? ids[r0] : 0u;
    nid1 = r0 + 8u < U ? ids[r0 + 8u] : 0u;
  }
  // when a tile takes more than one round of loads (rows longer than 256
  // bytes), the rows of the warp's next two tiles are prefetched into L2:
  // lane 2i + h (i < 8, h < 2) takes row i + 8h; the ids of a tile are loaded
  // one tile before its prefetch is issued.  With one round per tile the
  // prefetch costs more than it hides.
  const bool pf_lane = lane < 16 && JN > 4;
  const unsigned pf_row = (unsigned)(lane >> 1) + 8u * (unsigned)(lane & 1);
  const uint32_t pf_bytes = (uint32_t)row_bytes;
  uint32_t pf_id = kNoRow;
  if (pf_lane) {
    const unsigned r = (tile + nw) * 16u + pf_row;
    if (r < U) prefetch_l2(rows + (size_t)ids[r] * row_bytes, pf_bytes);
    const unsigned r2 = (tile + 2u * nw) * 16u + pf_row;
    pf_id = r2 < U ? ids[r2] : kNoRow;
  }
  for (; tile < ntiles; tile += nw) {
    if (pf_id != kNoRow) prefetch_l2(rows + (size_t)pf_id * row_bytes, pf_bytes);
    if (pf_lane) {
      const unsigned r3 = (tile + 3u * nw) * 16u + pf_row;
      pf_id = r3 < U ? ids[r3] : kNoRow;
    }
    const unsigned r0 = tile * 16u + g;
    const unsigned r1 = r0 + 8u;
    const bool l0 = r0 < U, l1 = r1 < U;
    const uint32_t id0 = nid0, id1 = nid1;
    {
      const unsigned n0 = r0 + 16u * (unsigned)nwarps;
      nid0 = n0 < U ? ids[n0] : 0u;
      nid1 = n0 + 8u < U ? ids[n0 + 8u] : 0u;
    }
    // the FP8 row scales are loaded together with the rows
    float f0 = 1.0f, f1 = 1.0f;
    if (MODE == kRowsFP8 && c == 0) {
      f0 = l0 ? __ldg(scale + id0) : 0.0f;
      f1 = l1 ? __ldg(scale + id1) : 0.0f;
    }
    const uint4* p0 = reinterpret_cast<const uint4*>(rows + (size_t)id0 * row_bytes) + c;
    const uint4* p1 = reinterpret_cast<const uint4*>(rows + (size_t)id1 * row_bytes) + c;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int j0 = 0; j0 < JN; j0 += 4) {
      uint4 x0[4], x1[4];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const bool ok = 4 * (j0 + jj) + c < nchunk;
        x0[jj] = (ok && l0) ? __ldg(p0 + 4 * (j0 + jj)) : zero;
        x1[jj] = (ok && l1) ? __ldg(p1 + 4 * (j0 + jj)) : zero;
      }
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        if (j0 + jj < JN) {
          const uint4 b = g < P::NP ? qpart[4 * (j0 + jj)] : zero;
          if (MODE == kRowsBF16) {
            mma_bf16_m16n8k16(acc, x0[jj].x, x1[jj].x, x0[jj].y, x1[jj].y, b.x, b.y);
            mma_bf16_m16n8k16(acc, x0[jj].z, x1[jj].z, x0[jj].w, x1[jj].w, b.z, b.w);
          } else {
            mma_e4m3_m16n8k32(acc, x0[jj].x, x1[jj].x, x0[jj].y, x1[jj].y, b.x, b.y);
            mma_e4m3_m16n8k32(acc, x0[jj].z, x1[jj].z, x0[jj].w, x1[jj].w, b.z, b.w);
          }
        }
      }
    }
    // row g: columns 2c, 2c+1 in acc[0..1]; row g + 8 in acc[2..3]
    float s0 = acc[0] + acc[1];
    float s1 = acc[2] + acc[3];
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    if (c == 0) {
      if (l0) {
        const float t = MODE == kRowsFP8 ? s0 * qscale * f0 : s0;
        score[r0] = __float_as_uint(t);
        if (hist11) atomicAdd(hist11 + (ord_key_bits(__float_as_uint(t)) >> 21), 1u);
      }
      if (l1) {
        const float t = MODE == kRowsFP8 ? s1 * qscale * f1 : s1;
        score[r1] = __float_as_uint(t);
        if (hist11) atomicAdd(hist11 + (ord_key_bits(__float_as_uint(t)) >> 21), 1u);
      }
    }
  }
}

// 16-byte cp.async from global memory into shared memory (cached in L2
// only), a 16-byte shared-memory load, and group control of the calling
// thread's outstanding copies
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gmem) : "memory");
}
__device__ __forceinline__ uint4 ld_shared_u4(uint32_t saddr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(saddr)
               : "memory");
  return v;
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// rerank_rows_mma with two tiles in flight per warp, both in shared memory:
// the warp's tiles alternate between two stages of 16 * row_bytes bytes
// (stage0, stage1), filled by cp.async and read back with 16-byte shared
// loads right before the mma, so no registers hold rows in flight.  Rows
// of one load round only (nchunk <= 16).  Each lane copies and later reads
// back only its own chunks (4j + c of rows g and g + 8), so waiting for its
// own copy groups suffices; a stage is refilled only after the mma that
// consume its chunks have been issued.  The products and their order are
// those of rerank_rows_mma, so the scores are the same bits.  Returns with
// no copy in flight.
template <int MODE>
__device__ __forceinline__ void rerank_rows_mma_2stage(const uint32_t* ids, unsigned U, uint32_t* score,
                                                       const unsigned char* qx, const unsigned char* rows,
                                                       size_t row_bytes, int nchunk, const float* scale, float qscale,
                                                       int warp, int nwarps, int lane, uint32_t* hist11,
                                                       unsigned char* stage0, unsigned char* stage1) {
  using P = QueryParts<MODE>;
  const int g = lane >> 2;
  const int c = lane & 3;
  const unsigned ntiles = (U + 15u) >> 4;
  const unsigned nw = (unsigned)nwarps;
  const int JN = (nchunk + 3) >> 2;  // chunk rounds of 4 (<= 4 here)
  const uint4* qpart = reinterpret_cast<const uint4*>(qx) + (g < P::NP ? g : 0) * P::PC + c;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  // shared address of the lane's chunk c of row g in each stage; row g + 8
  // is 8 rows further
  const uint32_t lane_off = (uint32_t)(g * row_bytes) + 16u * (uint32_t)c;
  const uint32_t sa0 = (uint32_t)__cvta_generic_to_shared(stage0) + lane_off;
  const uint32_t sa1 = (uint32_t)__cvta_generic_to_shared(stage1) + lane_off;
  const uint32_t rb8 = 8u * (uint32_t)row_bytes;
  auto tile_ids = [&](unsigned t, uint32_t& i0, uint32_t& i1) {
    i0 = i1 = kNoRow;
    if (t < ntiles) {
      const unsigned r0 = t * 16u + g;
      if (r0 < U) i0 = ids[r0];
      if (r0 + 8u < U) i1 = ids[r0 + 8u];
    }
  };
  // start copying the rows i0, i1 into the stage at sa (one commit group,
  // empty when both are absent); the FP8 row scales load at the same time
  auto issue = [&](uint32_t sa, uint32_t i0, uint32_t i1, float& f0, float& f1) {
    const unsigned char* p0 = rows + (size_t)(i0 != kNoRow ? i0 : 0u) * row_bytes + 16u * (unsigned)c;
    const unsigned char* p1 = rows + (size_t)(i1 != kNoRow ? i1 : 0u) * row_bytes + 16u * (unsigned)c;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      if (4 * jj + c < nchunk) {
        if (i0 != kNoRow) cp_async16(sa + 64u * jj, p0 + 64 * jj);
        if (i1 != kNoRow) cp_async16(sa + rb8 + 64u * jj, p1 + 64 * jj);
      }
    }
    cp_async_commit();
    f0 = f1 = 1.0f;
    if (MODE == kRowsFP8 && c == 0) {
      f0 = i0 != kNoRow ? __ldg(scale + i0) : 0.0f;
      f1 = i1 != kNoRow ? __ldg(scale + i1) : 0.0f;
    }
  };
  // the tile held in the stage at sa: mma over its chunks, then the scores
  // (row g: columns 2c, 2c+1 in acc[0..1]; row g + 8 in acc[2..3])
  auto compute = [&](unsigned t, uint32_t sa, uint32_t i0, uint32_t i1, float f0, float f1) {
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      if (jj < JN) {
        const bool ok = 4 * jj + c < nchunk;
        const uint4 a0 = (ok && i0 != kNoRow) ? ld_shared_u4(sa + 64u * jj) : zero;
        const uint4 a1 = (ok && i1 != kNoRow) ? ld_shared_u4(sa + rb8 + 64u * jj) : zero;
        const uint4 b = g < P::NP ? qpart[4 * jj] : zero;
        if (MODE == kRowsBF16) {
          mma_bf16_m16n8k16(acc, a0.x, a1.x, a0.y, a1.y, b.x, b.y);
          mma_bf16_m16n8k16(acc, a0.z, a1.z, a0.w, a1.w, b.z, b.w);
        } else {
          mma_e4m3_m16n8k32(acc, a0.x, a1.x, a0.y, a1.y, b.x, b.y);
          mma_e4m3_m16n8k32(acc, a0.z, a1.z, a0.w, a1.w, b.z, b.w);
        }
      }
    }
    const unsigned r0 = t * 16u + g;
    const unsigned r1 = r0 + 8u;
    float s0 = acc[0] + acc[1];
    float s1 = acc[2] + acc[3];
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    if (c == 0) {
      if (r0 < U) {
        const float v = MODE == kRowsFP8 ? s0 * qscale * f0 : s0;
        score[r0] = __float_as_uint(v);
        if (hist11) atomicAdd(hist11 + (ord_key_bits(__float_as_uint(v)) >> 21), 1u);
      }
      if (r1 < U) {
        const float v = MODE == kRowsFP8 ? s1 * qscale * f1 : s1;
        score[r1] = __float_as_uint(v);
        if (hist11) atomicAdd(hist11 + (ord_key_bits(__float_as_uint(v)) >> 21), 1u);
      }
    }
  };
  unsigned t = (unsigned)warp;
  uint32_t a0, a1, b0, b1, na0, na1, nb0, nb1;
  float fa0, fa1, fb0, fb1;
  // two commit groups always in order: stage 0's, then stage 1's
  tile_ids(t, a0, a1);
  tile_ids(t + nw, b0, b1);
  issue(sa0, a0, a1, fa0, fa1);
  issue(sa1, b0, b1, fb0, fb1);
  tile_ids(t + 2u * nw, na0, na1);
  tile_ids(t + 3u * nw, nb0, nb1);
  for (; t < ntiles; t += 2u * nw) {
    cp_async_wait_one();  // stage 0's group (the older one) has landed
    compute(t, sa0, a0, a1, fa0, fa1);
    a0 = na0;
    a1 = na1;
    issue(sa0, a0, a1, fa0, fa1);  // tile t + 2 nw (its mma above were issued first)
    cp_async_wait_one();  // stage 1's group has landed
    if (t + nw < ntiles) compute(t + nw, sa1, b0, b1, fb0, fb1);
    b0 = nb0;
    b1 = nb1;
    issue(sa1, b0, b1, fb0, fb1);  // tile t + 3 nw
    tile_ids(t + 4u * nw, na0, na1);
    tile_ids(t + 5u * nw, nb0, nb1);
  }
  cp_async_wait_all();
}

}  // namespace fpp
