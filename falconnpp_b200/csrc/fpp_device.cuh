// fpp_device.cuh — device building blocks shared by the build and query kernels:
// group-parallel HD3 rotation (random sign + fast Walsh-Hadamard transform),
// cross-polytope top-p selection with exact tie handling, block scans and the
// order-preserving float keys.
//
// Arithmetic contract (bit-exact with the reference's FP32 path):
//  * the sign step multiplies by +1 or -1 (src/FalconnPP.cpp:85-89); it is a
//    flip of the IEEE sign bit here;
//  * the FWHT is the unnormalised increasing-stride radix-2 transform
//    (h = 1, 2, 4, ...; (a, b) -> (a + b, a - b)), which is what the
//    reference's fht_float computes bit for bit (src/fht.h:11);
//  * all files are compiled without fast-math and with -fmad=false, so no
//    add is contracted or reassociated.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fpp_heap.h"

namespace fpp {

constexpr unsigned kFullMask = 0xffffffffu;

// A vector of FHT floats is held by a group of G lanes, E consecutive
// elements per lane (lane gl holds elements gl*E .. gl*E+E-1).
template <int FHT>
struct Geo {
  static constexpr int E = FHT < 32 ? FHT : 32;
  static constexpr int G = FHT / E;
  static constexpr int WORDS = FHT < 32 ? 1 : FHT / 32;  // sign words per vector
};

__device__ __forceinline__ uint32_t ord_key(float f) { return ord_key_bits(__float_as_uint(f)); }

// Two butterflies at once with Blackwell's packed FP32 instructions
// (add.rn.f32x2 / sub.rn.f32x2: each component rounds exactly like a scalar
// add / sub): (a0, a1) <- (a0 + b0, a1 + b1), (b0, b1) <- (a0 - b0, a1 - b1).
// Written in inline PTX over scalar registers: with the float2 intrinsics the
// compiler kept the lane's vector in local memory in some callers.
__device__ __forceinline__ void f32x2_butterfly(float& a0, float& a1, float& b0, float& b1) {
  asm("{\n .reg .b64 ra, rb, rs, rd;\n mov.b64 ra, {%0, %1};\n mov.b64 rb, {%2, %3};\n"
      " add.rn.f32x2 rs, ra, rb;\n sub.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rs;\n mov.b64 {%2, %3}, rd;\n}"
      : "+f"(a0), "+f"(a1), "+f"(b0), "+f"(b1));
}

// (y0, y1) <- (sg * y0 + o0, sg * y1 + o1) in one packed fma; with sg = +1
// or -1 the product is exact, so each component rounds like y + o or o - y.
__device__ __forceinline__ void f32x2_fma_sign(float& y0, float& y1, float sg, float o0, float o1) {
  asm("{\n .reg .b64 rs, ry, ro, rr;\n mov.b64 rs, {%2, %2};\n mov.b64 ry, {%0, %1};\n mov.b64 ro, {%3, %4};\n"
      " fma.rn.f32x2 rr, rs, ry, ro;\n mov.b64 {%0, %1}, rr;\n}"
      : "+f"(y0), "+f"(y1)
      : "f"(sg), "f"(o0), "f"(o1));
}

// In-place FWHT of the group's vector, stages in increasing stride.  EL is
// the number of elements per lane (lane gl holds elements [gl EL, gl EL + EL)):
// Geo<FHT>::E by default, 128 for the wide query-hash kernel.
//
// With 32 or more elements per lane, elements j and j + EL/2 travel as one
// pair through the packed instructions above, so every stage except h = EL/2
// (which pairs j with j + EL/2 itself) issues half the arithmetic instructions.
template <int FHT, int EL = Geo<FHT>::E>
__device__ __forceinline__ void fwht_group(float (&y)[EL], int gl) {
  constexpr int E = EL;
  constexpr int G = FHT / EL;
  if constexpr (E >= 32) {
    constexpr int HALF = E / 2;
#pragma unroll
    for (int h = 1; h < HALF; h <<= 1) {
#pragma unroll
      for (int i = 0; i < HALF; i += 2 * h) {
#pragma unroll
        for (int j = i; j < i + h; ++j) f32x2_butterfly(y[j], y[j + HALF], y[j + h], y[j + h + HALF]);
      }
    }
#pragma unroll
    for (int j = 0; j < HALF; ++j) {
      const float a = y[j];
      const float b = y[j + HALF];
      y[j] = __fadd_rn(a, b);
      y[j + HALF] = __fsub_rn(a, b);
    }
#pragma unroll
    for (int s = 1; s < G; s <<= 1) {
      const float sg = (gl & s) ? -1.0f : 1.0f;
#pragma unroll
      for (int e = 0; e < HALF; ++e) {
        const float o0 = __shfl_xor_sync(kFullMask, y[e], s);
        const float o1 = __shfl_xor_sync(kFullMask, y[e + HALF], s);
        f32x2_fma_sign(y[e], y[e + HALF], sg, o0, o1);
      }
    }
    return;
  }
#pragma unroll
  for (int h = 1; h < E; h <<= 1) {
#pragma unroll
    for (int i = 0; i < E; i += 2 * h) {
#pragma unroll
      for (int j = i; j < i + h; ++j) {
        const float a = y[j];
        const float b = y[j + h];
        y[j] = __fadd_rn(a, b);
        y[j + h] = __fsub_rn(a, b);
      }
    }
  }
  // Cross-lane stages: the lower lane needs y + o, the upper lane o - y.  Both
  // are fma(sgn, y, o) with sgn = +1 / -1: the product is exact, so the single
  // rounding of the fma equals the rounding of the add or subtract (zeros
  // included: -0 + -0 = -0 and -0 - -0 = +0 either way).
#pragma unroll
  for (int s = 1; s < G; s <<= 1) {
    const float sgn = (gl & s) ? -1.0f : 1.0f;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float o = __shfl_xor_sync(kFullMask, y[e], s);
      y[e] = __fmaf_rn(sgn, y[e], o);
    }
  }
}

// Flip the signs selected by the lane's flip words (bit e % 32 of word
// e / 32 -> element e).
template <int FHT, int EL = Geo<FHT>::E>
__device__ __forceinline__ void flip_signs(float (&y)[EL], const uint32_t (&w)[EL >= 32 ? EL / 32 : 1]) {
#pragma unroll
  for (int e = 0; e < EL; ++e)
    y[e] = __uint_as_float(__float_as_uint(y[e]) ^ (((w[e >> 5] >> (e & 31)) & 1u) << 31));
}

// Three rounds of (sign, FWHT) for one layer of one table.  `flips` points at
// the 3 x WORDS flip words of that (layer, table); bit i % 32 of word i / 32
// flips element i of the vector.
template <int FHT, int EL = Geo<FHT>::E>
__device__ __forceinline__ void hd3_rotate(float (&y)[EL], const uint32_t* flips, int gl) {
  constexpr int WORDS = Geo<FHT>::WORDS;
  constexpr int NW = EL >= 32 ? EL / 32 : 1;  // flip words per lane
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    uint32_t w[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) w[k] = flips[r * WORDS + (FHT < 32 ? 0 : gl * NW + k)];
    flip_signs<FHT, EL>(y, w);
    fwht_group<FHT, EL>(y, gl);
  }
}

// Cross-polytope value of a rotated coordinate: sgn(x)*x with sgn(x) = +1
// for x >= 0 (src/Utilities.h:26-31), and the bucket code r | neg << log2D.
__device__ __forceinline__ float cp_value(float x) { return (x >= 0.0f) ? x : -x; }
__device__ __forceinline__ int cp_code(float x, int r, int log2D) {
  return (x >= 0.0f) ? r : (r | (1 << log2D));
}

// Canonical "a before b": larger value first, then smaller position.
__device__ __forceinline__ bool cp_better(float av, int ar, float bv, int br) {
  return av > bv || (av == bv && ar < br);
}

// Top-`cnt` of cp_value over coordinates r < D, in canonical order,
// computed by the G lanes of the group.  Lane gl == 0 writes out_v[t],
// out_c[t] (bucket code) for t < found and returns found on every lane.
template <int FHT>
__device__ __forceinline__ int group_top_cp(const float (&y)[Geo<FHT>::E], int gl, int D, int log2D,
                                            int cnt, float* out_v, int* out_c) {
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  uint32_t taken = 0;
  int found = 0;
  for (int t = 0; t < cnt; ++t) {
    float bv = -1.0f;
    int br = 0x7fffffff;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int r = gl * E + e;
      const float v = cp_value(y[e]);
      if (r < D && !((taken >> e) & 1u) && cp_better(v, r, bv, br)) {
        bv = v;
        br = r;
      }
    }
#pragma unroll
    for (int s = 1; s < G; s <<= 1) {
      const float ov = __shfl_xor_sync(kFullMask, bv, s);
      const int orr = __shfl_xor_sync(kFullMask, br, s);
      if (cp_better(ov, orr, bv, br)) {
        bv = ov;
        br = orr;
      }
    }
    if (br == 0x7fffffff) break;  // fewer than cnt coordinates
    int code = 0;
    if (br / E == gl) {
      const int e = br - gl * E;
      taken |= 1u << e;
      float x = 0.0f;
#pragma unroll
      for (int k = 0; k < E; ++k)
        if (k == e) x = y[k];
      code = cp_code(x, br, log2D);
    }
    // the owner lane publishes the code
    const int owner = (threadIdx.x & 31 & ~(G - 1)) + br / E;
    code = __shfl_sync(kFullMask, code, owner);
    if (gl == 0) {
      out_v[t] = bv;
      out_c[t] = code;
    }
    ++found;
  }
  return found;
}

// Same result as group_top_cp for cnt <= K: one pass builds each lane's
// top-K (value desc, position asc), then cnt merge rounds take the group's
// best head (a lane can win at most cnt times, so K entries per lane suffice).
template <int FHT, int K>
__device__ __forceinline__ int group_top_cp_small(const float (&y)[Geo<FHT>::E], int gl, int D, int log2D,
                                                  int cnt, float* out_v, int* out_c) {
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  float bv[K];
  int br[K], bc[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    bv[i] = -1.0f;
    br[i] = 0x7fffffff;
    bc[i] = 0;
  }
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int r = gl * E + e;
    const float v = cp_value(y[e]);
    // positions rise within the lane, so a strictly larger value is required
    // to move ahead: equal values keep the earlier position first
    if (r < D && v > bv[K - 1]) {
      bv[K - 1] = v;
      br[K - 1] = r;
      bc[K - 1] = cp_code(y[e], r, log2D);
#pragma unroll
      for (int i = K - 1; i > 0; --i) {
        if (bv[i] > bv[i - 1]) {
          const float tv = bv[i];
          bv[i] = bv[i - 1];
          bv[i - 1] = tv;
          const int tr = br[i];
          br[i] = br[i - 1];
          br[i - 1] = tr;
          const int tc = bc[i];
          bc[i] = bc[i - 1];
          bc[i - 1] = tc;
        }
      }
    }
  }
  int head = 0, found = 0;
  for (int t = 0; t < cnt; ++t) {
    float hv = -1.0f;
    int hr = 0x7fffffff, hc = 0;
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (i == head) {
        hv = bv[i];
        hr = br[i];
        hc = bc[i];
      }
    float wv = hv;
    int wr = hr;
#pragma unroll
    for (int s = 1; s < G; s <<= 1) {
      const float ov = __shfl_xor_sync(kFullMask, wv, s);
      const int orr = __shfl_xor_sync(kFullMask, wr, s);
      if (cp_better(ov, orr, wv, wr)) {
        wv = ov;
        wr = orr;
      }
    }
    if (wr == 0x7fffffff) break;
    const bool mine = (wr == hr);
    const int owner = (threadIdx.x & 31 & ~(G - 1)) + wr / E;
    const int code = __shfl_sync(kFullMask, hc, owner);
    if (mine) ++head;
    if (gl == 0) {
      out_v[t] = wv;
      out_c[t] = code;
    }
    ++found;
  }
  return found;
}

// cnt <= 2 (the query path with one probe per layer, the build with
// iProbes = 1): lane-local top-2 on |y| with compile-time element indices,
// then at most two merge rounds.  |y| compares exactly like sgn(y)*y
// (-0 and +0 are equal); the reported value keeps the reference's sign rule.
template <int FHT>
__device__ __forceinline__ int group_top2_cp(const float (&y)[Geo<FHT>::E], int gl, int D, int log2D, int cnt,
                                             float* out_v, int* out_c) {
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  const int lim = D - gl * E;  // elements of this lane that are coordinates (< D)
  float b0 = -1.0f, b1 = -1.0f, s0 = 0.0f, s1 = 0.0f;
  int e0 = E, e1 = E;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const float v = fabsf(y[e]);
    const bool ok = e < lim;
    const bool g0 = ok && v > b0;
    const bool g1 = ok && v > b1;
    b1 = g0 ? b0 : (g1 ? v : b1);
    s1 = g0 ? s0 : (g1 ? y[e] : s1);
    e1 = g0 ? e0 : (g1 ? e : e1);
    b0 = g0 ? v : b0;
    s0 = g0 ? y[e] : s0;
    e0 = g0 ? e : e0;
  }
  int found = 0;
  bool took0 = false;
  for (int t = 0; t < cnt; ++t) {
    const float hv = took0 ? b1 : b0;
    const int he = took0 ? e1 : e0;
    float wv = hv;
    int wr = he < E ? gl * E + he : 0x7fffffff;
    const int myr = wr;
#pragma unroll
    for (int s = 1; s < G; s <<= 1) {
      const float ov = __shfl_xor_sync(kFullMask, wv, s);
      const int orr = __shfl_xor_sync(kFullMask, wr, s);
      if (cp_better(ov, orr, wv, wr)) {
        wv = ov;
        wr = orr;
      }
    }
    if (wr == 0x7fffffff) break;
    const bool mine = (wr == myr);
    const float sy = took0 ? s1 : s0;
    const int owner = (threadIdx.x & 31 & ~(G - 1)) + wr / E;
    const float wy = __shfl_sync(kFullMask, sy, owner);
    if (mine) took0 = true;
    if (gl == 0) {
      out_v[t] = cp_value(wy);
      out_c[t] = cp_code(wy, wr, log2D);
    }
    ++found;
  }
  return found;
}

// The top-1 of cp_value over coordinates r < D in canonical order (lane gl
// == 0 writes out_v[0], out_c[0]) and whether it is strict: true when no
// other coordinate has an equal value and D >= 2.  That is exactly the
// condition under which group_top2_cp's first two entries are in strict
// order, so callers that keep one entry per layer (m1 = 1, iProbes = 1) use
// it in place of the top-2 with the same tie replay.  Two passes: the group
// maximum of |y| (one max per element), then the count, first position and
// signed value of the elements equal to it.
template <int FHT, int EL = Geo<FHT>::E>
__device__ __forceinline__ bool group_top1_strict(const float (&y)[EL], int gl, int D, int log2D,
                                                  float* out_v, int* out_c) {
  constexpr int E = EL;
  constexpr int G = FHT / EL;
  const int lim = D - gl * E;  // elements of this lane that are coordinates (< D)
  int cnt = 0, pos = 0;
  float sy = 0.0f;
  float lm = -1.0f;
  if (lim >= E) {
#pragma unroll
    for (int e = 0; e < E; ++e) lm = fmaxf(lm, fabsf(y[e]));
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (e < lim) lm = fmaxf(lm, fabsf(y[e]));
  }
  float gm = lm;
#pragma unroll
  for (int s = 1; s < G; s <<= 1) gm = fmaxf(gm, __shfl_xor_sync(kFullMask, gm, s));
#pragma unroll
  for (int e = E - 1; e >= 0; --e) {
    const bool eq = e < lim && fabsf(y[e]) == gm;
    cnt += eq ? 1 : 0;
    pos = eq ? e : pos;
    sy = eq ? y[e] : sy;
  }
  int tot = cnt;
#pragma unroll
  for (int s = 1; s < G; s <<= 1) tot += __shfl_xor_sync(kFullMask, tot, s);
  const int base = (int)(threadIdx.x & 31) & ~(G - 1);
  const unsigned gbits = (__ballot_sync(kFullMask, cnt > 0) >> base) & (G == 32 ? kFullMask : ((1u << G) - 1u));
  const int owner_gl = gbits ? __ffs(gbits) - 1 : 0;
  const float wy = __shfl_sync(kFullMask, sy, base + owner_gl);
  const int wpos = __shfl_sync(kFullMask, pos, base + owner_gl);
  if (gl == 0) {
    out_v[0] = cp_value(wy);
    out_c[0] = cp_code(wy, owner_gl * E + wpos, log2D);
  }
  return tot == 1 && D >= 2;
}

// Dispatch: the single-pass selection when cnt is small, the round-based one
// otherwise.
template <int FHT>
__device__ __forceinline__ int group_top_cp_auto(const float (&y)[Geo<FHT>::E], int gl, int D, int log2D, int cnt,
                                                 float* out_v, int* out_c) {
  if (cnt <= 2) return group_top2_cp<FHT>(y, gl, D, log2D, cnt, out_v, out_c);
  if (cnt <= 4) return group_top_cp_small<FHT, 4>(y, gl, D, log2D, cnt, out_v, out_c);
  return group_top_cp<FHT>(y, gl, D, log2D, cnt, out_v, out_c);
}

// Top-cnt selection with the strictness check every caller applies: true
// when the group found cnt entries in strictly decreasing order (no tie can
// change the kept set), false when the reference's heap scan must be
// replayed.  keep is the number of entries the caller uses (cnt = keep + 1
// unless D is smaller); keeping one (m1 = 1 or iProbes = 1) takes the
// two-pass strict top-1, which writes only entry 0.
template <int FHT>
__device__ __forceinline__ bool group_top_cp_checked(const float (&y)[Geo<FHT>::E], int gl, int D, int log2D,
                                                     int keep, int cnt, float* out_v, int* out_c) {
  if (keep == 1 && cnt == 2) {
    const bool ok = group_top1_strict<FHT>(y, gl, D, log2D, out_v, out_c);
    __syncwarp();
    return ok;
  }
  const int f = group_top_cp_auto<FHT>(y, gl, D, log2D, cnt, out_v, out_c);
  __syncwarp();
  bool ok = (f == cnt);
  for (int t = 1; t < cnt; ++t)
    if (ok && !(out_v[t - 1] > out_v[t])) ok = false;
  return ok;
}

// Exact replay of the reference's per-layer top-p scan (FalconnPP.cpp:103-156,
// :386-452) over the dumped coordinates y[0..D).  Writes vec[0..p) in the
// reference's order (vec[0] = largest).  hv/hi are scratch of size p.
__device__ __forceinline__ void replay_layer_topp(const float* y, int D, int log2D, int p, float* hv,
                                                  int* hi, float* vec_v, int* vec_c) {
  int n = 0;
  for (int r = 0; r < D; ++r) {
    const float x = y[r];
    topp_offer<int>(hv, hi, n, p, cp_value(x), cp_code(x, r, log2D));
  }
  for (int k = p - 1; k >= 0; --k) {
    vec_v[k] = hv[0];
    vec_c[k] = hi[0];
    heap_pop<true, int>(hv, hi, n);
  }
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024,
// multiple of 32).  `tmp` holds 32 ints of shared memory.  Returns the
// exclusive prefix; *total receives the block sum.
__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* tmp, long long* total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(kFullMask, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < nwarps ? tmp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(kFullMask, w, o);
      if (lane >= o) w += y;
    }
    tmp[lane] = w;  // inclusive prefix over warps
  }
  __syncthreads();
  const long long before = (warp > 0 ? tmp[warp - 1] : 0) + x - v;
  if (total) *total = tmp[nwarps - 1];
  __syncthreads();
  return before;
}

// Ascending bitonic sort (all comparators ascending, length need not be a
// power of two: positions >= len act as +infinity and never move).
static __device__ __noinline__ void block_bitonic_sort_u32(uint32_t* key, uint32_t* val, int len) {
  int N = 1;
  while (N < len) N <<= 1;
  for (int k = 2; k <= N; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
        int lo, hi;
        if (j == (k >> 1)) {  // mirror step of the stage
          const int blk = t / j;
          const int off = t - blk * j;
          lo = blk * k + off;
          hi = blk * k + k - 1 - off;
        } else {
          const int blk = t / j;
          lo = blk * 2 * j + (t - blk * j);
          hi = lo + j;
        }
        if (hi < len) {
          const uint32_t a = key[lo], b = key[hi];
          if (a > b) {
            key[lo] = b;
            key[hi] = a;
            const uint32_t va = val[lo];
            val[lo] = val[hi];
            val[hi] = va;
          }
        }
      }
      __syncthreads();
    }
  }
}

__device__ __forceinline__ uint32_t ord_key_inv_dev(uint32_t k) {
  return (k & 0x80000000u) ? (k ^ 0x80000000u) : ~k;
}

}  // namespace fpp
