// fpp_hash_verify.cu — the query hash of the batched form with the rotation
// on the tensor cores and the reference's FP32 arithmetic wherever it can
// decide a probe (k_query_hash_verified).  fhtDim 256, one probe per table
// (2 qProbes <= L).
//
// One block of two warps per query (the warps split the tables, and block
// barriers join them; half-query work units keep the last wave short):
//   1. every table's two layers rotate on the tensor cores (tc_rotate_top1:
//      FP16 operands, FP32 accumulation) with the query scaled by a power of
//      two; each table gets an approximate score s~ = v1~ + v2~ and code;
//   2. every approximate score lies within delta of the table's exact FP32
//      score (the bound below, from the query's norm), so a table whose s~ is
//      below s* - 2 delta (s* = the qProbes-th largest s~) is below every
//      exact score of the qProbes best tables and can neither be probed nor
//      tie with a probe;
//   3. the other tables (usually a handful) are hashed again in the
//      reference's FP32 arithmetic (the plain path's hd3_rotate and strict
//      top-1, eight groups of 8 lanes), and their exact scores and codes
//      replace the approximate ones;
//   4. when those exact scores tie at the cut, or an approximate score is not
//      finite, every table of the query is hashed exactly, so the probe cut's
//      heap replay sees the reference's values.
// The probe cut (k_probe_cut) then ranks the lists: the same probes, with the
// same scores, as the exact hash for every query (FalconnPP.cpp:358-582).
//
// The bound.  With the query scaled by a power of two to ||x_s|| in [4, 8),
// a rotation round of the tensor-core path rounds its input and its
// intermediate product to FP16: six roundings, each of relative error 2^-11
// per element (2^-25 absolute below the FP16 normal range, 2^-21 in l2 over
// 256 elements).  The rest of the rotation is linear and scales l2 norms by
// exactly 4 per 16-point transform, so each rounding's error vector reaches
// the output with l2 norm at most 2^-11 ||y|| (||y|| = 4096 ||x_s||).  Below
// the normal range the absolute part is taken as if the tensor cores flushed
// FP16 inputs below 2^-14 to zero: 2^-10 in l2 per rounding, times at most
// 4^6 + 4^5 + ... + 4 < 5462 over the six, under 6 in the scaled output.
// Every intermediate
// then stays below 1024 * 8 = 8192 in magnitude (no FP16 overflow).  On top:
// the FP32 accumulation of each of the six products (taken as 2^-13 of
// ||y||, eight times the bound for 16 exact products summed with truncation),
// the key truncation of tc_rotate_top1 (2^-14 of the value) and the exact
// path's own FP32 rounding (24 butterfly stages, 2^-18 of ||y||).  Any
// coordinate, and so the best coordinate's value, moves by at most the
// error's l2 norm; delta per table = 2 layers x 2 (safety) x the sum.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "fpp_device.cuh"
#include "fpp_query.h"
#include "fpp_tc_rotate.cuh"

namespace fpp {
namespace {

constexpr int kVWarps = 2;          // warps per block; one block per query
constexpr int kVThreads = kVWarps * 32;
constexpr int kVMaxL = 128;         // tables per query
constexpr int kVFht = 256;
constexpr int kVGroups = 4 * kVWarps;  // 8-lane groups per block for the exact hash

// relative error per layer (of ||y||) and absolute error per layer (scaled
// units), before the factor 2 x 2
constexpr float kVRelLayer = 6.0f / 2048.0f + 6.0f / 8192.0f + 1.0f / 16384.0f + 1.0f / 262144.0f;
constexpr float kVAbsLayer = 6.0f;

struct VerifyArgs {
  const float* Q;                   // nq x d raw queries
  int nq, d;
  const uint32_t* flips;            // exact path: [2][L][3][8]
  const uint32_t* tflips;           // tensor-core path: the same words per rotation view
  int L, D, log2D;
  uint32_t NB;
  const int* q_qprobes;             // per-query qProbes (nullable: qp_max)
  int qp_max;
  float* list_v;                    // query q's L entries at list_v / list_b + q * stride
  uint32_t* list_b;
  long long stride;
  unsigned* n_exact;                // nullable: tables hashed exactly, summed over queries
};

struct VerifySmem {
  float qs[kVFht];               // the query, zero padded past d
  float sv[kVMaxL];              // per table: score (approximate or exact)
  uint32_t sb[kVMaxL];           // per table: global bucket id
  int rl[kVMaxL];                // tables to hash exactly
  float ydump[kVGroups][kVFht];  // exact path: the dump a tie replays
  float lv[kVGroups][2];         // exact path: per group, per layer
  int lc[kVGroups][2];
  float hv[kVGroups];            // replay heap (one entry)
  int hi[kVGroups];
};

// A non-negative score as an ordered key: its bits without the sign (a -0
// sorts as +0), which order as the values.
__device__ __forceinline__ uint32_t score_key(float v) { return __float_as_uint(v) & 0x7fffffffu; }

// The p-th largest (1 <= p <= n) of the warp's n <= 128 non-negative scores
// v[0..n), as its key: the largest T with #{i : key(v[i]) >= T} >= p, bit by
// bit.
__device__ __forceinline__ uint32_t warp_pth_largest(const float* v, int n, int p, int lane) {
  uint32_t k[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int i = lane + 32 * j;
    k[j] = i < n ? score_key(v[i]) : 0u;
  }
  uint32_t t = 0u;
#pragma unroll 1
  for (int b = 30; b >= 0; --b) {
    const uint32_t c = t | (1u << b);
    int cnt = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) cnt += __popc(__ballot_sync(kFullMask, k[j] >= c));
    if (cnt >= p) t = c;
  }
  return t;
}

// Hash exactly, in the plain path's arithmetic, the tables whose bit is set
// in mask[0..4) (table lane + 32 j <-> bit lane of mask[j]; the same mask in
// both warps); eight tables at a time, one per 8-lane group of the block,
// both layers.  Writes their exact scores and bucket ids into sv / sb
// (FalconnPP.cpp:358-485 for one probe per table).  Called by the whole
// block: it starts and ends with a block barrier.
__device__ __forceinline__ void exact_tables(const VerifyArgs& a, VerifySmem& sm, int warp, int lane,
                                             const uint32_t (&mask)[4]) {
  int* rl = sm.rl;
  int base = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (warp == 0 && ((mask[j] >> lane) & 1u)) rl[base + __popc(mask[j] & ((1u << lane) - 1u))] = lane + 32 * j;
    base += __popc(mask[j]);
  }
  __syncthreads();
  const int nr = base;
  const int gw = lane >> 3, gl = lane & 7;
  const int grp = warp * 4 + gw;
  const unsigned gmask = 0xffu << (lane & ~7);
  float xr[32];
#pragma unroll
  for (int e = 0; e < 32; ++e) xr[e] = sm.qs[gl * 32 + e];
  for (int r0 = 0; r0 < nr; r0 += kVGroups) {  // uniform over the block
    const bool act = r0 + grp < nr;
    const int l = rl[act ? r0 + grp : r0];
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
      float y[32];
#pragma unroll
      for (int e = 0; e < 32; ++e) y[e] = xr[e];
      hd3_rotate<kVFht>(y, a.flips + ((size_t)(layer * a.L + l) * 3) * 8, gl);
      float* ov = &sm.lv[grp][layer];
      int* oc = &sm.lc[grp][layer];
      const bool ok = group_top1_strict<kVFht>(y, gl, a.D, a.log2D, ov, oc);
      __syncwarp();
      if (!ok) {
        // a tie for the best coordinate (or D < 2): the reference's scan
        float* yd = sm.ydump[grp];
#pragma unroll
        for (int e = 0; e < 32; ++e) yd[gl * 32 + e] = y[e];
        __syncwarp(gmask);
        if (gl == 0) replay_layer_topp(yd, a.D, a.log2D, 1, &sm.hv[grp], &sm.hi[grp], ov, oc);
        __syncwarp(gmask);
      }
    }
    __syncwarp();
    if (gl == 0 && act) {
      sm.sv[l] = __fadd_rn(sm.lv[grp][0], sm.lv[grp][1]);
      sm.sb[l] = (uint32_t)l * a.NB + (uint32_t)(sm.lc[grp][0] * 2 * a.D + sm.lc[grp][1]);
    }
    __syncwarp();
  }
  __syncthreads();
}

// Every branch below that contains a block barrier depends only on values
// both warps compute alike from shared memory (the norm, the scores, the
// masks), so both warps take it.
__global__ void __launch_bounds__(kVThreads, 8) k_query_hash_verified(VerifyArgs a) {
  __shared__ VerifySmem sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = blockIdx.x;  // one query per block
  const int L = a.L;
  float* qs = sm.qs;
  float* sv = sm.sv;
  uint32_t* sb = sm.sb;
  for (int i = threadIdx.x; i < kVFht; i += kVThreads) qs[i] = i < a.d ? __ldg(a.Q + (size_t)q * a.d + i) : 0.0f;
  __syncthreads();
  float ss = 0.0f;  // the same sum, in the same order, in both warps
  for (int i = lane; i < kVFht; i += 32) ss = fmaf(qs[i], qs[i], ss);
#pragma unroll
  for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(kFullMask, ss, o);
  const float nrm = sqrtf(ss);
  // far from FP32's range limits (and finite), the bound holds; otherwise
  // every table is hashed exactly
  bool all = !(nrm > 0x1p-60f && nrm < 0x1p60f);
  uint32_t valid[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int lo = 32 * j;
    valid[j] = L - lo >= 32 ? kFullMask : (L - lo <= 0 ? 0u : (1u << (L - lo)) - 1u);
  }
  const int qp = min(max(a.q_qprobes ? __ldg(a.q_qprobes + q) : a.qp_max, 1), a.qp_max);
  uint32_t first[4] = {valid[0], valid[1], valid[2], valid[3]};
  if (!all) {
    int ex = 0;
    frexpf(nrm, &ex);  // nrm in [2^(ex-1), 2^ex)
    const float scale = __int_as_float((127 + 3 - ex) << 23);  // ||x scale|| in [4, 8)
    const float inv = __int_as_float((127 - 3 + ex) << 23);
    const H16Frags hf(lane);
    uint32_t qb[2][2];
    tc_query_frags(qs, scale, lane, qb);
    // the warps take alternate pairs of tables
    for (int l = 2 * warp; l < L; l += 2 * kVWarps) {
      const int l2 = l + 1 < L ? l + 1 : l;
      const uint32_t* const tw[4] = {a.tflips + (size_t)l * 24, a.tflips + (size_t)(L + l) * 24,
                                     a.tflips + (size_t)l2 * 24, a.tflips + (size_t)(L + l2) * 24};
      float v[4];
      int c[4];
      tc_rotate_top1<4>(qb, tw, hf, lane, a.D, a.log2D, v, c);
      if (lane == 0) {
        sv[l] = (v[0] + v[1]) * inv;
        sb[l] = (uint32_t)l * a.NB + (uint32_t)(c[0] * 2 * a.D + c[1]);
        if (l2 != l) {
          sv[l2] = (v[2] + v[3]) * inv;
          sb[l2] = (uint32_t)l2 * a.NB + (uint32_t)(c[2] * 2 * a.D + c[3]);
        }
      }
    }
    __syncthreads();
    // delta per table in the query's own units; the norm rounded up
    const float ny = nrm * (1.0f + 0x1p-12f) * 4096.0f;
    const float delta = 4.0f * (kVRelLayer * ny + kVAbsLayer * inv);
    bool fin = true;
    for (int i = lane; i < L; i += 32) fin = fin && isfinite(sv[i]);
    fin = __all_sync(kFullMask, fin);
    if (!fin) {
      all = true;
    } else {
      const float s_cut = __uint_as_float(warp_pth_largest(sv, L, qp, lane));  // >= +0
      const float thr = s_cut - 2.0f * delta;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = lane + 32 * j;
        first[j] = __ballot_sync(kFullMask, i < L && sv[i < L ? i : 0] >= thr) & valid[j];
      }
    }
  }
  exact_tables(a, sm, warp, lane, first);
  if (!all) {
    // the exact scores of every table that can reach the cut are in place; a
    // tie at the cut makes the probe cut replay the reference's heap over all
    // L entries, so then the rest are hashed exactly too
    const uint32_t e_cut = warp_pth_largest(sv, L, qp, lane);
    int ge = 0;
    for (int i = lane; i < L; i += 32) ge += score_key(sv[i]) >= e_cut ? 1 : 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) ge += __shfl_xor_sync(kFullMask, ge, o);
    if (ge > qp) {
      uint32_t rest[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) rest[j] = valid[j] & ~first[j];
      exact_tables(a, sm, warp, lane, rest);
      all = true;
    }
  }
  if (a.n_exact && threadIdx.x == 0) {
    unsigned n = 0;
    if (all) {
      n = (unsigned)L;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) n += (unsigned)__popc(first[j]);
    }
    atomicAdd(a.n_exact, n);
  }
  float* ov = a.list_v + (size_t)q * a.stride;
  uint32_t* ob = a.list_b + (size_t)q * a.stride;
  for (int i = threadIdx.x; i < L; i += kVThreads) {
    ov[i] = sv[i];
    ob[i] = sb[i];
  }
}

}  // namespace

long long hash_verified_wave_queries() {
  int dev = 0, nsm = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_query_hash_verified, kVThreads, 0) != cudaSuccess)
    return 0;
  return (long long)nsm * per_sm;  // one query per block
}

cudaError_t hash_lists_verified(const Params& P, const DeviceIndex& di, const float* Q, int nq, const int* q_qprobes,
                                int qp_max, float* list_v, uint32_t* list_b, long long stride, unsigned* n_exact,
                                cudaStream_t s) {
  const int L = P.n_tables, D = P.n_proj;
  if (P.fhtDim != kVFht || !di.tflips || L < 1 || L > kVMaxL || qp_max < 1 || 2 * qp_max > L || stride < L)
    return cudaErrorInvalidValue;
  if (nq <= 0) return cudaSuccess;
  int log2D = 0;
  while ((1 << log2D) < D) ++log2D;
  VerifyArgs a;
  a.Q = Q;
  a.nq = nq;
  a.d = P.n_features;
  a.flips = di.flips;
  a.tflips = di.tflips;
  a.L = L;
  a.D = D;
  a.log2D = log2D;
  a.NB = 4u * (uint32_t)D * (uint32_t)D;
  a.q_qprobes = q_qprobes;
  a.qp_max = qp_max;
  a.list_v = list_v;
  a.list_b = list_b;
  a.stride = stride;
  a.n_exact = n_exact;
  k_query_hash_verified<<<(unsigned)nq, kVThreads, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace fpp
