// fpp_query.cu — the query path (FalconnPP::query2Layers_1D,
// src/FalconnPP.cpp:310-707) as three kernels per batch of queries:
//
//   k_query_hash      one group of FHT/32 lanes per (query, table): the same
//                     HD3 rotations as the build, top-m1 codes per layer,
//                     top-m of the m1 x m1 two-layer pairs -> the table's
//                     probe list sorted by score (FalconnPP.cpp:358-531);
//   k_probe_select    one block per query: the global top-qProbes of the
//                     L x m lists (the reference pops a max-heap, :540-611),
//                     by radix selection on the scores; a tie at the cut
//                     replays the reference's heap exactly;
//   k_gather_rerank   persistent blocks, one query at a time per block: gather
//                     the ids of the probed buckets, deduplicate them with a
//                     per-block bitset in global scratch (set with atomicOr,
//                     cleared again from the unique list), FP32 dot products
//                     of the unique rows (warp per row, coalesced float4), and
//                     the top-k (FalconnPP.cpp:552-673).  Ties that could make
//                     the reference's min-heap answer differ from
//                     (score desc, id asc) are replayed exactly.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "fpp_device.cuh"
#include "fpp_query.h"

namespace fpp {

constexpr int kMaxM1 = 64;        // per-layer probes kept per table

// ------------------------------------------------------------ query hashing
struct QHashArgs {
  const float* Q;  // nq x d (raw queries, not centred: FalconnPP.cpp:350)
  int nq, d;
  const uint32_t* flips;
  int L, D, log2D;
  uint32_t NB;
  int m, m1;
  float* list_v;      // [nq][L][m]
  uint32_t* list_b;   // [nq][L][m] global bucket ids
  // batched form (nullable): per-query qProbes, clamped to [1, qp_max]; each
  // query then keeps its own m = ceil(2 qProbes / L) probes per table at
  // list_v + q * stride + l * m (m above is the largest, stride = L * m)
  const int* q_qprobes;
  int qp_max;
  long long stride;
};

template <int FHT>
struct QHashSmem {
  static constexpr int G = Geo<FHT>::G;
  static constexpr int GROUPS = 128 / G;
  static constexpr size_t per_group = FHT * 4 + 2 * (kMaxM1 + 1) * 8 + kMaxM1 * 8;
  static constexpr size_t bytes = GROUPS * per_group;
};

template <int FHT>
__global__ void __launch_bounds__(128, 4) k_query_hash(QHashArgs a, float* heap_v, int* heap_i) {
  constexpr int E = Geo<FHT>::E;
  constexpr int G = Geo<FHT>::G;
  constexpr int WORDS = Geo<FHT>::WORDS;
  constexpr int GROUPS = QHashSmem<FHT>::GROUPS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);
  const int grp = threadIdx.x / G;
  const unsigned gmask = (G == 32) ? kFullMask : (((1u << G) - 1u) << (lane & ~(G - 1)));
  unsigned char* gs = smem_raw + grp * QHashSmem<FHT>::per_group;
  float* ydump = reinterpret_cast<float*>(gs);
  float* lv1 = reinterpret_cast<float*>(gs + FHT * 4);
  int* lc1 = reinterpret_cast<int*>(lv1 + (kMaxM1 + 1));
  float* lv2 = reinterpret_cast<float*>(lc1 + (kMaxM1 + 1));
  int* lc2 = reinterpret_cast<int*>(lv2 + (kMaxM1 + 1));
  float* hv = reinterpret_cast<float*>(lc2 + (kMaxM1 + 1));
  int* hi = reinterpret_cast<int*>(hv + kMaxM1);

  const int m_all = a.m, m1_all = a.m1;
  const long long items = (long long)a.nq * a.L;
  const long long groups_total = (long long)gridDim.x * GROUPS;
  const long long n_iter = (items + groups_total - 1) / groups_total;
  const long long gid = (long long)blockIdx.x * GROUPS + grp;
  // per-group pair heap (size m) lives in global scratch when m is large
  float* ph_v = heap_v + gid * (long long)m_all;
  int* ph_i = heap_i + gid * (long long)m_all;
  for (long long it = 0; it < n_iter; ++it) {
    const long long item = it * groups_total + gid;
    const bool active = item < items;
    const long long itm = active ? item : 0;
    const int q = (int)(itm / a.L);
    const int l = (int)(itm - (long long)q * a.L);
    int m = m_all, m1 = m1_all;
    if (a.q_qprobes) {
      const int qp = min(max(a.q_qprobes[q], 1), a.qp_max);
      m = (2 * qp + a.L - 1) / a.L;  // ceil(2.0 * qProbes / L)
      m1 = 0;
      while (m1 * m1 < m) ++m1;      // ceil(sqrt(m))
    }
    // the selection runs warp-uniform (its shuffles span the warp): the
    // largest m1 of the warp's groups; a group with a smaller m1 then checks
    // strictness over more entries than it needs, which can only add replays
    const int m1w = a.q_qprobes ? __reduce_max_sync(kFullMask, m1) : m1;
    const int cnt = min(m1w + 1, a.D);
    float xr[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = gl * E + e;
      xr[e] = (active && idx < a.d) ? __ldg(a.Q + (size_t)q * a.d + idx) : 0.0f;
    }
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {
      float y[E];
#pragma unroll
      for (int e = 0; e < E; ++e) y[e] = xr[e];
      hd3_rotate<FHT>(y, a.flips + ((size_t)(layer * a.L + l) * 3) * WORDS, gl);
      float* lv = layer == 0 ? lv1 : lv2;
      int* lc = layer == 0 ? lc1 : lc2;
      const bool ok = group_top_cp_checked<FHT>(y, gl, a.D, a.log2D, m1w, cnt, lv, lc);
      if (!ok) {
#pragma unroll
        for (int e = 0; e < E; ++e) ydump[gl * E + e] = y[e];
        __syncwarp(gmask);
        if (gl == 0) replay_layer_topp(ydump, a.D, a.log2D, m1, hv, hi, lv, lc);
        __syncwarp(gmask);
      }
    }
    if (gl == 0 && active) {
      float* ov = a.list_v + (size_t)q * a.stride + (size_t)l * m;
      uint32_t* ob = a.list_b + (size_t)q * a.stride + (size_t)l * m;
      const uint32_t tbase = (uint32_t)l * a.NB;
      const int twoD = 2 * a.D;
      if (m == 1) {
        // sums are monotone in both arguments, so pair (0,0) is a maximum and
        // a later pair never replaces it (FalconnPP.cpp:478-485)
        ov[0] = __fadd_rn(lv1[0], lv2[0]);
        ob[0] = tbase + (uint32_t)(lc1[0] * twoD + lc2[0]);
      } else {
        // FalconnPP.cpp:455-487 then the drain into positions m-1..0 (:508-527)
        int hn = 0;
        for (int i = 0; i < m1; ++i)
          for (int j = 0; j < m1; ++j)
            topp_offer<int>(ph_v, ph_i, hn, m, __fadd_rn(lv1[i], lv2[j]), lc1[i] * twoD + lc2[j]);
        for (int j = m - 1; j >= 0; --j) {
          ov[j] = ph_v[0];
          ob[j] = tbase + (uint32_t)ph_i[0];
          heap_pop<true, int>(ph_v, ph_i, hn);
        }
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------ probe selection
struct SelectArgs {
  const float* list_v;
  const uint32_t* list_b;
  int nq, L, m, qProbes;
  const uint32_t* bucket_off;
  uint32_t* probes;       // [nq][qProbes] global bucket ids
  float* probe_v;         // optional [nq][qProbes]
  long long* cand;        // [nq] candidates incl. duplicates
  int* empty;             // [nq] empty probed buckets
  int* n_tie;             // count of queries that took the exact replay
};

// Block of 256 threads per query.
__global__ void __launch_bounds__(256) k_probe_select(SelectArgs a, float* hv_g, int* hi_g) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_prefix, s_remaining;
  __shared__ unsigned s_gt, s_ge;
  __shared__ long long tmp[32];
  const int M = a.L * a.m;
  const int Qp = a.qProbes;
  for (int q = blockIdx.x; q < a.nq; q += gridDim.x) {
    const float* lv = a.list_v + (size_t)q * M;
    const uint32_t* lb = a.list_b + (size_t)q * M;
    uint32_t* out = a.probes + (size_t)q * Qp;
    uint32_t t = 0;  // key of the qProbes-th largest score
    bool exact = true;
    if (Qp < M) {
      if (threadIdx.x == 0) {
        s_prefix = 0;
        s_remaining = (uint32_t)Qp;
      }
      uint32_t mask = 0;
      for (int shift = 24; shift >= 0; shift -= 8) {
        hist[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t pre = s_prefix;
        for (int i = threadIdx.x; i < M; i += blockDim.x) {
          const uint32_t k = ord_key(lv[i]);
          if ((k & mask) == pre) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          uint32_t rem = s_remaining;
          int dg = 255;
          for (; dg > 0; --dg) {
            if (hist[dg] >= rem) break;
            rem -= hist[dg];
          }
          s_prefix = pre | ((uint32_t)dg << shift);
          s_remaining = rem;
        }
        mask |= 255u << shift;
        __syncthreads();
      }
      t = s_prefix;
      if (threadIdx.x == 0) {
        s_gt = 0;
        s_ge = 0;
      }
      __syncthreads();
      unsigned gt = 0, ge = 0;
      for (int i = threadIdx.x; i < M; i += blockDim.x) {
        const uint32_t k = ord_key(lv[i]);
        gt += k > t;
        ge += k >= t;
      }
      atomicAdd(&s_gt, gt);
      atomicAdd(&s_ge, ge);
      __syncthreads();
      exact = (s_ge == (unsigned)Qp);
    }
    if (exact) {
      // the selected set is {score >= t}; keep list order (table, rank)
      long long run = 0;
      __syncthreads();
      for (int base = 0; base < M; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const bool take = i < M && (Qp >= M || ord_key(lv[i]) >= t);
        long long tot;
        const long long pos = block_exclusive_scan(take ? 1 : 0, tmp, &tot) + run;
        if (take) {
          out[pos] = lb[i];
          if (a.probe_v) a.probe_v[(size_t)q * Qp + pos] = lv[i];
        }
        run += tot;
      }
    } else {
      // replay FalconnPP.cpp:540-582 exactly: max-heap of each table's head
      if (threadIdx.x == 0) {
        atomicAdd(a.n_tie, 1);
        float* hv = hv_g + (size_t)blockIdx.x * a.L;
        int* hi = hi_g + (size_t)blockIdx.x * 2 * a.L;
        int* track = hi + a.L;
        int n = 0;
        for (int l = 0; l < a.L; ++l) {
          heap_push<false, int>(hv, hi, n, lv[(size_t)l * a.m], l * a.m);
          track[l] = 0;
        }
        for (int pc = 0; pc < Qp; ++pc) {
          const int pos = hi[0];
          heap_pop<false, int>(hv, hi, n);
          out[pc] = lb[pos];
          if (a.probe_v) a.probe_v[(size_t)q * Qp + pc] = lv[pos];
          const int tb = pos / a.m;
          track[tb]++;
          if (track[tb] < a.m) heap_push<false, int>(hv, hi, n, lv[(size_t)tb * a.m + track[tb]], tb * a.m + track[tb]);
        }
      }
    }
    __syncthreads();
    // candidates incl. duplicates and empty buckets (verbose statistics)
    long long c = 0;
    int e = 0;
    for (int i = threadIdx.x; i < Qp; i += blockDim.x) {
      const uint32_t g = out[i];
      const uint32_t sz = a.bucket_off[g + 1] - a.bucket_off[g];
      c += sz;
      e += sz == 0;
    }
    long long tc, te;
    block_exclusive_scan(c, tmp, &tc);
    block_exclusive_scan(e, tmp, &te);
    if (threadIdx.x == 0) {
      a.cand[q] = tc;
      a.empty[q] = (int)te;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ gather + rerank
struct RerankArgs {
  const uint32_t* probes;  // [nq][qProbes]
  int nq, qProbes, k;
  const uint32_t* bucket_off;
  const int32_t* ids;
  const float* Xc;
  int ld;
  const float* Q;  // nq x d
  int d;
  int n;
  // per-block scratch (global memory beyond inputs and outputs)
  uint32_t* bitset;        // [grid][nwords]
  long long nwords;
  uint32_t* uniq;          // [grid][cap]
  uint32_t* score;         // [grid][cap] float bits
  long long cap;
  int32_t* out;            // [nq][k]
  float* out_v;            // optional [nq][k]
  long long* n_unique;     // optional [nq]
  int32_t* cand_dump;      // optional [nq][cap]
  int* n_tie;
};

constexpr int kRrThreads = 256;
constexpr int kRrWarps = kRrThreads / 32;
constexpr int kProbeChunk = 2048;
constexpr int kMaxK = 1024;
constexpr int kMaxChunksPerLane = 8;  // d <= 1024

// canonical dot: lane t accumulates float4 chunks t, t+32, ... (fmaf, element
// order), then the xor butterfly 16..1 — the same order as the oracle
__device__ __forceinline__ float warp_dot_rows(const float4* qc, int nchunk, const float* row, int lane) {
  float acc = 0.0f;
  const float4* r4 = reinterpret_cast<const float4*>(row);
#pragma unroll
  for (int i = 0; i < kMaxChunksPerLane; ++i) {
    const int c = lane + 32 * i;
    if (c < nchunk) {
      const float4 x = __ldg(r4 + c);
      acc = fmaf(qc[i].x, x.x, acc);
      acc = fmaf(qc[i].y, x.y, acc);
      acc = fmaf(qc[i].z, x.z, acc);
      acc = fmaf(qc[i].w, x.w, acc);
    }
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(kFullMask, acc, o));
  return acc;
}

__global__ void __launch_bounds__(kRrThreads) k_gather_rerank(RerankArgs a) {
  __shared__ uint32_t s_po[kProbeChunk];
  __shared__ uint32_t s_ps[kProbeChunk];
  __shared__ uint32_t hist[256];
  __shared__ unsigned s_u, s_gt, s_ge, s_sel;
  __shared__ uint32_t s_prefix, s_remaining;
  __shared__ unsigned long long s_top[kMaxK];
  __shared__ float s_hv[kMaxK];
  __shared__ int s_hi[kMaxK];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  uint32_t* bits = a.bitset + (size_t)blockIdx.x * a.nwords;
  uint32_t* uq = a.uniq + (size_t)blockIdx.x * a.cap;
  uint32_t* sc = a.score + (size_t)blockIdx.x * a.cap;
  const int nchunk = (a.d + 3) / 4;
  const int k = a.k;

  for (int q = blockIdx.x; q < a.nq; q += gridDim.x) {
    if (tid == 0) s_u = 0;
    __syncthreads();
    // 1. gather + dedupe (FalconnPP.cpp:556-606)
    const uint32_t* pr = a.probes + (size_t)q * a.qProbes;
    for (int p0 = 0; p0 < a.qProbes; p0 += kProbeChunk) {
      const int np = min(kProbeChunk, a.qProbes - p0);
      for (int i = tid; i < np; i += kRrThreads) {
        const uint32_t g = pr[p0 + i];
        const uint32_t o = a.bucket_off[g];
        s_po[i] = o;
        s_ps[i] = a.bucket_off[g + 1] - o;
      }
      __syncthreads();
      for (int p = warp; p < np; p += kRrWarps) {
        const uint32_t o = s_po[p], sz = s_ps[p];
        for (uint32_t i = lane; i < ((sz + 31u) & ~31u); i += 32) {
          bool fresh = false;
          uint32_t id = 0;
          if (i < sz) {
            id = (uint32_t)a.ids[o + i];
            const uint32_t bit = 1u << (id & 31u);
            fresh = (atomicOr(bits + (id >> 5), bit) & bit) == 0u;
          }
          const unsigned bal = __ballot_sync(kFullMask, fresh);
          if (bal) {
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(&s_u, (unsigned)__popc(bal));
            base = __shfl_sync(kFullMask, base, 0);
            if (fresh) uq[base + __popc(bal & ((1u << lane) - 1u))] = id;
          }
        }
      }
      __syncthreads();
    }
    const unsigned U = s_u;
    // 2. FP32 rerank of the unique rows: q . x_c (FalconnPP.cpp:647)
    {
      float4 qc[kMaxChunksPerLane];
      const float* qv = a.Q + (size_t)q * a.d;
#pragma unroll
      for (int i = 0; i < kMaxChunksPerLane; ++i) {
        const int c = lane + 32 * i;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < nchunk) {
          const int j = 4 * c;
          v.x = j < a.d ? qv[j] : 0.f;
          v.y = j + 1 < a.d ? qv[j + 1] : 0.f;
          v.z = j + 2 < a.d ? qv[j + 2] : 0.f;
          v.w = j + 3 < a.d ? qv[j + 3] : 0.f;
        }
        qc[i] = v;
      }
      for (unsigned r = warp; r < U; r += kRrWarps) {
        const uint32_t id = uq[r];
        const float s = warp_dot_rows(qc, nchunk, a.Xc + (size_t)id * a.ld, lane);
        if (lane == 0) sc[r] = __float_as_uint(s);
      }
    }
    __syncthreads();
    if (a.cand_dump) {
      for (unsigned i = tid; i < U; i += kRrThreads) a.cand_dump[(size_t)q * a.cap + i] = (int32_t)uq[i];
    }
    // 3. top-k (FalconnPP.cpp:633-673)
    const unsigned kk = (unsigned)k;
    bool exact = true;
    uint32_t t = 0;
    unsigned nsel = U;
    if (U > kk) {
      if (tid == 0) {
        s_prefix = 0;
        s_remaining = kk;
      }
      uint32_t mask = 0;
      for (int shift = 24; shift >= 0; shift -= 8) {
        hist[tid] = 0;
        __syncthreads();
        const uint32_t pre = s_prefix;
        for (unsigned i = tid; i < U; i += kRrThreads) {
          const uint32_t key = ord_key_bits(sc[i]);
          if ((key & mask) == pre) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (tid == 0) {
          uint32_t rem = s_remaining;
          int dg = 255;
          for (; dg > 0; --dg) {
            if (hist[dg] >= rem) break;
            rem -= hist[dg];
          }
          s_prefix = pre | ((uint32_t)dg << shift);
          s_remaining = rem;
        }
        mask |= 255u << shift;
        __syncthreads();
      }
      t = s_prefix;
      if (tid == 0) {
        s_gt = 0;
        s_ge = 0;
      }
      __syncthreads();
      unsigned gt = 0, ge = 0;
      for (unsigned i = tid; i < U; i += kRrThreads) {
        const uint32_t key = ord_key_bits(sc[i]);
        gt += key > t;
        ge += key >= t;
      }
      atomicAdd(&s_gt, gt);
      atomicAdd(&s_ge, ge);
      __syncthreads();
      exact = (s_ge == kk);
      nsel = kk;
    }
    if (exact) {
      // collect the selected entries and sort them by (score desc, id asc)
      if (tid == 0) s_sel = 0;
      __syncthreads();
      for (unsigned i = tid; i < U; i += kRrThreads) {
        const uint32_t key = ord_key_bits(sc[i]);
        if (U <= kk || key >= t) {
          const unsigned pos = atomicAdd(&s_sel, 1u);
          s_top[pos] = ((unsigned long long)(~key) << 32) | uq[i];
        }
      }
      __syncthreads();
      // bitonic sort of nsel 64-bit keys in shared memory
      int N = 1;
      while (N < (int)nsel) N <<= 1;
      for (int kk2 = 2; kk2 <= N; kk2 <<= 1) {
        for (int j = kk2 >> 1; j > 0; j >>= 1) {
          for (int tt = tid; tt < N / 2; tt += kRrThreads) {
            int lo, hi;
            const int blk = tt / j;
            if (j == (kk2 >> 1)) {
              lo = blk * kk2 + (tt - blk * j);
              hi = blk * kk2 + kk2 - 1 - (tt - blk * j);
            } else {
              lo = blk * 2 * j + (tt - blk * j);
              hi = lo + j;
            }
            if (hi < (int)nsel) {
              const unsigned long long x = s_top[lo], y = s_top[hi];
              if (x > y) {
                s_top[lo] = y;
                s_top[hi] = x;
              }
            }
          }
          __syncthreads();
        }
      }
      // equal scores anywhere in the kept list: the heap order decides
      unsigned dup = 0;
      for (unsigned i = tid; i + 1 < nsel; i += kRrThreads) dup |= (s_top[i] >> 32) == (s_top[i + 1] >> 32);
      exact = !__syncthreads_or(dup);
    }
    int32_t* orow = a.out + (size_t)q * k;
    if (exact) {
      for (int j = tid; j < k; j += kRrThreads) {
        if ((unsigned)j < nsel) {
          orow[j] = (int32_t)(uint32_t)s_top[j];
          if (a.out_v) a.out_v[(size_t)q * k + j] = __uint_as_float(ord_key_inv_dev(~(uint32_t)(s_top[j] >> 32)));
        } else {
          orow[j] = 0;
          if (a.out_v) a.out_v[(size_t)q * k + j] = 0.0f;
        }
      }
    } else {
      // exact replay: ascending-id walk with the reference's min-heap
      if (tid == 0) atomicAdd(a.n_tie, 1);
      block_bitonic_sort_u32(uq, sc, (int)U);
      if (tid == 0) {
        int n = 0;
        for (unsigned i = 0; i < U; ++i) topp_offer<int>(s_hv, s_hi, n, k, __uint_as_float(sc[i]), (int)uq[i]);
        for (int j = n; j < k; ++j) {
          orow[j] = 0;
          if (a.out_v) a.out_v[(size_t)q * k + j] = 0.0f;
        }
        for (int j = n - 1; j >= 0; --j) {  // FalconnPP.cpp:667-673
          orow[j] = s_hi[0];
          if (a.out_v) a.out_v[(size_t)q * k + j] = s_hv[0];
          heap_pop<true, int>(s_hv, s_hi, n);
        }
      }
    }
    if (a.n_unique && tid == 0) a.n_unique[q] = U;
    __syncthreads();
    // 4. clear the bits this query set
    for (unsigned i = tid; i < U; i += kRrThreads) bits[uq[i] >> 5] = 0u;
    __syncthreads();
  }
}

// ------------------------------------------------------------ host side
template <int FHT>
static cudaError_t launch_qhash(const QHashArgs& a, int nsm, float* hv, int* hi, long long max_groups,
                                cudaStream_t s) {
  const size_t smem = QHashSmem<FHT>::bytes;
  cudaError_t e = cudaFuncSetAttribute(k_query_hash<FHT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_query_hash<FHT>, 128, smem);
  if (e != cudaSuccess) return e;
  const long long items = (long long)a.nq * a.L;
  long long grid = std::min<long long>((long long)nsm * std::max(per_sm, 1),
                                       (items + QHashSmem<FHT>::GROUPS - 1) / QHashSmem<FHT>::GROUPS);
  grid = std::min<long long>(grid, max_groups / QHashSmem<FHT>::GROUPS);
  grid = std::max(1LL, grid);
  k_query_hash<FHT><<<(unsigned)grid, 128, smem, s>>>(a, hv, hi);
  return cudaGetLastError();
}

static cudaError_t dispatch_qhash(int fht, const QHashArgs& a, int nsm, float* hv, int* hi, long long max_groups,
                                  cudaStream_t s) {
  switch (fht) {
    case 2: return launch_qhash<2>(a, nsm, hv, hi, max_groups, s);
    case 4: return launch_qhash<4>(a, nsm, hv, hi, max_groups, s);
    case 8: return launch_qhash<8>(a, nsm, hv, hi, max_groups, s);
    case 16: return launch_qhash<16>(a, nsm, hv, hi, max_groups, s);
    case 32: return launch_qhash<32>(a, nsm, hv, hi, max_groups, s);
    case 64: return launch_qhash<64>(a, nsm, hv, hi, max_groups, s);
    case 128: return launch_qhash<128>(a, nsm, hv, hi, max_groups, s);
    case 256: return launch_qhash<256>(a, nsm, hv, hi, max_groups, s);
    case 512: return launch_qhash<512>(a, nsm, hv, hi, max_groups, s);
    case 1024: return launch_qhash<1024>(a, nsm, hv, hi, max_groups, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t hash_lists(const Params& P, const DeviceIndex& di, const float* Q, int nq, const int* q_qprobes, int qp_max,
                       float* list_v, uint32_t* list_b, long long stride, float* heap_v, int* heap_i,
                       long long max_groups, cudaStream_t s) {
  const int L = P.n_tables, D = P.n_proj;
  int log2D = 0;
  while ((1 << log2D) < D) ++log2D;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  QHashArgs qa;
  qa.Q = Q;
  qa.nq = nq;
  qa.d = P.n_features;
  qa.flips = di.flips;
  qa.L = L;
  qa.D = D;
  qa.log2D = log2D;
  qa.NB = 4u * (uint32_t)D * (uint32_t)D;
  qa.m = (2 * qp_max + L - 1) / L;
  int m1 = 0;
  while (m1 * m1 < qa.m) ++m1;
  qa.m1 = m1;
  qa.list_v = list_v;
  qa.list_b = list_b;
  qa.q_qprobes = q_qprobes;
  qa.qp_max = qp_max;
  qa.stride = stride;
  return dispatch_qhash(P.fhtDim, qa, nsm, heap_v, heap_i, max_groups, s);
}

template <typename T>
static cudaError_t ensure(T*& p, size_t& cap_elems, size_t need) {
  if (need <= cap_elems && p) return cudaSuccess;
  cudaFree(p);
  p = nullptr;
  cap_elems = 0;
  const size_t n = std::max<size_t>(need, 1);
  cudaError_t e = fpp::dev_malloc(&p, n * sizeof(T));
  if (e == cudaSuccess) cap_elems = n;
  return e;
}

void QueryWorkspace::release() {
  cudaFree(Qd);
  cudaFree(list_v);
  cudaFree(list_b);
  cudaFree(probes);
  cudaFree(probe_v);
  cudaFree(cand);
  cudaFree(empty);
  cudaFree(n_unique);
  cudaFree(heap_v);
  cudaFree(heap_i);
  cudaFree(bitset);
  cudaFree(uniq);
  cudaFree(score);
  cudaFree(out);
  cudaFree(out_v);
  cudaFree(counters);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  const bool timing = stage_timing;
  *this = QueryWorkspace();
  stage_timing = timing;
}

int query_index(const Params& P, const DeviceIndex& di, const float* Q, bool q_on_device, int nq, int k,
                int32_t* out, bool out_on_device, QueryWorkspace& ws, QueryStats& st, cudaStream_t s,
                Error& err, QueryDumps* dumps) {
  const int L = P.n_tables, D = P.n_proj, d = P.n_features, F = P.fhtDim;
  const uint32_t NB = 4u * (uint32_t)D * (uint32_t)D;
  const int m = (int)ceil(2.0 * P.qProbes / L);  // FalconnPP.cpp:336
  const int m1 = (int)ceil(sqrt(1.0 * m));       // FalconnPP.cpp:337
  int log2D = 0;
  while ((1 << log2D) < D) ++log2D;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int Qp = P.qProbes;
  const long long M = (long long)L * m;
  auto fail = [&](cudaError_t e, const char* what) {
    err.code = (e == cudaErrorMemoryAllocation) ? kErrOutOfMemory : kErrCuda;
    err.msg = std::string(what) + ": " + cudaGetErrorString(e);
    return err.code;
  };
  cudaError_t e;
  st = QueryStats();
  if (nq <= 0) return kOk;

  // inputs
  const float* Qd = Q;
  if (!q_on_device) {
    if ((e = ensure(ws.Qd, ws.cap_Qd, (size_t)nq * d)) != cudaSuccess) return fail(e, "alloc queries");
    if ((e = cudaMemcpyAsync(ws.Qd, Q, sizeof(float) * nq * d, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return fail(e, "copy queries");
    Qd = ws.Qd;
  }
  if ((e = ensure(ws.list_v, ws.cap_list, (size_t)nq * M)) != cudaSuccess) return fail(e, "alloc lists");
  {
    size_t c2 = ws.cap_list_b;
    if ((e = ensure(ws.list_b, c2, (size_t)nq * M)) != cudaSuccess) return fail(e, "alloc lists");
    ws.cap_list_b = c2;
  }
  if ((e = ensure(ws.probes, ws.cap_probes, (size_t)nq * Qp)) != cudaSuccess) return fail(e, "alloc probes");
  if ((e = ensure(ws.cand, ws.cap_cand, (size_t)nq)) != cudaSuccess) return fail(e, "alloc stats");
  if ((e = ensure(ws.empty, ws.cap_empty, (size_t)nq)) != cudaSuccess) return fail(e, "alloc stats");
  if ((e = ensure(ws.n_unique, ws.cap_nu, (size_t)nq)) != cudaSuccess) return fail(e, "alloc stats");
  if ((e = ensure(ws.counters, ws.cap_counters, 4)) != cudaSuccess) return fail(e, "alloc counters");
  if (dumps && dumps->probe_v)
    if ((e = ensure(ws.probe_v, ws.cap_probe_v, (size_t)nq * Qp)) != cudaSuccess) return fail(e, "alloc");
  if (!out_on_device)
    if ((e = ensure(ws.out, ws.cap_out, (size_t)nq * k)) != cudaSuccess) return fail(e, "alloc out");
  if (dumps && dumps->topk_v)
    if ((e = ensure(ws.out_v, ws.cap_out_v, (size_t)nq * k)) != cudaSuccess) return fail(e, "alloc");
  if ((e = cudaMemsetAsync(ws.counters, 0, sizeof(int) * 4, s)) != cudaSuccess) return fail(e, "memset");

  if (ws.stage_timing && !ws.ev[0])
    for (auto& ev : ws.ev)
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail(e, "event create");
  if (ws.stage_timing) cudaEventRecord(ws.ev[0], s);
  // 1. rotate + hash every (query, table)
  {
    // heap scratch: pair heaps of k_query_hash (one per concurrent group) and
    // the replay heaps of k_probe_select (one per block); both allocated here,
    // before any launch, because cudaFree would wait for running kernels
    const long long max_groups = (long long)nsm * 64;
    const int sel_grid = std::min(nq, nsm * 8);
    const size_t need_v = std::max<size_t>((size_t)max_groups * m, (size_t)sel_grid * L);
    const size_t need_i = std::max<size_t>((size_t)max_groups * m, (size_t)sel_grid * 2 * L);
    if ((e = ensure(ws.heap_v, ws.cap_heap_v, need_v)) != cudaSuccess) return fail(e, "alloc heap");
    if ((e = ensure(ws.heap_i, ws.cap_heap_i, need_i)) != cudaSuccess) return fail(e, "alloc heap");
    QHashArgs qa;
    qa.Q = Qd;
    qa.nq = nq;
    qa.d = d;
    qa.flips = di.flips;
    qa.L = L;
    qa.D = D;
    qa.log2D = log2D;
    qa.NB = NB;
    qa.m = m;
    qa.m1 = m1;
    qa.list_v = ws.list_v;
    qa.list_b = ws.list_b;
    qa.q_qprobes = nullptr;
    qa.qp_max = Qp;
    qa.stride = M;
    if ((e = dispatch_qhash(F, qa, nsm, ws.heap_v, ws.heap_i, max_groups, s)) != cudaSuccess)
      return fail(e, "k_query_hash");
  }
  // 2. global probe selection
  {
    const int grid = std::min(nq, nsm * 8);
    float* pv = nullptr;
    if (dumps && dumps->probe_v) pv = ws.probe_v;
    SelectArgs sa;
    sa.list_v = ws.list_v;
    sa.list_b = ws.list_b;
    sa.nq = nq;
    sa.L = L;
    sa.m = m;
    sa.qProbes = Qp;
    sa.bucket_off = di.bucket_off;
    sa.probes = ws.probes;
    sa.probe_v = pv;
    sa.cand = ws.cand;
    sa.empty = ws.empty;
    sa.n_tie = ws.counters + 0;
    if (ws.stage_timing) cudaEventRecord(ws.ev[1], s);
    k_probe_select<<<grid, 256, 0, s>>>(sa, ws.heap_v, ws.heap_i);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "k_probe_select");
    if (ws.stage_timing) cudaEventRecord(ws.ev[2], s);
  }
  // 3. scratch sizing: the largest candidate count of the batch
  std::vector<long long> hcand(nq);
  if ((e = cudaMemcpyAsync(hcand.data(), ws.cand, sizeof(long long) * nq, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fail(e, "copy cand");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "query hash/select");
  long long maxc = 1;
  for (long long c : hcand) {
    maxc = std::max(maxc, c);
    st.total_cand += c;
  }
  const long long cap = std::min<long long>(maxc, P.n_points);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather_rerank, kRrThreads, 0);
  const int grid = std::max(1, std::min(nq, nsm * std::max(1, per_sm)));
  const long long nwords = (P.n_points + 31) / 32;
  if (ws.bitset == nullptr || ws.bitset_grid < grid || ws.bitset_words != nwords) {
    cudaFree(ws.bitset);
    ws.bitset = nullptr;
    if ((e = fpp::dev_malloc(&ws.bitset, sizeof(uint32_t) * (size_t)grid * nwords)) != cudaSuccess)
      return fail(e, "alloc bitset");
    if ((e = cudaMemsetAsync(ws.bitset, 0, sizeof(uint32_t) * (size_t)grid * nwords, s)) != cudaSuccess)
      return fail(e, "memset bitset");
    ws.bitset_grid = grid;
    ws.bitset_words = nwords;
  }
  if ((e = ensure(ws.uniq, ws.cap_uniq, (size_t)grid * cap)) != cudaSuccess) return fail(e, "alloc uniq");
  if ((e = ensure(ws.score, ws.cap_score, (size_t)grid * cap)) != cudaSuccess) return fail(e, "alloc score");
  int32_t* outd = out_on_device ? out : ws.out;
  float* outv = (dumps && dumps->topk_v) ? ws.out_v : nullptr;
  RerankArgs ra;
  ra.probes = ws.probes;
  ra.nq = nq;
  ra.qProbes = Qp;
  ra.k = k;
  ra.bucket_off = di.bucket_off;
  ra.ids = di.ids;
  ra.Xc = di.Xc;
  ra.ld = di.ld;
  ra.Q = Qd;
  ra.d = d;
  ra.n = P.n_points;
  ra.bitset = ws.bitset;
  ra.nwords = nwords;
  ra.uniq = ws.uniq;
  ra.score = ws.score;
  ra.cap = cap;
  ra.out = outd;
  ra.out_v = outv;
  ra.n_unique = ws.n_unique;
  int32_t* cand_dev = nullptr;
  if (dumps && dumps->want_cands) {
    if ((e = fpp::dev_malloc(&cand_dev, sizeof(int32_t) * (size_t)nq * cap)) != cudaSuccess)
      return fail(e, "alloc candidate dump");
    dumps->cand_stride = cap;
  }
  ra.cand_dump = cand_dev;
  ra.n_tie = ws.counters + 1;
  if (ws.stage_timing) cudaEventRecord(ws.ev[3], s);
  k_gather_rerank<<<grid, kRrThreads, 0, s>>>(ra);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "k_gather_rerank");
  if (ws.stage_timing) cudaEventRecord(ws.ev[4], s);
  st.launches = 3;
  if (!out_on_device) {
    if ((e = cudaMemcpyAsync(out, ws.out, sizeof(int32_t) * nq * k, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return fail(e, "copy out");
  }
  std::vector<long long> hu(nq);
  std::vector<int> hempty(nq);
  int hc[4] = {0, 0, 0, 0};
  cudaMemcpyAsync(hu.data(), ws.n_unique, sizeof(long long) * nq, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hempty.data(), ws.empty, sizeof(int) * nq, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hc, ws.counters, sizeof(int) * 4, cudaMemcpyDeviceToHost, s);
  if (dumps) {
    if (dumps->probes) cudaMemcpyAsync(dumps->probes, ws.probes, sizeof(uint32_t) * nq * Qp, cudaMemcpyDeviceToHost, s);
    if (dumps->probe_v) cudaMemcpyAsync(dumps->probe_v, ws.probe_v, sizeof(float) * nq * Qp, cudaMemcpyDeviceToHost, s);
    if (dumps->topk_v) cudaMemcpyAsync(dumps->topk_v, ws.out_v, sizeof(float) * nq * k, cudaMemcpyDeviceToHost, s);
    if (dumps->cand_count) memcpy(dumps->cand_count, hcand.data(), sizeof(long long) * nq);
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
    cudaFree(cand_dev);
    return fail(e, "k_gather_rerank");
  }
  if (cand_dev) {
    dumps->cands.resize((size_t)nq * cap);
    e = cudaMemcpy(dumps->cands.data(), cand_dev, sizeof(int32_t) * (size_t)nq * cap, cudaMemcpyDeviceToHost);
    cudaFree(cand_dev);
    if (e != cudaSuccess) return fail(e, "copy candidate dump");
  }
  for (int i = 0; i < nq; ++i) {
    st.total_unique += hu[i];
    st.total_empty += hempty[i];
  }
  st.total_probes = (long long)nq * Qp;
  if (ws.stage_timing) {
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, ws.ev[0], ws.ev[1]);
    cudaEventElapsedTime(&b, ws.ev[1], ws.ev[2]);
    cudaEventElapsedTime(&c, ws.ev[3], ws.ev[4]);
    st.ms_hash = a;
    st.ms_select = b;
    st.ms_rerank = c;
  }
  st.n_select_ties = hc[0];
  st.n_topk_ties = hc[1];
  if (dumps && dumps->unique_count) memcpy(dumps->unique_count, hu.data(), sizeof(long long) * nq);
  return kOk;
}

}  // namespace fpp
